// mlp.cuh -- learned warm start of the constraint solve.
//
// A per-particle MLP maps 16 neighbourhood features to an effective
// multiplier lambda0 whose single position pass moves x* close to where the
// plain constraint iterations would take it.  Network: 16 -> 64 -> 64 -> 64
// (ReLU) -> 1; BF16 weights and activations on the 5th-generation
// tensor cores (tcgen05.mma, FP32 accumulators in tensor memory), FP32 last
// layer.  Parameter vector (FP32, 9473 values):
//   W1[64][16] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] w4[64] b4
// plus a fixed normalisation (not trained): mean[16] inv_std[16] out_scale.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "sphpc_dev.cuh"

namespace sphpc {

constexpr int kMlpIn = 16;
constexpr int kMlpHidden = 64;
constexpr int kMlpParams = kMlpHidden * kMlpIn + kMlpHidden + 2 * (kMlpHidden * kMlpHidden + kMlpHidden) +
                           kMlpHidden + 1;  // 9473
constexpr int kMlpNorm = 2 * kMlpIn + 1;     // mean, inv_std, out_scale
constexpr int kMlpTile = 128;                // particles per tensor-core tile (M)

// Offsets into the parameter vector.
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpHidden * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpHidden;
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;
constexpr int kOffW3 = kOffB2 + kMlpHidden;
constexpr int kOffB3 = kOffW3 + kMlpHidden * kMlpHidden;
constexpr int kOffW4 = kOffB3 + kMlpHidden;
constexpr int kOffB4 = kOffW4 + kMlpHidden;

// Device copy of a network: FP32 parameters and normalisation, and the
// BF16 weight matrices W1, W2, W3 (row-major [out][in]).
struct MlpDevice {
  float* params = nullptr;         // kMlpParams
  float* norm = nullptr;           // kMlpNorm
  __nv_bfloat16* wbf = nullptr;    // W1 | W2 | W3 in BF16
};

struct MlpState {
  bool ready = false;
  MlpDevice dev;
  float* feat = nullptr;           // [n][16] features of the current step
  int feat_cap = 0;
  uint32_t* err = nullptr;         // error bits of the MLP kernels
};

void mlp_release(MlpState& m);

// Uploads host parameters/normalisation into m.dev (allocating on first use).
int mlp_upload(MlpDevice& d, const float* params, const float* norm, cudaStream_t st);
void mlp_free(MlpDevice& d);

// Forward pass of n feature rows feat[n][16] -> out[n] (lambda0), or when
// rec_in/rec_out are given, 16-byte neighbour records rec_out[p] = rec_in[p]
// with the payload min(Lambda, rec_in[p] payload): the input records carry
// the plain first multiplier lambda_0 <= 0, and the target sum_k s_k lambda_k
// (s_0 = 1, every lambda_k <= 0) never exceeds it.
void launch_mlp_forward(const MlpDevice& d, const float* feat, int n, float* out,
                        const uint4* rec_in, uint4* rec_out, uint32_t* err, cudaStream_t st,
                        float extra_scale = 1.0f);

// The same from rows already normalised to BF16 (xbf[n][16]) into records.
void launch_mlp_forward_bf16(const MlpDevice& d, const __nv_bfloat16* xbf, int n,
                             const uint4* rec_in, uint4* rec_out, uint32_t* err, cudaStream_t st,
                             float extra_scale = 1.0f);

// Reserves `want` rows of the process's training set (fewer when it is
// nearly full: *got) and returns their feature and target pointers.
int mlp_dataset_claim(long long want, float** feat, float** target, long long* got);

// Failure-detection check of the bounded mbarrier wait: one block waits,
// with a poll limit of `limit`, on an mbarrier that nothing arrives on;
// returns the error bits it raised (kErrMlpWait, 1 << 4, when it gave up).
cudaError_t mbar_wait_probe(int limit, uint32_t* err_bits);

}  // namespace sphpc
