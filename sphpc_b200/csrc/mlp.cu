// mlp.cu -- tensor-core (tcgen05) kernels of the warm-start network.
//
// One CTA of 128 threads works on tiles of 128 particles.  Each hidden layer
// is one D[128 x 64] = A[128 x K] * W[64 x K]^T product on the tensor cores:
// A (activations) and W (weights) sit in shared memory as K-major BF16 "core
// matrices" (8 rows x 16 bytes, no swizzle), D accumulates in FP32 in tensor
// memory (64 columns), issued by one thread as K/16 tcgen05.mma instructions
// and completed through tcgen05.commit on an mbarrier.  Thread t then owns
// particle t of the tile: it reads row t of D (tcgen05.ld 32x32b), adds the
// bias, applies GELU and writes row t of the next layer's A.
#include <cstring>

#include "host_internal.h"
#include "mlp.cuh"

namespace sphpc {

namespace tc {

// Byte offset of element (r, k) of a K-major tile with KC = K/8 core
// matrices per 8-row group: core matrix (r/8, k/8) is 128 contiguous bytes,
// K-adjacent core matrices 128 bytes apart, 8-row groups KC*128 apart.
__device__ __forceinline__ uint32_t core_off(int r, int k, int kc) {
  return (uint32_t)((((r >> 3) * kc + (k >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

// Shared-memory matrix descriptor (sm_100 UMMA): start, leading-dimension
// byte offset (K direction), stride byte offset (8-row groups), version 1,
// no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: kind::f16, A = B = BF16, D = F32, both K-major,
// M = 128, N = 64.
constexpr uint32_t kIdescM128N64 = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) |
                                   ((128u >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         int accumulate) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(mbar))
               : "memory");
}

// Bounded wait for the mbarrier phase; false after ~1e6 polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity) {
  const uint32_t addr = smem_u32(mbar);
  for (int i = 0; i < (1 << 20); ++i) {
    uint32_t ok;
    asm volatile(
        "{\n.reg .pred P1;\nmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n"
        "selp.b32 %0, 1, 0, P1;\n}\n"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;"); }

// 16 FP32 columns of this warp's 32 lanes.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;"); }

}  // namespace tc

// GELU, tanh form (Hendrycks & Gimpel 2016): 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))).
__device__ __forceinline__ float gelu_tanh(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
  return 0.5f * x * (1.0f + t);
}

namespace {

constexpr uint32_t kErrMlpWait = 1u << 4;

struct MlpSmem {
  alignas(128) uint8_t w1[kMlpHidden * kMlpIn * 2];
  alignas(128) uint8_t w2[kMlpHidden * kMlpHidden * 2];
  alignas(128) uint8_t w3[kMlpHidden * kMlpHidden * 2];
  alignas(128) uint8_t act[kMlpTile * kMlpHidden * 2];
  float b1[kMlpHidden], b2[kMlpHidden], b3[kMlpHidden], w4[kMlpHidden];
  float mean[kMlpIn], istd[kMlpIn];
  alignas(8) uint64_t mbar;
  uint32_t taddr;
};

// Copies a row-major BF16 [64][K] matrix into its core-matrix layout.
__device__ void load_weights(const __nv_bfloat16* __restrict__ w, int K, uint8_t* dst) {
  const int kc = K / 8;
  for (int i = threadIdx.x; i < kMlpHidden * K; i += blockDim.x) {
    const int r = i / K, k = i % K;
    *reinterpret_cast<__nv_bfloat16*>(dst + tc::core_off(r, k, kc)) = w[i];
  }
}

// One layer on the tensor cores: TMEM[128 x 64] = act[128 x K] * W[64 x K]^T.
__device__ __forceinline__ void issue_layer(MlpSmem& s, const uint8_t* w, int K, uint32_t taddr) {
  const int kc = K / 8;
  const uint32_t a0 = tc::smem_u32(s.act), b0 = tc::smem_u32(w);
  for (int step = 0; step < K / 16; ++step) {
    const uint64_t da = tc::smem_desc(a0 + step * 256, 128, kc * 128);
    const uint64_t db = tc::smem_desc(b0 + step * 256, 128, kc * 128);
    tc::mma_bf16(taddr, da, db, tc::kIdescM128N64, step > 0);
  }
  tc::commit(&s.mbar);
}

// Row t of D (64 columns) for this thread's lane.
__device__ __forceinline__ void read_row(uint32_t taddr, float* v) {
  const uint32_t lane_base = taddr + ((uint32_t)((threadIdx.x >> 5) * 32) << 16);
#pragma unroll
  for (int c = 0; c < kMlpHidden; c += 16) tc::tmem_ld16(lane_base + c, v + c);
  tc::tmem_wait_ld();
}

// Row t of the next layer's A (K = 64), BF16.
__device__ __forceinline__ void write_row(MlpSmem& s, const float* h) {
  const int r = threadIdx.x;
#pragma unroll
  for (int k0 = 0; k0 < kMlpHidden; k0 += 8) {
    __align__(16) __nv_bfloat16 pk[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) pk[i] = __float2bfloat16_rn(h[k0 + i]);
    *reinterpret_cast<uint4*>(s.act + tc::core_off(r, k0, kMlpHidden / 8)) =
        *reinterpret_cast<const uint4*>(pk);
  }
}

__global__ void __launch_bounds__(kMlpTile)
    k_mlp_forward(const float* __restrict__ params, const float* __restrict__ norm,
                  const __nv_bfloat16* __restrict__ wbf, const float* __restrict__ feat, int n,
                  float* __restrict__ out, const PD* __restrict__ pd_in, PD* __restrict__ pd_out,
                  uint32_t* __restrict__ err) {
  __shared__ MlpSmem s;
  const int t = threadIdx.x;
  load_weights(wbf, kMlpIn, s.w1);
  load_weights(wbf + kMlpHidden * kMlpIn, kMlpHidden, s.w2);
  load_weights(wbf + kMlpHidden * kMlpIn + kMlpHidden * kMlpHidden, kMlpHidden, s.w3);
  for (int i = t; i < kMlpHidden; i += blockDim.x) {
    s.b1[i] = params[kOffB1 + i];
    s.b2[i] = params[kOffB2 + i];
    s.b3[i] = params[kOffB3 + i];
    s.w4[i] = params[kOffW4 + i];
  }
  if (t < kMlpIn) {
    s.mean[t] = norm[t];
    s.istd[t] = norm[kMlpIn + t];
  }
  const float b4 = params[kOffB4];
  const float out_scale = norm[2 * kMlpIn];
  if (t < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;" ::"r"(
        tc::smem_u32(&s.taddr)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc::smem_u32(&s.mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t taddr = s.taddr;
  uint32_t phase = 0;
  float h[kMlpHidden];
  for (int tile = blockIdx.x; tile * kMlpTile < n; tile += gridDim.x) {
    const int p = tile * kMlpTile + t;
    // input layer operand: normalised features, K = 16
    {
      float f[kMlpIn];
      if (p < n) {
        const float4* fp = reinterpret_cast<const float4*>(feat + (size_t)p * kMlpIn);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 v = __ldg(fp + q);
          f[4 * q] = v.x; f[4 * q + 1] = v.y; f[4 * q + 2] = v.z; f[4 * q + 3] = v.w;
        }
      } else {
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) f[k] = s.mean[k];
      }
#pragma unroll
      for (int k0 = 0; k0 < kMlpIn; k0 += 8) {
        __align__(16) __nv_bfloat16 pk[8];
#pragma unroll
        for (int i = 0; i < 8; ++i)
          pk[i] = __float2bfloat16_rn((f[k0 + i] - s.mean[k0 + i]) * s.istd[k0 + i]);
        *reinterpret_cast<uint4*>(s.act + tc::core_off(t, k0, kMlpIn / 8)) =
            *reinterpret_cast<const uint4*>(pk);
      }
    }
    const uint8_t* layer_w[3] = {s.w1, s.w2, s.w3};
    const float* layer_b[3] = {s.b1, s.b2, s.b3};
    bool ok = true;
#pragma unroll 1
    for (int l = 0; l < 3; ++l) {
      tc::fence_async_smem();
      tc::fence_before();
      __syncthreads();
      if (t == 0) {
        tc::fence_after();
        issue_layer(s, layer_w[l], l == 0 ? kMlpIn : kMlpHidden, taddr);
      }
      // the whole CTA takes the same branch: a wait that gave up anywhere aborts
      ok = __syncthreads_and(tc::mbar_wait(&s.mbar, phase) ? 1 : 0) != 0;
      phase ^= 1u;
      tc::fence_after();
      if (!ok) break;
      read_row(taddr, h);
      const float* b = layer_b[l];
#pragma unroll
      for (int j = 0; j < kMlpHidden; ++j) h[j] = gelu_tanh(h[j] + b[j]);
      // every thread has read D and the MMA has consumed act: act may change
      tc::fence_before();
      __syncthreads();
      if (l < 2) write_row(s, h);
    }
    if (!ok) {
      if (t == 0) atomicOr(err, kErrMlpWait);
      break;
    }
    if (p < n) {
      float y = b4;
#pragma unroll
      for (int j = 0; j < kMlpHidden; ++j) y = fmaf(s.w4[j], h[j], y);
      y *= out_scale;
      if (out) out[p] = y;
      if (pd_out) {
        float4 x, d;
        ld_pd(pd_in, p, x, d);
        d.w = y;
        st_pd(pd_out, p, x, d);
      }
    }
  }
  tc::fence_before();
  __syncthreads();
  if (t < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(taddr));
}

__global__ void k_to_bf16(const float* __restrict__ src, __nv_bfloat16* __restrict__ dst, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = __float2bfloat16_rn(src[i]);
}

}  // namespace

// BF16 copy of W1 | W2 | W3 from the FP32 parameter vector.
static void pack_bf16(const MlpDevice& d, cudaStream_t st) {
  const int n1 = kMlpHidden * kMlpIn, n2 = kMlpHidden * kMlpHidden;
  k_to_bf16<<<(n1 + 255) / 256, 256, 0, st>>>(d.params + kOffW1, d.wbf, n1);
  k_to_bf16<<<(n2 + 255) / 256, 256, 0, st>>>(d.params + kOffW2, d.wbf + n1, n2);
  k_to_bf16<<<(n2 + 255) / 256, 256, 0, st>>>(d.params + kOffW3, d.wbf + n1 + n2, n2);
}

int mlp_upload(MlpDevice& d, const float* params, const float* norm, cudaStream_t st) {
  cudaError_t e = cudaSuccess;
  if (!d.params) e = cudaMalloc(&d.params, sizeof(float) * kMlpParams);
  if (e == cudaSuccess && !d.norm) e = cudaMalloc(&d.norm, sizeof(float) * kMlpNorm);
  if (e == cudaSuccess && !d.wbf)
    e = cudaMalloc(&d.wbf, sizeof(__nv_bfloat16) * (kMlpHidden * kMlpIn + 2 * kMlpHidden * kMlpHidden));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d.params, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d.norm, norm, sizeof(float) * kMlpNorm, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return set_error(SPHPC_ECUDA, "MLP upload: %s", cudaGetErrorString(e));
  pack_bf16(d, st);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(SPHPC_ECUDA, "MLP upload: %s", cudaGetErrorString(e));
  return SPHPC_OK;
}

void mlp_free(MlpDevice& d) {
  if (d.params) cudaFree(d.params);
  if (d.norm) cudaFree(d.norm);
  if (d.wbf) cudaFree(d.wbf);
  d = MlpDevice{};
}

void mlp_release(MlpState& m) {
  mlp_free(m.dev);
  if (m.feat) cudaFree(m.feat);
  if (m.err) cudaFree(m.err);
  m.feat = nullptr;
  m.err = nullptr;
  m.feat_cap = 0;
  m.ready = false;
}

void launch_mlp_forward(const MlpDevice& d, const float* feat, int n, float* out,
                        const PD* pd_in, PD* pd_out, uint32_t* err, cudaStream_t st) {
  if (n <= 0) return;
  const int tiles = (n + kMlpTile - 1) / kMlpTile;
  const int grid = tiles < 148 * 4 ? tiles : 148 * 4;
  k_mlp_forward<<<grid, kMlpTile, 0, st>>>(d.params, d.norm, d.wbf, feat, n, out, pd_in, pd_out,
                                           err);
}

int mlp_warm_start(MlpState& m, const DevParams&, const NbrView&, const PD*, PD*, const float4*,
                   const uint8_t*, cudaStream_t) {
  if (!m.ready) return set_error(SPHPC_ENOTREADY, "warm start: no network loaded");
  return set_error(SPHPC_ENOTREADY, "warm start: features not built yet");
}

}  // namespace sphpc

using namespace sphpc;

// Test entry: forward pass of n feature rows on device memory.
extern "C" int sphpc_mlp_forward(const float* d_feat, int n, const float* params,
                                 const float* norm, float* d_out, void* cuda_stream) {
  if (n < 0 || !params || !norm || (n > 0 && (!d_feat || !d_out)))
    return set_error(SPHPC_EINVAL, "sphpc_mlp_forward: bad arguments");
  cudaStream_t st = (cudaStream_t)cuda_stream;
  MlpDevice d;
  uint32_t* err = nullptr;
  int rc = mlp_upload(d, params, norm, st);
  if (!rc && cudaMalloc(&err, sizeof(uint32_t)) != cudaSuccess)
    rc = set_error(SPHPC_ENOMEM, "sphpc_mlp_forward: error word");
  if (!rc) {
    cudaMemsetAsync(err, 0, sizeof(uint32_t), st);
    launch_mlp_forward(d, d_feat, n, d_out, nullptr, nullptr, err, st);
    uint32_t h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = set_error(SPHPC_ECUDA, "sphpc_mlp_forward: %s", cudaGetErrorString(e));
    else if (h) rc = set_error(SPHPC_EKERNEL, "sphpc_mlp_forward: tensor-core wait gave up (0x%x)", h);
  }
  if (err) cudaFree(err);
  mlp_free(d);
  return rc;
}
