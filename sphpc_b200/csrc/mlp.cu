// mlp.cu -- tensor-core (tcgen05) kernels of the warm-start network.
//
// One CTA of 128 threads works on tiles of 128 particles.  Each hidden layer
// is one D[128 x 64] = A[128 x K] * W[64 x K]^T product on the tensor cores:
// A (activations) and W (weights) sit in shared memory as K-major BF16 "core
// matrices" (8 rows x 16 bytes, no swizzle), D accumulates in FP32 in tensor
// memory (64 columns), issued by one thread as K/16 tcgen05.mma instructions
// and completed through tcgen05.commit on an mbarrier.  Thread t then owns
// particle t of the tile: it reads row t of D (tcgen05.ld 32x32b), adds the
// bias, applies ReLU and writes row t of the next layer's A.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

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

// Instruction descriptor of kind::f16 with A = B = BF16 and D = F32: M x N,
// A and B each K-major (0) or MN-major (1).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
constexpr uint32_t kIdescM128N64 = idesc_bf16(128, 64, 0, 0);

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

// Bounded wait for the mbarrier phase; false after `limit` polls (~1e6 by
// default).
constexpr int kMbarPollLimit = 1 << 20;
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity,
                                          int limit = kMbarPollLimit) {
  const uint32_t addr = smem_u32(mbar);
  for (int i = 0; i < limit; ++i) {
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

// The hidden activation, ReLU: one min/max per element on the FMA pipe, so
// the epilogues between the tensor-core layers cost next to nothing (a
// smooth activation would spend a multi-function-unit op per element, which
// bounds a 64-wide layer well below the tensor cores).
__device__ __forceinline__ float act(float x) { return fmaxf(x, 0.0f); }

namespace {

constexpr uint32_t kErrMlpWait = 1u << 4;

// Shared-memory operand widths (in 8-element core-matrix columns): the input
// rows hold 16 features, a ones column (16) and zeros up to 32; hidden rows
// 64 activations, a ones column (64) and zeros up to 80.  The weight rows
// match: W | bias | 0, so every bias rides in the MMA (as a BF16 value).
constexpr int kKcX = 4, kKcH = 10, kKcD = 16;
constexpr int kKX = kKcX * 8, kKH = kKcH * 8;

// Weight rows [64][kc*8] = W[j][0..K) | bf16(b[j]) | 0 in the core layout.
__device__ void load_weights_ext(const __nv_bfloat16* __restrict__ w,
                                 const float* __restrict__ bias, int K, int kc, uint8_t* dst) {
  // one 16-byte core-matrix row (8 columns) per iteration; K is a multiple of 8
  for (int i = threadIdx.x; i < kMlpHidden * kc; i += blockDim.x) {
    const int r = i / kc, k0 = (i % kc) * 8;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (k0 < K) {
      v = __ldg(reinterpret_cast<const uint4*>(w + r * K + k0));
    } else if (k0 == K) {
      const __nv_bfloat162 b2 = __floats2bfloat162_rn(bias[r], 0.0f);
      v.x = *reinterpret_cast<const uint32_t*>(&b2);
    }
    *reinterpret_cast<uint4*>(dst + tc::core_off(r, k0, kc)) = v;
  }
}

// 8 consecutive values of row r starting at column k0 (multiple of 8), BF16.
__device__ __forceinline__ void put8(uint8_t* buf, int kc, int r, int k0, const float* v) {
  uint32_t w[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    w[i] = *reinterpret_cast<const uint32_t*>(&b2);
  }
  *reinterpret_cast<uint4*>(buf + tc::core_off(r, k0, kc)) = make_uint4(w[0], w[1], w[2], w[3]);
}

__device__ __forceinline__ void put8_const(uint8_t* buf, int kc, int r, int k0, float first) {
  float v[8] = {first, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  put8(buf, kc, r, k0, v);
}

// 64 FP32 columns starting at TMEM column `col` of this thread's lane.
__device__ __forceinline__ void tmem_row64(uint32_t lane_base, uint32_t col, float* v) {
#pragma unroll
  for (int c = 0; c < 64; c += 16) tc::tmem_ld16(lane_base + col + c, v + c);
  tc::tmem_wait_ld();
}

// K-major A [128 x K] x K-major B [N x K]^T, K in steps of 16.
__device__ __forceinline__ void mma_kk(uint32_t d, uint32_t a, int kca, uint32_t b, int kcb, int K,
                                       uint32_t idesc) {
  for (int st = 0; st < K / 16; ++st)
    tc::mma_bf16(d, tc::smem_desc(a + st * 256, 128, kca * 128),
                 tc::smem_desc(b + st * 256, 128, kcb * 128), idesc, st > 0);
}

struct MlpSmem {
  alignas(128) uint8_t w1[kMlpHidden * kKcX * 16];
  alignas(128) uint8_t w2[kMlpHidden * kKcH * 16];
  alignas(128) uint8_t w3[kMlpHidden * kKcH * 16];
  alignas(128) uint8_t x0[kMlpTile * kKcX * 16];
  alignas(128) uint8_t h[kMlpTile * kKcH * 16];
  alignas(16) float w4[kMlpHidden];
  float mean[kMlpIn], istd[kMlpIn];
  alignas(8) uint64_t mbar;
  uint32_t taddr;
};

size_t fwd_smem_bytes() { return sizeof(MlpSmem) + 128; }

// One CTA of 128 threads per tile of 128 rows, tiles strided over the grid;
// thread t owns row t.  Per tile: input row to x0, then three layers, each
// one tcgen05.mma group into tensor memory (64 FP32 columns) followed by the
// row's ReLU epilogue; the last layer's FP32 activations meet w4 on the
// CUDA cores.  BF16_IN: the rows are already the normalised BF16 input (32
// bytes each); otherwise FP32 features normalised here.
template <bool BF16_IN>
__global__ void __launch_bounds__(kMlpTile)
    k_mlp_forward(const float* __restrict__ params, const float* __restrict__ norm,
                  const __nv_bfloat16* __restrict__ wbf, const void* __restrict__ in, int n,
                  float* __restrict__ out, const uint4* __restrict__ rec_in,
                  uint4* __restrict__ rec_out, uint32_t* __restrict__ err, float extra_scale) {
  extern __shared__ __align__(128) uint8_t fwd_raw[];
  const uint32_t mis = tc::smem_u32(fwd_raw) & 127u;
  MlpSmem& s = *reinterpret_cast<MlpSmem*>(fwd_raw + ((128u - mis) & 127u));
  const int t = threadIdx.x;
  load_weights_ext(wbf, params + kOffB1, kMlpIn, kKcX, s.w1);
  load_weights_ext(wbf + kMlpHidden * kMlpIn, params + kOffB2, kMlpHidden, kKcH, s.w2);
  load_weights_ext(wbf + kMlpHidden * kMlpIn + kMlpHidden * kMlpHidden, params + kOffB3,
                   kMlpHidden, kKcH, s.w3);
  for (int i = t; i < kMlpHidden; i += blockDim.x) s.w4[i] = params[kOffW4 + i];
  if (t < kMlpIn) {
    s.mean[t] = norm[t];
    s.istd[t] = norm[kMlpIn + t];
  }
  // constant columns of this thread's rows
  put8_const(s.x0, kKcX, t, 16, 1.0f);
  put8_const(s.x0, kKcX, t, 24, 0.0f);
  put8_const(s.h, kKcH, t, 64, 1.0f);
  put8_const(s.h, kKcH, t, 72, 0.0f);
  const float b4 = params[kOffB4];
  const float out_scale = norm[2 * kMlpIn] * extra_scale;
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
  const uint32_t lane_base = taddr + ((uint32_t)((t >> 5) * 32) << 16);
  const uint32_t sx0 = tc::smem_u32(s.x0), sh = tc::smem_u32(s.h);
  const uint32_t sw[3] = {tc::smem_u32(s.w1), tc::smem_u32(s.w2), tc::smem_u32(s.w3)};
  uint32_t phase = 0;
  bool ok = true;
  float h[kMlpHidden];
  // BF16 rows of the next tile are loaded one tile ahead, so their latency
  // overlaps the current tile's MMA round trips
  uint4 nlo = make_uint4(0, 0, 0, 0), nhi = nlo;
  if (BF16_IN) {
    const int p0 = blockIdx.x * kMlpTile + t;
    if (p0 < n) {
      const uint4* xr = reinterpret_cast<const uint4*>(in) + (size_t)p0 * 2;
      nlo = __ldg(xr);
      nhi = __ldg(xr + 1);
    }
  }
  for (int tile = blockIdx.x; tile * kMlpTile < n; tile += gridDim.x) {
    const int p = tile * kMlpTile + t;
    uint4 rec = make_uint4(0, 0, 0, 0);  // this row's record, read early for the same reason
    if (rec_out && p < n) rec = ld_nr(rec_in, p);
    if (BF16_IN) {
      *reinterpret_cast<uint4*>(s.x0 + tc::core_off(t, 0, kKcX)) = nlo;
      *reinterpret_cast<uint4*>(s.x0 + tc::core_off(t, 8, kKcX)) = nhi;
      const int pn = p + gridDim.x * kMlpTile;
      nlo = make_uint4(0, 0, 0, 0);
      nhi = nlo;
      if (pn < n) {
        const uint4* xr = reinterpret_cast<const uint4*>(in) + (size_t)pn * 2;
        nlo = __ldg(xr);
        nhi = __ldg(xr + 1);
      }
    } else {
      const float* feat = reinterpret_cast<const float*>(in);
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
      for (int k = 0; k < kMlpIn; ++k) f[k] = (f[k] - s.mean[k]) * s.istd[k];
      put8(s.x0, kKcX, t, 0, f);
      put8(s.x0, kKcX, t, 8, f + 8);
    }
#pragma unroll 1
    for (int l = 0; l < 3; ++l) {
      tc::fence_async_smem();
      tc::fence_before();
      __syncthreads();
      if (t == 0) {
        tc::fence_after();
        if (l == 0) mma_kk(taddr, sx0, kKcX, sw[0], kKcX, kKX, tc::kIdescM128N64);
        else mma_kk(taddr, sh, kKcH, sw[l], kKcH, kKH, tc::kIdescM128N64);
        tc::commit(&s.mbar);
      }
      // the whole CTA takes the same branch: a wait that gave up anywhere aborts
      ok = __syncthreads_and(tc::mbar_wait(&s.mbar, phase) ? 1 : 0) != 0;
      phase ^= 1u;
      tc::fence_after();
      if (!ok) break;
      tmem_row64(lane_base, 0, h);
#pragma unroll
      for (int j = 0; j < kMlpHidden; ++j) h[j] = act(h[j]);
      if (l < 2) {
#pragma unroll
        for (int k0 = 0; k0 < kMlpHidden; k0 += 8) put8(s.h, kKcH, t, k0, h + k0);
      }
    }
    if (!ok) {
      if (t == 0) atomicOr(err, kErrMlpWait);
      break;
    }
    if (p < n) {
      float y = b4;
      const float4* w4 = reinterpret_cast<const float4*>(s.w4);
#pragma unroll
      for (int j = 0; j < kMlpHidden / 4; ++j) {
        const float4 w = w4[j];
        y = fmaf(w.x, h[4 * j], y);
        y = fmaf(w.y, h[4 * j + 1], y);
        y = fmaf(w.z, h[4 * j + 2], y);
        y = fmaf(w.w, h[4 * j + 3], y);
      }
      y *= out_scale;
      if (out) out[p] = y;
      if (rec_out) {
        // the record carries lambda_0 of the plain first substep; the target
        // sum_k s_k lambda_k (s_0 = 1, lambda_k <= 0) never exceeds it
        rec.w = __float_as_uint(fminf(y, __uint_as_float(rec.w)));
        rec_out[p] = rec;
      }
    }
  }
  tc::fence_before();
  __syncthreads();
  if (t < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(taddr));
}

// ---------------------------------------------------------------------------
// Training: one batch of rows through forward, backward and the weight
// gradients, all on the tensor cores.  Shared-memory operands (BF16, core
// matrices of 8 rows x 16 bytes, K-adjacent core matrices 128 bytes apart):
//   x0 [128 x 32]  normalised features, column 16 = 1 (bias), rest 0
//   h1, h2, h3 [128 x 80]  activations, column 64 = 1, rest 0
//   dz [128 x 128] the current layer's pre-activation gradient, columns
//                  64..127 = 0
// Forward   z_l  = [h_{l-1} | 1] [W_l | b_l]^T    A, B K-major (bias in the MMA)
// Backward  dh_l = dz_l W_l                 A K-major, B = W_l read MN-major
// Gradient  G_l += dz_l^T [h_{l-1} | 1]     A = dz read MN-major (M = 128 over
//           output neurons, rows 64..127 unused), B = h read MN-major, K =
//           the 128 rows of the tile; column 64 (16 for the input layer) of
//           the result is the bias gradient.
// The gradients accumulate in tensor memory over every tile the CTA takes;
// each CTA writes its sums once, in parameter-vector order, to its slice of
// `partial`; k_mlp_update reduces the slices and applies AdamW.
// Tensor-memory columns (512 allocated, one CTA per SM):
//   z1 0..63, z2 64..127, z3 128..191 (dh2 reuses z3, dh1 reuses z2),
//   G4 192..271, G3 272..351, G2 352..431, G1 432..463.
// ---------------------------------------------------------------------------
constexpr uint32_t kTZ1 = 0, kTZ2 = 64, kTZ3 = 128, kTG4 = 192, kTG3 = 272, kTG2 = 352,
                   kTG1 = 432;
constexpr uint32_t kTrainCols = 512;

struct TrainSmem {
  alignas(1024) uint8_t w1[kMlpHidden * kKcX * 16];
  alignas(128) uint8_t w2[kMlpHidden * kKcH * 16];
  alignas(128) uint8_t w3[kMlpHidden * kKcH * 16];
  alignas(128) uint8_t x0[kMlpTile * kKcX * 16];
  alignas(128) uint8_t h1[kMlpTile * kKcH * 16];
  alignas(128) uint8_t h2[kMlpTile * kKcH * 16];
  alignas(128) uint8_t h3[kMlpTile * kKcH * 16];
  alignas(128) uint8_t dz[kMlpTile * kKcD * 16];
  float w4[kMlpHidden];
  float mean[kMlpIn], istd[kMlpIn];
  float red[kMlpTile / 32];
  // keeps every operand read of the descriptors above inside the CTA's shared
  // memory even if the strides were read with the other core-matrix order
  uint8_t guard[28 * 1024];
  alignas(8) uint64_t mbar;
  uint32_t taddr;
};

size_t train_smem_bytes() { return sizeof(TrainSmem) + 1024; }

// d/dz of act: 1 for z > 0, else 0.
__device__ __forceinline__ float act_grad(float z) { return z > 0.0f ? 1.0f : 0.0f; }

// Weight gradient over the 128 rows of a tile: D[M=128][N] (+)= A^T B with A
// = dz [rows x 128] and B = activations [rows x N], both read MN-major.
__device__ __forceinline__ void mma_grad(uint32_t d, uint32_t a, uint32_t b, int kcb, int N,
                                         bool acc) {
  const uint32_t idesc = tc::idesc_bf16(128, N, 1, 1);
  for (int st = 0; st < kMlpTile / 16; ++st)
    tc::mma_bf16(d, tc::smem_desc(a + st * 2 * kKcD * 128, kKcD * 128, 128),
                 tc::smem_desc(b + st * 2 * kcb * 128, kcb * 128, 128), idesc, acc || st > 0);
}

// dh [128 x 64] = dz [128 x 64] . W [64 x 64] with the weight rows (W | b,
// core layout K-major for the forward, kKcH core columns) read MN-major over
// their first 64 columns.
__device__ __forceinline__ void mma_dh(uint32_t d, uint32_t a, uint32_t w) {
  const uint32_t idesc = tc::idesc_bf16(128, 64, 0, 1);
  for (int st = 0; st < kMlpHidden / 16; ++st)
    tc::mma_bf16(d, tc::smem_desc(a + st * 256, 128, kKcD * 128),
                 tc::smem_desc(w + st * 2 * kKcH * 128, kKcH * 128, 128), idesc, st > 0);
}

__global__ void __launch_bounds__(kMlpTile, 1)
    k_mlp_grad(const float* __restrict__ params, const float* __restrict__ norm,
               const __nv_bfloat16* __restrict__ wbf, const float* __restrict__ feat,
               const float* __restrict__ target, long long n_data, long long base,
               unsigned long long mul, unsigned long long add, int batch,
               float* __restrict__ partial, uint32_t* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  const uint32_t mis = tc::smem_u32(smem_raw) & 1023u;
  TrainSmem& s = *reinterpret_cast<TrainSmem*>(smem_raw + ((1024u - mis) & 1023u));
  const int t = threadIdx.x, warp = t >> 5;
  load_weights_ext(wbf, params + kOffB1, kMlpIn, kKcX, s.w1);
  load_weights_ext(wbf + kMlpHidden * kMlpIn, params + kOffB2, kMlpHidden, kKcH, s.w2);
  load_weights_ext(wbf + kMlpHidden * kMlpIn + kMlpHidden * kMlpHidden, params + kOffB3,
                   kMlpHidden, kKcH, s.w3);
  for (int i = t; i < kMlpHidden; i += blockDim.x) s.w4[i] = params[kOffW4 + i];
  if (t < kMlpIn) {
    s.mean[t] = norm[t];
    s.istd[t] = norm[kMlpIn + t];
  }
  const float b4 = params[kOffB4];
  const float inv_scale = 1.0f / norm[2 * kMlpIn];
  const float inv_batch = 1.0f / (float)batch;
  // constant columns of this thread's rows: bias ones and zero padding
  put8_const(s.x0, kKcX, t, 16, 1.0f);
  put8_const(s.x0, kKcX, t, 24, 0.0f);
  put8_const(s.h1, kKcH, t, 64, 1.0f);
  put8_const(s.h1, kKcH, t, 72, 0.0f);
  put8_const(s.h2, kKcH, t, 64, 1.0f);
  put8_const(s.h2, kKcH, t, 72, 0.0f);
  put8_const(s.h3, kKcH, t, 64, 1.0f);
  put8_const(s.h3, kKcH, t, 72, 0.0f);
  for (int k0 = 64; k0 < 128; k0 += 8) put8_const(s.dz, kKcD, t, k0, 0.0f);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32(&s.taddr)),
                 "r"(kTrainCols));
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
  const uint32_t lane_base = taddr + ((uint32_t)(warp * 32) << 16);
  const uint32_t sx0 = tc::smem_u32(s.x0), sh1 = tc::smem_u32(s.h1), sh2 = tc::smem_u32(s.h2),
                 sh3 = tc::smem_u32(s.h3), sdz = tc::smem_u32(s.dz), sw1 = tc::smem_u32(s.w1),
                 sw2 = tc::smem_u32(s.w2), sw3 = tc::smem_u32(s.w3);
  uint32_t phase = 0;
  bool ok = true, acc = false;
  float loss = 0.0f;
  float v[kMlpHidden];
  // Makes this thread's shared-memory writes visible to the tensor cores,
  // lets thread 0 issue `body` and commit, and waits (bounded) for it; the
  // whole CTA sees the same outcome.
  auto run = [&](auto body) -> bool {
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    if (t == 0) {
      tc::fence_after();
      body();
      tc::commit(&s.mbar);
    }
    const bool done = __syncthreads_and(tc::mbar_wait(&s.mbar, phase) ? 1 : 0) != 0;
    phase ^= 1u;
    tc::fence_after();
    return done;
  };
  const int ntiles = (batch + kMlpTile - 1) / kMlpTile;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int r = tile * kMlpTile + t;
    const bool valid = r < batch;
    float tgt = 0.0f;
    {
      float f[kMlpIn];
      if (valid) {
        const unsigned long long row = (unsigned long long)((base + r) % n_data);
        const unsigned long long idx = (row * mul + add) % (unsigned long long)n_data;
        const float4* fp = reinterpret_cast<const float4*>(feat + idx * kMlpIn);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 a4 = __ldg(fp + q);
          f[4 * q] = a4.x; f[4 * q + 1] = a4.y; f[4 * q + 2] = a4.z; f[4 * q + 3] = a4.w;
        }
        tgt = __ldg(target + idx) * inv_scale;
      } else {
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) f[k] = s.mean[k];
      }
#pragma unroll
      for (int k = 0; k < kMlpIn; ++k) f[k] = (f[k] - s.mean[k]) * s.istd[k];
      put8(s.x0, kKcX, t, 0, f);
      put8(s.x0, kKcX, t, 8, f + 8);
    }
    // forward
    if (!(ok = run([&] { mma_kk(taddr + kTZ1, sx0, kKcX, sw1, kKcX, kKX, tc::kIdescM128N64); })))
      break;
    tmem_row64(lane_base, kTZ1, v);
#pragma unroll
    for (int j = 0; j < kMlpHidden; ++j) v[j] = act(v[j]);
#pragma unroll
    for (int k0 = 0; k0 < kMlpHidden; k0 += 8) put8(s.h1, kKcH, t, k0, v + k0);
    if (!(ok = run([&] { mma_kk(taddr + kTZ2, sh1, kKcH, sw2, kKcH, kKH, tc::kIdescM128N64); })))
      break;
    tmem_row64(lane_base, kTZ2, v);
#pragma unroll
    for (int j = 0; j < kMlpHidden; ++j) v[j] = act(v[j]);
#pragma unroll
    for (int k0 = 0; k0 < kMlpHidden; k0 += 8) put8(s.h2, kKcH, t, k0, v + k0);
    if (!(ok = run([&] { mma_kk(taddr + kTZ3, sh2, kKcH, sw3, kKcH, kKH, tc::kIdescM128N64); })))
      break;
    tmem_row64(lane_base, kTZ3, v);
    float u = b4;
#pragma unroll
    for (int j = 0; j < kMlpHidden; ++j) {
      v[j] = act(v[j]);
      u = fmaf(s.w4[j], v[j], u);
    }
#pragma unroll
    for (int k0 = 0; k0 < kMlpHidden; k0 += 8) put8(s.h3, kKcH, t, k0, v + k0);
    const float res = valid ? u - tgt : 0.0f;
    loss = fmaf(res, res, loss);
    const float g = res * inv_batch;
    // output layer: dz column 0 = g
    put8_const(s.dz, kKcD, t, 0, g);
#pragma unroll
    for (int k0 = 8; k0 < kMlpHidden; k0 += 8) put8_const(s.dz, kKcD, t, k0, 0.0f);
    if (!(ok = run([&] { mma_grad(taddr + kTG4, sdz, sh3, kKcH, 80, acc); }))) break;
    // layer 3
    tmem_row64(lane_base, kTZ3, v);
#pragma unroll
    for (int j = 0; j < kMlpHidden; ++j) v[j] = g * s.w4[j] * act_grad(v[j]);
#pragma unroll
    for (int k0 = 0; k0 < kMlpHidden; k0 += 8) put8(s.dz, kKcD, t, k0, v + k0);
    if (!(ok = run([&] {
          mma_grad(taddr + kTG3, sdz, sh2, kKcH, 80, acc);
          mma_dh(taddr + kTZ3, sdz, sw3);
        })))
      break;
    // layer 2: dz2 = dh2 * act'(z2)
#pragma unroll
    for (int c = 0; c < kMlpHidden; c += 16) {
      float dh[16], z[16];
      tc::tmem_ld16(lane_base + kTZ3 + c, dh);
      tc::tmem_ld16(lane_base + kTZ2 + c, z);
      tc::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 16; ++i) dh[i] *= act_grad(z[i]);
      put8(s.dz, kKcD, t, c, dh);
      put8(s.dz, kKcD, t, c + 8, dh + 8);
    }
    if (!(ok = run([&] {
          mma_grad(taddr + kTG2, sdz, sh1, kKcH, 80, acc);
          mma_dh(taddr + kTZ2, sdz, sw2);
        })))
      break;
    // layer 1
#pragma unroll
    for (int c = 0; c < kMlpHidden; c += 16) {
      float dh[16], z[16];
      tc::tmem_ld16(lane_base + kTZ2 + c, dh);
      tc::tmem_ld16(lane_base + kTZ1 + c, z);
      tc::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 16; ++i) dh[i] *= act_grad(z[i]);
      put8(s.dz, kKcD, t, c, dh);
      put8(s.dz, kKcD, t, c + 8, dh + 8);
    }
    if (!(ok = run([&] { mma_grad(taddr + kTG1, sdz, sx0, kKcX, 32, acc); }))) break;
    acc = true;
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (!ok) {
    if (t == 0) atomicOr(err, kErrMlpWait);
  } else {
    float* out = partial + (size_t)blockIdx.x * (kMlpParams + 1);
    if (warp < 2) {
      const int j = t;  // gradient row = output neuron
#pragma unroll 1
      for (int l = 0; l < 3; ++l) {
        const uint32_t col = l == 0 ? kTG3 : (l == 1 ? kTG2 : kTG1);
        const int ncol = l == 2 ? 32 : 80, nin = l == 2 ? kMlpIn : kMlpHidden;
        const int ow = l == 0 ? kOffW3 : (l == 1 ? kOffW2 : kOffW1);
        const int ob = l == 0 ? kOffB3 : (l == 1 ? kOffB2 : kOffB1);
        for (int c = 0; c < ncol; c += 16) {
          float g16[16];
          tc::tmem_ld16(lane_base + col + c, g16);
          tc::tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int k = c + i;
            if (k < nin) out[ow + j * nin + k] = g16[i];
            else if (k == nin) out[ob + j] = g16[i];
          }
        }
      }
    }
    if (warp == 0) {
      for (int c = 0; c < 80; c += 16) {
        float g16[16];
        tc::tmem_ld16(lane_base + kTG4 + c, g16);
        tc::tmem_wait_ld();
        if (t == 0) {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int k = c + i;
            if (k < kMlpHidden) out[kOffW4 + k] = g16[i];
            else if (k == kMlpHidden) out[kOffB4] = g16[i];
          }
        }
      }
    }
    // sum of squared residuals of the CTA's rows
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if ((t & 31) == 0) s.red[warp] = loss;
    __syncthreads();
    if (t == 0) {
      float tot = 0.0f;
      for (int w = 0; w < kMlpTile / 32; ++w) tot += s.red[w];
      out[kMlpParams] = tot;
    }
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr),
                 "r"(kTrainCols));
}

__device__ __forceinline__ bool mlp_is_weight(int k) {
  return (k >= kOffW1 && k < kOffB1) || (k >= kOffW2 && k < kOffB2) ||
         (k >= kOffW3 && k < kOffB3) || (k >= kOffW4 && k < kOffB4);
}

// Sums the CTAs' gradient slices (FP64, fixed order) and, when m is given,
// applies one AdamW step (decoupled weight decay on weights only) and
// refreshes the BF16 copy of W1..W3.  Slot kMlpParams of each slice is the
// CTA's sum of squared residuals; its total goes to *loss_sum.
__global__ void k_mlp_update(const float* __restrict__ partial, int nparts,
                             float* __restrict__ params, float* __restrict__ m,
                             float* __restrict__ v, __nv_bfloat16* __restrict__ wbf,
                             float* __restrict__ grad_out, float* __restrict__ loss_sum,
                             float lr, float beta1, float beta2, float eps, float wd, float bc1,
                             float bc2) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > kMlpParams) return;
  double g = 0.0;
  for (int c = 0; c < nparts; ++c) g += (double)partial[(size_t)c * (kMlpParams + 1) + k];
  if (k == kMlpParams) {
    if (loss_sum) *loss_sum = (float)g;
    return;
  }
  const float gf = (float)g;
  if (grad_out) grad_out[k] = gf;
  if (!m) return;
  const float mk = beta1 * m[k] + (1.0f - beta1) * gf;
  const float vk = beta2 * v[k] + (1.0f - beta2) * gf * gf;
  m[k] = mk;
  v[k] = vk;
  float p = params[k];
  const float upd = (mk * bc1) / (sqrtf(vk * bc2) + eps) + (mlp_is_weight(k) ? wd * p : 0.0f);
  p -= lr * upd;
  params[k] = p;
  const int n1 = kMlpHidden * kMlpIn, n2 = kMlpHidden * kMlpHidden;
  if (k < kOffB1) wbf[k] = __float2bfloat16_rn(p);
  else if (k >= kOffW2 && k < kOffB2) wbf[n1 + (k - kOffW2)] = __float2bfloat16_rn(p);
  else if (k >= kOffW3 && k < kOffB3) wbf[n1 + n2 + (k - kOffW3)] = __float2bfloat16_rn(p);
}

// Per-column FP64 sums and sums of squares of feat[n][16] and target[n]
// (17 columns) for the normalisation.
__global__ void k_mlp_moments(const float* __restrict__ feat, const float* __restrict__ target,
                              long long n, double* __restrict__ acc) {
  double s[17], q[17];
#pragma unroll
  for (int c = 0; c < 17; ++c) s[c] = q[c] = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float4* fp = reinterpret_cast<const float4*>(feat + i * kMlpIn);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float4 a = __ldg(fp + k);
      const float e[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        s[4 * k + c] += e[c];
        q[4 * k + c] += (double)e[c] * e[c];
      }
    }
    const double tv = __ldg(target + i);
    s[16] += tv;
    q[16] += tv * tv;
  }
#pragma unroll
  for (int c = 0; c < 17; ++c) {
    double a = s[c], b = q[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(acc + c, a);
      atomicAdd(acc + 17 + c, b);
    }
  }
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

static int set_mlp_attrs();

// Uploads the parameters and the normalisation, and readies the network's
// kernels on this device (their shared-memory opt-in, which also makes the
// runtime load them), so that the first step that runs the network does not
// pay for that.
int mlp_upload(MlpDevice& d, const float* params, const float* norm, cudaStream_t st) {
  SPHPC_RC(set_mlp_attrs());
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

// Opts the MLP kernels into their dynamic shared memory (once per device).
static int set_mlp_attrs() {
  static int done_mask = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 32 && (done_mask >> dev & 1)) return SPHPC_OK;
  cudaError_t e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)train_smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_mlp_forward<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)fwd_smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_mlp_forward<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)fwd_smem_bytes());
  if (e != cudaSuccess) return set_error(SPHPC_ECUDA, "MLP kernel attributes: %s", cudaGetErrorString(e));
  if (dev < 32) done_mask |= 1 << dev;
  return SPHPC_OK;
}

void launch_mlp_forward(const MlpDevice& d, const float* feat, int n, float* out,
                        const uint4* rec_in, uint4* rec_out, uint32_t* err, cudaStream_t st,
                        float extra_scale) {
  if (n <= 0 || set_mlp_attrs() != SPHPC_OK) return;
  const int tiles = (n + kMlpTile - 1) / kMlpTile;
  const int grid = tiles < 148 * 4 ? tiles : 148 * 4;
  k_mlp_forward<false><<<grid, kMlpTile, fwd_smem_bytes(), st>>>(d.params, d.norm, d.wbf, feat, n, out, rec_in,
                                                  rec_out, err, extra_scale);
}

void launch_mlp_forward_bf16(const MlpDevice& d, const __nv_bfloat16* xbf, int n,
                             const uint4* rec_in, uint4* rec_out, uint32_t* err, cudaStream_t st,
                             float extra_scale) {
  if (n <= 0 || set_mlp_attrs() != SPHPC_OK) return;
  const int tiles = (n + kMlpTile - 1) / kMlpTile;
  const int grid = tiles < 148 * 4 ? tiles : 148 * 4;
  k_mlp_forward<true><<<grid, kMlpTile, fwd_smem_bytes(), st>>>(d.params, d.norm, d.wbf, xbf, n, nullptr, rec_in,
                                                 rec_out, err, extra_scale);
}

// ---- device-resident training set (one per process, on the device that
// made it) ----
namespace {
struct MlpDataset {
  float* feat = nullptr;    // [cap][16]
  float* target = nullptr;  // [cap]
  long long n = 0, cap = 0;
  int device = -1;
};
MlpDataset g_ds;
std::mutex g_ds_mu;

int dataset_check_device() {
  int dev = -1;
  cudaGetDevice(&dev);
  if (g_ds.cap > 0 && dev != g_ds.device)
    return set_error(SPHPC_EINVAL, "training set lives on device %d, current device is %d",
                     g_ds.device, dev);
  return SPHPC_OK;
}

int train_grid(int batch) {
  const int tiles = (batch + kMlpTile - 1) / kMlpTile;
  return tiles < 148 ? tiles : 148;
}

// Scratch of a gradient/AdamW run.
struct TrainBufs {
  float* partial = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  float* grad = nullptr;
  float* loss = nullptr;
  uint32_t* err = nullptr;
  ~TrainBufs() {
    if (partial) cudaFree(partial);
    if (m) cudaFree(m);
    if (v) cudaFree(v);
    if (grad) cudaFree(grad);
    if (loss) cudaFree(loss);
    if (err) cudaFree(err);
  }
};

uint64_t splitmix64(uint64_t& x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

uint64_t gcd_u64(uint64_t a, uint64_t b) {
  while (b) {
    const uint64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}
}  // namespace

int mlp_dataset_claim(long long want, float** feat, float** target, long long* got) {
  std::lock_guard<std::mutex> lk(g_ds_mu);
  *got = 0;
  if (g_ds.cap == 0) return set_error(SPHPC_ENOTREADY, "no training set reserved");
  SPHPC_RC(dataset_check_device());
  const long long room = g_ds.cap - g_ds.n;
  *got = want < room ? want : room;
  *feat = g_ds.feat + g_ds.n * kMlpIn;
  *target = g_ds.target + g_ds.n;
  g_ds.n += *got;
  return SPHPC_OK;
}

namespace {

// Failure-detection check of the bounded mbarrier wait of the tensor-core
// kernels: an mbarrier that nothing ever arrives on, waited on through the
// same helper with a poll limit of `limit`.  The block decides together, as
// the kernels do, and records kErrMlpWait when the wait gave up.
__global__ void k_mbar_wait_probe(int limit, uint32_t* err) {
  __shared__ __align__(8) uint64_t mbar;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc::smem_u32(&mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  __syncthreads();
  const bool done = __syncthreads_and(tc::mbar_wait(&mbar, 0, limit) ? 1 : 0) != 0;
  if (!done && threadIdx.x == 0) atomicOr(err, kErrMlpWait);
  __syncthreads();
  if (threadIdx.x == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(tc::smem_u32(&mbar)));
}

}  // namespace

cudaError_t mbar_wait_probe(int limit, uint32_t* err_bits) {
  uint32_t* err = nullptr;
  cudaError_t e = cudaMalloc(&err, sizeof(uint32_t));
  if (e != cudaSuccess) return e;
  e = cudaMemset(err, 0, sizeof(uint32_t));
  if (e == cudaSuccess) {
    k_mbar_wait_probe<<<1, 128>>>(limit, err);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(err_bits, err, sizeof(uint32_t), cudaMemcpyDeviceToHost);
  cudaFree(err);
  return e;
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

// Gradient of the batch loss L = 1/(2n) sum (u - t/out_scale)^2 over n rows
// of device memory, through the training kernels; grad_out[9473] and
// *loss_out on the host.
extern "C" int sphpc_mlp_grad(const float* d_feat, const float* d_target, int n,
                              const float* params, const float* norm, float* grad_out,
                              float* loss_out, void* cuda_stream) {
  if (n <= 0 || !d_feat || !d_target || !params || !norm || !grad_out)
    return set_error(SPHPC_EINVAL, "sphpc_mlp_grad: bad arguments");
  cudaStream_t st = (cudaStream_t)cuda_stream;
  SPHPC_RC(set_mlp_attrs());
  MlpDevice d;
  TrainBufs b;
  int rc = mlp_upload(d, params, norm, st);
  const int grid = train_grid(n);
  if (!rc && (cudaMalloc(&b.partial, sizeof(float) * (size_t)grid * (kMlpParams + 1)) != cudaSuccess ||
              cudaMalloc(&b.grad, sizeof(float) * kMlpParams) != cudaSuccess ||
              cudaMalloc(&b.loss, sizeof(float)) != cudaSuccess ||
              cudaMalloc(&b.err, sizeof(uint32_t)) != cudaSuccess))
    rc = set_error(SPHPC_ENOMEM, "sphpc_mlp_grad: scratch");
  if (!rc) {
    cudaMemsetAsync(b.err, 0, sizeof(uint32_t), st);
    k_mlp_grad<<<grid, kMlpTile, train_smem_bytes(), st>>>(d.params, d.norm, d.wbf, d_feat, d_target,
                                                         n, 0, 1, 0, n, b.partial, b.err);
    k_mlp_update<<<(kMlpParams + 256) / 256, 256, 0, st>>>(b.partial, grid, nullptr, nullptr, nullptr,
                                                          nullptr, b.grad, b.loss, 0.f, 0.f, 0.f,
                                                          0.f, 0.f, 0.f, 0.f);
    uint32_t h = 0;
    float ls = 0.0f;
    cudaError_t e = cudaMemcpyAsync(grad_out, b.grad, sizeof(float) * kMlpParams,
                                    cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&ls, b.loss, sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, b.err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = set_error(SPHPC_ECUDA, "sphpc_mlp_grad: %s", cudaGetErrorString(e));
    else if (h) rc = set_error(SPHPC_EKERNEL, "sphpc_mlp_grad: tensor-core wait gave up (0x%x)", h);
    if (!rc && loss_out) *loss_out = ls / (2.0f * (float)n);
  }
  mlp_free(d);
  return rc;
}

extern "C" int sphpc_mlp_dataset_reserve(long long capacity) {
  std::lock_guard<std::mutex> lk(g_ds_mu);
  if (capacity <= 0 || capacity > (1ll << 31))
    return set_error(SPHPC_EINVAL, "sphpc_mlp_dataset_reserve: capacity %lld out of (0, 2^31]",
                     capacity);
  if (g_ds.cap > 0) SPHPC_RC(dataset_check_device());
  if (capacity <= g_ds.cap) return SPHPC_OK;
  float *f = nullptr, *t = nullptr;
  if (cudaMalloc(&f, sizeof(float) * kMlpIn * (size_t)capacity) != cudaSuccess ||
      cudaMalloc(&t, sizeof(float) * (size_t)capacity) != cudaSuccess) {
    if (f) cudaFree(f);
    cudaGetLastError();
    return set_error(SPHPC_ENOMEM, "sphpc_mlp_dataset_reserve: %lld rows", capacity);
  }
  if (g_ds.n > 0) {
    cudaMemcpy(f, g_ds.feat, sizeof(float) * kMlpIn * (size_t)g_ds.n, cudaMemcpyDeviceToDevice);
    cudaMemcpy(t, g_ds.target, sizeof(float) * (size_t)g_ds.n, cudaMemcpyDeviceToDevice);
  }
  if (g_ds.feat) cudaFree(g_ds.feat);
  if (g_ds.target) cudaFree(g_ds.target);
  g_ds.feat = f;
  g_ds.target = t;
  g_ds.cap = capacity;
  cudaGetDevice(&g_ds.device);
  return SPHPC_OK;
}

extern "C" int sphpc_mlp_dataset_size(long long* n) {
  if (!n) return set_error(SPHPC_EINVAL, "sphpc_mlp_dataset_size: null");
  std::lock_guard<std::mutex> lk(g_ds_mu);
  *n = g_ds.n;
  return SPHPC_OK;
}

extern "C" int sphpc_mlp_dataset_clear(void) {
  std::lock_guard<std::mutex> lk(g_ds_mu);
  g_ds.n = 0;
  return SPHPC_OK;
}

extern "C" int sphpc_mlp_dataset_free(void) {
  std::lock_guard<std::mutex> lk(g_ds_mu);
  if (g_ds.feat) cudaFree(g_ds.feat);
  if (g_ds.target) cudaFree(g_ds.target);
  g_ds = MlpDataset{};
  return SPHPC_OK;
}

// Appends rows from host memory (feat[count][16], target[count]).
extern "C" int sphpc_mlp_dataset_append(const float* feat, const float* target, long long count) {
  if (count < 0 || (count > 0 && (!feat || !target)))
    return set_error(SPHPC_EINVAL, "sphpc_mlp_dataset_append: bad arguments");
  float *f = nullptr, *t = nullptr;
  long long got = 0;
  SPHPC_RC(mlp_dataset_claim(count, &f, &t, &got));
  if (got < count)
    return set_error(SPHPC_ENOMEM, "sphpc_mlp_dataset_append: %lld of %lld rows fit", got, count);
  cudaError_t e = cudaMemcpy(f, feat, sizeof(float) * kMlpIn * (size_t)count, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(t, target, sizeof(float) * (size_t)count, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return set_error(SPHPC_ECUDA, "sphpc_mlp_dataset_append: %s", cudaGetErrorString(e));
  return SPHPC_OK;
}

// Copies rows [offset, offset + count) to host memory.
extern "C" int sphpc_mlp_dataset_read(long long offset, long long count, float* feat, float* target) {
  std::lock_guard<std::mutex> lk(g_ds_mu);
  if (offset < 0 || count < 0 || offset + count > g_ds.n)
    return set_error(SPHPC_EINVAL, "sphpc_mlp_dataset_read: rows [%lld, %lld) outside [0, %lld)",
                     offset, offset + count, g_ds.n);
  cudaError_t e = cudaSuccess;
  if (feat)
    e = cudaMemcpy(feat, g_ds.feat + offset * kMlpIn, sizeof(float) * kMlpIn * (size_t)count,
                   cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && target)
    e = cudaMemcpy(target, g_ds.target + offset, sizeof(float) * (size_t)count, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_error(SPHPC_ECUDA, "sphpc_mlp_dataset_read: %s", cudaGetErrorString(e));
  return SPHPC_OK;
}

// Normalisation of the training set: norm[0..15] = feature means,
// norm[16..31] = 1 / standard deviations (1 for a constant feature),
// norm[32] = standard deviation of the targets (1 if constant).
extern "C" int sphpc_mlp_dataset_stats(float* norm) {
  if (!norm) return set_error(SPHPC_EINVAL, "sphpc_mlp_dataset_stats: null");
  std::lock_guard<std::mutex> lk(g_ds_mu);
  if (g_ds.n < 2) return set_error(SPHPC_ENOTREADY, "sphpc_mlp_dataset_stats: fewer than 2 rows");
  SPHPC_RC(dataset_check_device());
  double* acc = nullptr;
  if (cudaMalloc(&acc, sizeof(double) * 34) != cudaSuccess)
    return set_error(SPHPC_ENOMEM, "sphpc_mlp_dataset_stats: scratch");
  cudaMemset(acc, 0, sizeof(double) * 34);
  k_mlp_moments<<<148 * 4, 256>>>(g_ds.feat, g_ds.target, g_ds.n, acc);
  double h[34];
  const cudaError_t e = cudaMemcpy(h, acc, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(acc);
  if (e != cudaSuccess) return set_error(SPHPC_ECUDA, "sphpc_mlp_dataset_stats: %s", cudaGetErrorString(e));
  const double nn = (double)g_ds.n;
  for (int c = 0; c < 17; ++c) {
    const double mean = h[c] / nn;
    const double var = std::max(h[17 + c] / nn - mean * mean, 0.0);
    const double sd = std::sqrt(var);
    if (c < kMlpIn) {
      norm[c] = (float)mean;
      norm[kMlpIn + c] = sd > 1e-12 * std::max(1.0, std::fabs(mean)) ? (float)(1.0 / sd) : 1.0f;
    } else {
      norm[2 * kMlpIn] = sd > 0.0 ? (float)sd : 1.0f;
    }
  }
  return SPHPC_OK;
}

// AdamW training on the training set: `steps` steps of `batch` rows drawn
// without replacement within each pass over the set (a fresh affine
// permutation of the row indices per pass, seeded by `seed`), learning rate
// from lr down to lr_final on a half cosine (lr_final = lr: constant),
// decoupled weight decay on the weights, beta = (0.9, 0.999), eps 1e-8.
// params_out[9473] receives the trained parameters; loss_out[steps], if
// given, the batch loss of every step (before its update).
extern "C" int sphpc_mlp_train(const float* params_in, const float* norm, int steps, int batch,
                               float lr, float lr_final, float weight_decay,
                               unsigned long long seed, float* params_out, float* loss_out) {
  if (!params_in || !norm || !params_out || steps < 0 || batch <= 0 || !(lr > 0.0f) ||
      !(lr_final >= 0.0f) || weight_decay < 0.0f)
    return set_error(SPHPC_EINVAL, "sphpc_mlp_train: bad arguments");
  long long N = 0;
  float *feat = nullptr, *target = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_ds_mu);
    N = g_ds.n;
    feat = g_ds.feat;
    target = g_ds.target;
    if (N > 0) SPHPC_RC(dataset_check_device());
  }
  if (N < 1) return set_error(SPHPC_ENOTREADY, "sphpc_mlp_train: empty training set");
  SPHPC_RC(set_mlp_attrs());
  cudaStream_t st = 0;
  MlpDevice d;
  TrainBufs b;
  int rc = mlp_upload(d, params_in, norm, st);
  const int grid = train_grid(batch);
  if (!rc && (cudaMalloc(&b.partial, sizeof(float) * (size_t)grid * (kMlpParams + 1)) != cudaSuccess ||
              cudaMalloc(&b.m, sizeof(float) * kMlpParams) != cudaSuccess ||
              cudaMalloc(&b.v, sizeof(float) * kMlpParams) != cudaSuccess ||
              cudaMalloc(&b.loss, sizeof(float) * (size_t)(steps > 0 ? steps : 1)) != cudaSuccess ||
              cudaMalloc(&b.err, sizeof(uint32_t)) != cudaSuccess))
    rc = set_error(SPHPC_ENOMEM, "sphpc_mlp_train: scratch");
  if (rc) {
    mlp_free(d);
    return rc;
  }
  cudaMemsetAsync(b.m, 0, sizeof(float) * kMlpParams, st);
  cudaMemsetAsync(b.v, 0, sizeof(float) * kMlpParams, st);
  cudaMemsetAsync(b.err, 0, sizeof(uint32_t), st);
  const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
  uint64_t rng = seed;
  long long epoch = -1;
  unsigned long long mul = 1, add = 0;
  for (int k = 1; k <= steps; ++k) {
    const long long first = (long long)(k - 1) * batch;
    const long long e = first / N;
    if (e != epoch) {
      epoch = e;
      if (N > 1) {
        do {
          mul = 1 + splitmix64(rng) % (uint64_t)(N - 1);
        } while (gcd_u64(mul, (uint64_t)N) != 1);
      }
      add = splitmix64(rng) % (uint64_t)N;
    }
    k_mlp_grad<<<grid, kMlpTile, train_smem_bytes(), st>>>(d.params, d.norm, d.wbf, feat, target, N,
                                                         first % N, mul, add, batch, b.partial,
                                                         b.err);
    // cosine from lr to lr_final over the run
    const double frac = steps > 1 ? (double)(k - 1) / (double)(steps - 1) : 0.0;
    const float lr_k = (float)(lr_final + 0.5 * (lr - lr_final) * (1.0 + std::cos(M_PI * frac)));
    const float bc1 = (float)(1.0 / (1.0 - std::pow((double)beta1, (double)k)));
    const float bc2 = (float)(1.0 / (1.0 - std::pow((double)beta2, (double)k)));
    k_mlp_update<<<(kMlpParams + 256) / 256, 256, 0, st>>>(b.partial, grid, d.params, b.m, b.v,
                                                          d.wbf, nullptr, b.loss + (k - 1), lr_k,
                                                          beta1, beta2, eps, weight_decay, bc1,
                                                          bc2);
  }
  uint32_t h = 0;
  cudaError_t ce = cudaMemcpyAsync(params_out, d.params, sizeof(float) * kMlpParams,
                                   cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess && loss_out && steps > 0)
    ce = cudaMemcpyAsync(loss_out, b.loss, sizeof(float) * steps, cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(&h, b.err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  if (ce != cudaSuccess) rc = set_error(SPHPC_ECUDA, "sphpc_mlp_train: %s", cudaGetErrorString(ce));
  else if (h) rc = set_error(SPHPC_EKERNEL, "sphpc_mlp_train: tensor-core wait gave up (0x%x)", h);
  if (!rc && loss_out)
    for (int k = 0; k < steps; ++k) loss_out[k] /= 2.0f * (float)batch;
  mlp_free(d);
  return rc;
}
