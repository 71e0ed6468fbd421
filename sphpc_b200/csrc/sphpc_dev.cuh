// sphpc_dev.cuh -- device-side layout, parameters and shared primitives of
// the B200 PBF pipeline.
//
// State layout in HBM (slot order = particles sorted by uniform-grid cell
// key, rebuilt every step):
//   pd[n]    PD      32-byte record {x, d}: x the step-start position (.w
//                    unused), d = x* - x the predicted-position displacement
//                    (.w carries lambda after the density/lambda pass and the
//                    density after the position pass).  A neighbour's record
//                    is one 256-bit load.
//   nr[n]    uint4   16-byte neighbour record {X, Y, Z, w}: x* in fixed
//                    point (2^-k units, wrapping mod 2^32, so the difference
//                    of two records is exact for any box) and a payload (w:
//                    lambda after a density/lambda pass, the density after
//                    a position pass).  Neighbour sums gather only these.
//   xsa[n]   float4  x* as absolute FP32 (neighbour-build candidate test),
//                    in pair blocks: slots 2b, 2b+1 share {x0, x1, y0, y1},
//                    {z0, z1, 0, 0} at float4 index 2b
//   vel[n]   float4  v
//   ids[n]   u32     original particle index of each slot
//   cellp[n] u32     packed grid cell (cx | cy<<bx | cz<<(bx+by)) of x* at
//                    neighbour-build time
//   nbr4[15][n] uint4  neighbour slots of every particle in the reference's
//                    bucket order, four per block (block b of all particles
//                    contiguous, so a warp reads four 128-byte lines per
//                    block); the last block's entries past the count are p
//                    (nbr_entry, nbr_block)
//   ncount[n] u8     bucket sizes
//   cstart[C+1] u32  start slot of every cell (lower bound), cstart[C] = n
//
// The canonical predicted position is the double fl64(x + d): the hash, the
// neighbour test, the box clamp and the SDF lookup are evaluated on it in
// FP64 exactly as the reference evaluates its double x_star.  Pair
// differences inside the neighbour sums are integer differences of the
// fixed-point records (2^-k units, k = 28 - ceil(log2 h): 7.5e-9 for h = 2)
// converted to FP32, so their precision does not depend on the box size.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sphpc {

constexpr int kMaxNeighbors = 60;   // MAX_NEIGHBORS, neighbors.h:6

// 32-byte record for the post-solve passes that gather a second quantity of
// each neighbour: the 16-byte neighbour record r = {X, Y, Z, w} and a float4
// e (colour gradient, or velocity), so a neighbour costs one 256-bit gather
// instead of two 128-bit ones.
struct __align__(32) NV {
  uint4 r;
  float4 e;
};

// Position record of one particle: step-start x and displacement d = x* - x.
struct __align__(32) PD {
  float4 x;
  float4 d;
};

// Packed FP32x2 (sm_100): two independent IEEE single-precision operations
// per instruction, each rounded to nearest as its scalar form.
__device__ __forceinline__ uint64_t f2_dup(float a) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %1};" : "=l"(r) : "f"(a));
  return r;
}
__device__ __forceinline__ uint64_t f2_sub(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t f2_mul(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t f2_fma(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
__device__ __forceinline__ float f2_lo(uint64_t a) { return __uint_as_float((uint32_t)a); }
__device__ __forceinline__ float f2_hi(uint64_t a) { return __uint_as_float((uint32_t)(a >> 32)); }

// One 256-bit read-only load of a record (ld.global.nc.v8.f32, sm_100).
__device__ __forceinline__ void ld_pd(const PD* __restrict__ base, int i, float4& x, float4& d) {
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(x.x), "=f"(x.y), "=f"(x.z), "=f"(x.w), "=f"(d.x), "=f"(d.y), "=f"(d.z), "=f"(d.w)
      : "l"(base + i));
}

__device__ __forceinline__ void st_pd(PD* base, int i, const float4 x, const float4 d) {
  asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(base + i),
               "f"(x.x), "f"(x.y), "f"(x.z), "f"(x.w), "f"(d.x), "f"(d.y), "f"(d.z), "f"(d.w)
               : "memory");
}

// 16-byte neighbour record: fixed-point x* and a payload, one 128-bit load.
__device__ __forceinline__ uint4 ld_nr(const uint4* __restrict__ base, int i) {
  uint4 r;
  asm("ld.global.nc.v4.u32 {%0,%1,%2,%3}, [%4];"
      : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
      : "l"(base + i));
  return r;
}

__device__ __forceinline__ float nr_w(const uint4 r) { return __uint_as_float(r.w); }

// |(x, y, z)|^2 as fma(z, z, fma(y, y, x x)).  The neighbour sums spell out
// every fused multiply-add (fmaf) and every product or sum that must not be
// fused (__fmul_rn, __fadd_rn), so their rounding is the same in every build
// of the library, whatever contractions the compiler would choose.
__device__ __forceinline__ float norm2(float x, float y, float z) {
  return fmaf(z, z, fmaf(y, y, __fmul_rn(x, x)));
}

// Error bits raised by kernels (host reads them back).
enum : uint32_t {
  kErrSortSpin = 1u << 1,          // radix-sort look-back wait gave up
  kErrCellRange = 1u << 2,         // a particle hashed outside the grid
  kErrScanSpin = 1u << 3,
  kErrNbrTail = 1u << 5,           // a list block's entries past the count are not p
};

struct DevParams {
  int n;
  int nx, ny, nz;
  uint32_t nxny;
  uint32_t ncells;      // C = nx*ny*nz
  int bx, by;           // packed-cell bit widths of x and y
  uint32_t mx, my;      // masks for cx and cy
  double hd;            // smoothing radius (double)
  double fx_scale;      // 2^k: fixed-point units per length of the records
  float fx_inv;         // 2^-k
  float fx_inv2;        // 2^-2k
  float h_fx;           // h in fixed-point units (h 2^k)
  float rmin2_fx;       // (1e-4 h)^2 in fixed-point units squared
  double h2d;
  // neighbour-build FP32 pre-test band: pairs with FP32 r^2 in [lo, hi] go
  // to the exact FP64 test (lo = -1, hi = inf: every pair does)
  float bld_h2lo, bld_h2hi;
  float h, h2;
  float rmin;           // r floor 1e-4 h (particles.c:636)
  // smoothing-kernel constants; *_m variants carry the particle mass
  float W0m;            // m * W(0)
  float Wn, Wn_m;       // poly6 norm
  float DWn, DWn_m;     // spiky gradient norm
  float DWPn;           // poly6 gradient norm
  float m, rho0, inv_rho0, inv_rho0_sq;
  double rho0_d;
  float lambda_eps;
  float scorr_k;        // s_corr = -k (W/W(dq))^n
  int scorr_n;
  float inv_Wdq;
  float scorr_u;        // 1 / (h^2 - dq^2): W(r)/W(dq) = ((h^2 - r^2) scorr_u)^3
  float scorr_u_fx;     // scorr_u 2^-2k (for r^2 in fixed-point units squared)
  float scorr_uh2;      // scorr_u h^2
  float c_xsph;
  int xsph_exact;       // 0: reference r expression (particles.c:439)
  float gamma, C_norm;  // surface tension
  float vort_eps;
  float dt, inv_dt, v_max;
  double dt_d, gdt_d;   // gravity increment (-g*dt) in double
  int gaxis;
  float gdt_f;
  double bmin[3], bmax[3], bmax_eps[3];  // clamp (particles.c:842-867)
  // obstacle SDF (x fastest), tex3D-style sampling
  int has_sdf;
  int sdim[3];
  const float* sdf;
  double ob_min[3], ob_max[3];
  float ob_len[3];      // world extents as float (obstacle_cuda.cu:74-85)
  float tex_sp[3];      // 1/dim in normalised coordinates
  float model_to_world;
};

// View of the per-step neighbour structure.
struct NbrView {
  const uint32_t* __restrict__ nbr;     // [kMaxNeighbors / 4][n] blocks of 4 entries
  const uint8_t* __restrict__ ncount;   // [n]
  const uint32_t* __restrict__ cstart;  // [C+1]
  int n;
  int nx, ny, nz;
  uint32_t nxny;
  int bx, by;
  uint32_t mx, my;
};

__device__ __forceinline__ void unpack_cell(const NbrView& v, uint32_t cp, int& cx,
                                            int& cy, int& cz) {
  cx = (int)(cp & v.mx);
  cy = (int)((cp >> v.bx) & v.my);
  cz = (int)(cp >> (v.bx + v.by));
}

// Neighbour lists, nbr4[15][n] (uint4): block b of particle p holds its list
// entries 4b .. 4b+3 (column b of all particles contiguous, so a warp reads
// four whole 128-byte lines per block index); the entries of the last block
// past the count hold p itself.  Entry j of particle p:
__device__ __forceinline__ uint32_t nbr_entry(const NbrView& v, int p, int j) {
  return __ldg(v.nbr + (((size_t)(j >> 2) * v.n + p) << 2) + (j & 3));
}
__device__ __forceinline__ uint4 nbr_block(const NbrView& v, int p, int b) {
  return __ldg(reinterpret_cast<const uint4*>(v.nbr) + (size_t)b * v.n + p);
}

// Visits the neighbour slots of particle p in the reference's bucket order
// (FillNeighbors, neighbors.c:247-295: dz, dy, dx, then ascending sorted
// index), as stored by the neighbour build.
template <class F>
__device__ __forceinline__ void for_each_neighbor(const NbrView& v, int p, F&& f) {
  const int cnt = (int)__ldg(v.ncount + p);
#pragma unroll 2
  for (int j = 0; j < cnt; ++j) f((int)nbr_entry(v, p, j));
}

// The batched visits below take a batch of four list entries per 128-bit
// load (one block) and load the next block before the bodies of this batch
// run, so a batch waits only for its record gathers (the list read from HBM
// overlaps the previous batch).  The entries of the last block past the count
// are p: those slots load the particle's own record and are skipped, or, with
// kPadSlots, visited as the pair (p, p) (for bodies whose every term carries
// the pair difference, which is 0).
#define SPHPC_NBR_BATCH_HEAD                                      \
  static_assert(B == 4, "a batch is one four-entry list block"); \
  const int cnt = (int)__ldg(v.ncount + p);                      \
  uint4 blk = cnt > 0 ? nbr_block(v, p, 0) : make_uint4(p, p, p, p)
#define SPHPC_NBR_BATCH_NEXT(j0)                                                         \
  const int q[4] = {(int)blk.x, (int)blk.y, (int)blk.z, (int)blk.w};                    \
  if ((j0) + 4 < cnt) blk = nbr_block(v, p, ((j0) >> 2) + 1)

// Each neighbour's 16-byte record loaded for f(q, rq).
template <int B, bool kPadSlots = false, class F>
__device__ __forceinline__ void for_each_neighbor_nr(const NbrView& v, const uint4* __restrict__ nr,
                                                     int p, F&& f) {
  SPHPC_NBR_BATCH_HEAD;
  for (int j0 = 0; j0 < cnt; j0 += 4) {
    SPHPC_NBR_BATCH_NEXT(j0);
    uint4 r[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) r[u] = ld_nr(nr, q[u]);
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (kPadSlots || j0 + u < cnt) f(q[u], r[u]);
  }
}

// The same batched visit with the whole batch handed to f(r[B], nvalid):
// r[u] is the record of list entry j0 + u for u < nvalid = min(B, cnt - j0)
// and the particle's own record past the count (the pair (p, p), difference
// 0), so a body can combine the batch's terms before adding them to a sum.
template <int B, class F>
__device__ __forceinline__ void for_each_batch_nr(const NbrView& v, const uint4* __restrict__ nr,
                                                  int p, F&& f) {
  SPHPC_NBR_BATCH_HEAD;
  for (int j0 = 0; j0 < cnt; j0 += 4) {
    SPHPC_NBR_BATCH_NEXT(j0);
    uint4 r[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) r[u] = ld_nr(nr, q[u]);
    f(r, cnt - j0);
  }
}

__device__ __forceinline__ void ld_nv(const NV* __restrict__ base, int i, uint4& r, float4& e) {
  asm("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w), "=f"(e.x), "=f"(e.y), "=f"(e.z), "=f"(e.w)
      : "l"(base + i));
}

__device__ __forceinline__ void st_nv(NV* base, int i, const uint4 r, const float4 e) {
  asm volatile("st.global.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(base + i), "r"(r.x),
               "r"(r.y), "r"(r.z), "r"(r.w), "f"(e.x), "f"(e.y), "f"(e.z), "f"(e.w)
               : "memory");
}

// Batched visit over the 32-byte records {r, e}: f(q, rq, eq), as
// for_each_neighbor_nr with one 256-bit gather per neighbour.
template <int B, bool kPadSlots = false, class F>
__device__ __forceinline__ void for_each_neighbor_nv(const NbrView& v, const NV* __restrict__ nv,
                                                     int p, F&& f) {
  SPHPC_NBR_BATCH_HEAD;
  for (int j0 = 0; j0 < cnt; j0 += 4) {
    SPHPC_NBR_BATCH_NEXT(j0);
    uint4 r[4];
    float4 e[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) ld_nv(nv, q[u], r[u], e[u]);
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (kPadSlots || j0 + u < cnt) f(q[u], r[u], e[u]);
  }
}

// Batched visit over the 32-byte particle records with the batch handed to
// f(x[B], d[B], nvalid), nvalid = min(B, cnt - j0); slots past the count
// hold the particle's own record and are the body's to skip.
template <int B, class F>
__device__ __forceinline__ void for_each_batch_pd(const NbrView& v, const PD* __restrict__ pd,
                                                  int p, F&& f) {
  SPHPC_NBR_BATCH_HEAD;
  for (int j0 = 0; j0 < cnt; j0 += 4) {
    SPHPC_NBR_BATCH_NEXT(j0);
    float4 x[4], d[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) ld_pd(pd, q[u], x[u], d[u]);
    f(x, d, cnt - j0);
  }
}

#undef SPHPC_NBR_BATCH_HEAD
#undef SPHPC_NBR_BATCH_NEXT

// ---------------------------------------------------------------------------
// Canonical double predicted position and the reference's box clamp.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double xstar_d(float x, float d) {
  return __dadd_rn((double)x, (double)d);
}

// ApplyBoundaryConditions, particles.c:842-867, on one axis.
__device__ __forceinline__ double clamp_axis(double x, double lo, double hi,
                                             double hi_eps) {
  if (x < lo) return lo;
  if (x >= hi) return hi_eps;
  return x;
}

// Fixed-point coordinate of a double position (round to nearest, mod 2^32).
__device__ __forceinline__ uint32_t fx_of(const DevParams& P, double x) {
  return (uint32_t)(unsigned long long)__double2ll_rn(__dmul_rn(x, P.fx_scale));
}

__device__ __forceinline__ uint4 make_nr(const DevParams& P, double x, double y, double z,
                                         float w) {
  return make_uint4(fx_of(P, x), fx_of(P, y), fx_of(P, z), __float_as_uint(w));
}

// HashVal, neighbors.c:79-98, per axis: floor(x / spacing) in FP64.
__device__ __forceinline__ int grid_coord(double x, double h) {
  return (int)(unsigned)floor(__ddiv_rn(x, h));
}

// ---------------------------------------------------------------------------
// SDF obstacle: tex3D<float> (linear filter, clamp addressing, normalised
// coordinates; obstacle_cuda.cu:166-181) with exact FP32 weights.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float sdf_texel(const DevParams& P, int i, int j, int k) {
  i = min(max(i, 0), P.sdim[0] - 1);
  j = min(max(j, 0), P.sdim[1] - 1);
  k = min(max(k, 0), P.sdim[2] - 1);
  return __ldg(P.sdf + ((size_t)k * P.sdim[1] + j) * P.sdim[0] + i);
}

__device__ __forceinline__ float lerp_rn(float a, float b, float t) {
  return __fmaf_rn(t, __fsub_rn(b, a), a);
}

__device__ __forceinline__ float sdf_sample(const DevParams& P, float u, float v, float w) {
  const float xb = __fsub_rn(__fmul_rn(u, (float)P.sdim[0]), 0.5f);
  const float yb = __fsub_rn(__fmul_rn(v, (float)P.sdim[1]), 0.5f);
  const float zb = __fsub_rn(__fmul_rn(w, (float)P.sdim[2]), 0.5f);
  const float fx = floorf(xb), fy = floorf(yb), fz = floorf(zb);
  const float ax = __fsub_rn(xb, fx), ay = __fsub_rn(yb, fy), az = __fsub_rn(zb, fz);
  const int i = (int)fx, j = (int)fy, k = (int)fz;
  const float c00 = lerp_rn(sdf_texel(P, i, j, k), sdf_texel(P, i + 1, j, k), ax);
  const float c10 = lerp_rn(sdf_texel(P, i, j + 1, k), sdf_texel(P, i + 1, j + 1, k), ax);
  const float c01 = lerp_rn(sdf_texel(P, i, j, k + 1), sdf_texel(P, i + 1, j, k + 1), ax);
  const float c11 = lerp_rn(sdf_texel(P, i, j + 1, k + 1), sdf_texel(P, i + 1, j + 1, k + 1), ax);
  const float c0 = lerp_rn(c00, c10, ay);
  const float c1 = lerp_rn(c01, c11, ay);
  return lerp_rn(c0, c1, az);
}

// CalculateParticleCollisions_kernel body (obstacle_cuda.cu:62-115) on one
// double position.  Returns true and updates xyz when the particle is pushed.
__device__ __forceinline__ bool sdf_collide(const DevParams& P, double& x, double& y,
                                            double& z) {
  if (!(x > P.ob_min[0] && x < P.ob_max[0] && y > P.ob_min[1] && y < P.ob_max[1] &&
        z > P.ob_min[2] && z < P.ob_max[2]))
    return false;
  const float xt = (float)__ddiv_rn(__dsub_rn(x, P.ob_min[0]), (double)P.ob_len[0]);
  const float yt = (float)__ddiv_rn(__dsub_rn(y, P.ob_min[1]), (double)P.ob_len[1]);
  const float zt = (float)__ddiv_rn(__dsub_rn(z, P.ob_min[2]), (double)P.ob_len[2]);
  const float dist = sdf_sample(P, xt, yt, zt);
  if (!(dist < 0.0f)) return false;
  const float gx = __fsub_rn(sdf_sample(P, __fadd_rn(xt, P.tex_sp[0]), yt, zt),
                             sdf_sample(P, __fsub_rn(xt, P.tex_sp[0]), yt, zt));
  const float gy = __fsub_rn(sdf_sample(P, xt, __fadd_rn(yt, P.tex_sp[1]), zt),
                             sdf_sample(P, xt, __fsub_rn(yt, P.tex_sp[1]), zt));
  const float gz = __fsub_rn(sdf_sample(P, xt, yt, __fadd_rn(zt, P.tex_sp[2])),
                             sdf_sample(P, xt, yt, __fsub_rn(zt, P.tex_sp[2])));
  const float dot = __fadd_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)),
                              __fmul_rn(gz, gz));
  const float inv = __fdiv_rn(1.0f, __fsqrt_rn(dot));
  const float dw = __fmul_rn(fabsf(dist), P.model_to_world);
  y = __dadd_rn(y, (double)__fmul_rn(dw, __fmul_rn(gy, inv)));
  x = __dadd_rn(x, (double)__fmul_rn(dw, __fmul_rn(gx, inv)));
  z = __dadd_rn(z, (double)__fmul_rn(dw, __fmul_rn(gz, inv)));
  return true;
}

}  // namespace sphpc
