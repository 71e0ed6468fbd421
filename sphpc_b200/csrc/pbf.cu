// pbf.cu -- the neighbour passes and pointwise steps of one PBF time step.
//
// Every pass is one thread per particle in slot (cell-sorted) order; the
// neighbour loop visits the bucket of the particle in the reference's order
// (for_each_neighbor).  Sums are FP32 (density with Kahan compensation);
// the box clamp, the SDF lookup and the position update are FP64 on the
// canonical double x* = x + d of the particle's own record.  Neighbours are
// read from the 16-byte records (fixed-point x* and a payload) with one
// 128-bit load each; the pair difference is their exact integer difference.
#include "kernels.cuh"

namespace sphpc {

namespace {

struct Pair {
  float dx, dy, dz, r2;
};

// neighbours whose list entries and records are fetched together
constexpr int kNbrBatch = 4;
// resident 256-thread blocks per SM asked of the compiler for the neighbour
// passes (register caps of 40, 48 and 64; more resident warps hide the gather
// latency better than the registers a larger allocation would keep, as long
// as the neighbour loop itself does not spill).  The position pass runs at 48:
// at 40 its FP64 epilogue spills up to 88 bytes a thread through the L1 that
// its gathers already keep busy (2.4-3.5% slower at 16.7M particles).
constexpr int kMinBlocksDensity = 6;
constexpr int kMinBlocksPosition = 5;
constexpr int kMinBlocksColor = 5;
constexpr int kMinBlocksVorticity = 5;
constexpr int kMinBlocksConfinement = 6;
constexpr int kMinBlocksTension = 4;  // 64 registers: at 48 the loop spills
constexpr int kMinBlocksXsph = 4;
constexpr int kMinBlocksFeatures = 4;

// x*_p - x*_q as (x_p - x_q) + (d_p - d_q): exact in the first term for any
// box size, so the FP32 pair geometry keeps its relative precision.
__device__ __forceinline__ void ld_rw(const PD* base, int i, float4& x, float4& d) {
  x = base[i].x;
  d = base[i].d;
}

// x*_p - x*_q from two 16-byte records: the wrapping integer difference is
// exact, its conversion to FP32 rounds like any FP32 difference.
__device__ __forceinline__ Pair pair_nr(const DevParams& P, const uint4 a, const uint4 b) {
  Pair g;
  g.dx = __fmul_rn((float)(int)(a.x - b.x), P.fx_inv);
  g.dy = __fmul_rn((float)(int)(a.y - b.y), P.fx_inv);
  g.dz = __fmul_rn((float)(int)(a.z - b.z), P.fx_inv);
  g.r2 = norm2(g.dx, g.dy, g.dz);
  return g;
}

__device__ __forceinline__ Pair pair_geom(const float4 xp, const float4 dp, const float4 xq,
                                          const float4 dq) {
  Pair g;
  g.dx = (xp.x - xq.x) + (dp.x - dq.x);
  g.dy = (xp.y - xq.y) + (dp.y - dq.y);
  g.dz = (xp.z - xq.z) + (dp.z - dq.z);
  g.r2 = norm2(g.dx, g.dy, g.dz);
  return g;
}

// r_mag floored at 1e-4 h (particles.c:635-637): returns r and 1/r.
__device__ __forceinline__ void floored_r(const DevParams& P, float r2, float& r, float& rinv) {
  const float r2c = fmaxf(r2, P.rmin * P.rmin);
  rinv = rsqrtf(r2c);
  r = __fmul_rn(r2c, rinv);
}

// The same in fixed-point units (r2f = |d|^2 of the record difference):
// r2c = max(r2f, r_min^2) and rinv_f = 2^-k / r, so the loops need no
// rescaling of r^2; r_f = r 2^k is r2c rinv (fx_r), and h_f - r_f, floored at
// 0, one fused multiply-add (fx_hm).
__device__ __forceinline__ void floored_r_fx(const DevParams& P, float r2f, float& r2c,
                                             float& rinv) {
  r2c = fmaxf(r2f, P.rmin2_fx);
  rinv = rsqrtf(r2c);
}
__device__ __forceinline__ float fx_r(float r2c, float rinv) { return __fmul_rn(r2c, rinv); }
__device__ __forceinline__ float fx_hm(const DevParams& P, float r2c, float rinv) {
  return fmaxf(fmaf(-r2c, rinv, P.h_fx), 0.0f);
}

// 1/x by the hardware's approximate reciprocal (PTX rcp.approx.ftz.f32, at
// most 1 ulp from the rounded quotient): one instruction where the correctly
// rounded reciprocal takes a refinement sequence.  Used for the neighbour
// densities of the post passes (x near rho0, never subnormal).
__device__ __forceinline__ float rcp_fast(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void block_resid(double e, double* resid) {
  // max and sum of the per-particle density error over the block (FP64).
  double m = e, s = e;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    s += __shfl_xor_sync(0xffffffffu, s, o);
  }
  __shared__ double sm[kBlock / 32], ss[kBlock / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sm[warp] = m;
    ss[warp] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double bm = 0.0, bs = 0.0;
    for (int w = 0; w < kBlock / 32; ++w) {
      bm = fmax(bm, sm[w]);
      bs += ss[w];
    }
    atomicMax(reinterpret_cast<unsigned long long*>(resid),
              (unsigned long long)__double_as_longlong(bm));
    atomicAdd(resid + 1, bs);
  }
}

template <int MODE, bool RESID>
__global__ void __launch_bounds__(kBlock, kMinBlocksDensity)
    k_density_lambda(const DevParams P, const NbrView V, const PassArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  double err = 0.0;
  if (p < P.n) {
    const uint4 rp = ld_nr(a.nr, p);
    // The loop keeps only what varies per pair: the density sums t^3 with
    // t = h^2 - r^2 and the gradient sums c d with c = (h - r)^2 / r and d
    // the pair difference, both in fixed-point units; the kernel norms, the
    // mass and 2^-2k multiply the sums once afterwards.  The density sum is
    // Kahan-compensated per batch: a batch's four terms are added pairwise
    // (relative error at most 2 ulp of the batch sum, all terms >= 0) and the
    // batch sum enters the compensated running sum.  Padding slots past the
    // count are the pair (p, p): their density term is masked, their gradient
    // terms carry d = 0.
    float st = 0.0f, comp = 0.0f;
    float sgx = 0.f, sgy = 0.f, sgz = 0.f, sC = 0.f;
    for_each_batch_nr<kNbrBatch>(V, a.nr, p, [&](const uint4 (&rq)[kNbrBatch], int nvalid) {
      float t3[kNbrBatch];
#pragma unroll
      for (int u = 0; u < kNbrBatch; ++u) {
        const float fx = (float)(int)(rp.x - rq[u].x);
        const float fy = (float)(int)(rp.y - rq[u].y);
        const float fz = (float)(int)(rp.z - rq[u].z);
        const float r2f = norm2(fx, fy, fz);
        if (MODE != 2) {
          float t = fmaxf(fmaf(-P.fx_inv2, r2f, P.h2), 0.0f);
          t = u < nvalid ? t : 0.0f;
          t3[u] = t;
        }
        if (MODE != 1) {
          // in fixed-point units: c_f = (h_f - r_f)^2 / r_f = 2^k c
          float r2c, rinv;
          floored_r_fx(P, r2f, r2c, rinv);
          const float hm = fx_hm(P, r2c, rinv);
          const float c = __fmul_rn(__fmul_rn(hm, hm), rinv);
          // |c d|^2 = c^2 |d|^2: three fused accumulations and one for the norm
          sgx = fmaf(c, fx, sgx);
          sgy = fmaf(c, fy, sgy);
          sgz = fmaf(c, fz, sgz);
          sC = fmaf(__fmul_rn(c, c), r2f, sC);
        }
      }
      if (MODE != 2) {
        static_assert(kNbrBatch == 4, "batch sum of four terms");
        // t0^3 + t1^3 + t2^3 + t3^3 as a chain of fused multiply-adds
        const float* t = t3;
        const float yb = fmaf(__fmul_rn(t[0], t[0]), t[0],
                              fmaf(__fmul_rn(t[1], t[1]), t[1],
                                   fmaf(__fmul_rn(t[2], t[2]), t[2],
                                        __fmul_rn(__fmul_rn(t[3], t[3]), t[3]))));
        const float y = yb - comp;
        const float s = st + y;
        comp = (s - st) - y;
        st = s;
      }
    });
    float rho;
    if (MODE == 2) rho = a.rho[p];
    if (MODE != 2) {
      rho = fmaf(P.Wn_m, st - comp, P.W0m);
      a.rho[p] = rho;
    }
    if (MODE != 1) {
      // ComputeLambda's constraint (particles.c:616-617) in FP64
      const float C = (float)fmax(__ddiv_rn((double)rho, P.rho0_d) - 1.0, 0.0);
      const float g = P.DWn_m * P.fx_inv2;  // gradient scale (2^-2k is exact)
      sC = __fadd_rn(sC, norm2(sgx, sgy, sgz));
      sC *= (g * g) * P.inv_rho0_sq;
      const float lam = -C / (sC + P.lambda_eps);
      if (a.nr_out) a.nr_out[p] = make_uint4(rp.x, rp.y, rp.z, __float_as_uint(lam));
      if (a.lam) a.lam[p] = lam;
    }
    if (RESID) err = fmax((double)rho / (double)P.rho0 - 1.0, 0.0);
  }
  if (RESID) block_resid(err, a.resid);
}

// The first density/lambda pass of a step (mode 0, with residual) that also
// forms the 16 warm-start features of each particle p < limit:
//   0 rho/rho0 - 1       1 C = max(rho/rho0 - 1, 0)     2 lambda
//   3 sum_q |grad_q C|^2 4 |grad_p C|^2 (both with the 1/rho0^2 of lambda)
//   5 neighbour count    6-8 mean neighbour offset (x*_q - x*_p) / h
//   9-11 mean relative predicted displacement (d_q - d_p) / h, d = x* - x
//        (= the mean relative velocity * dt / h away from the box walls)
//   12 SDF distance at x* / h, clamped to [-4, 4] (4 without an obstacle)
//   13 nearest-neighbour distance / h (1 without neighbours)
//   14 distance to the nearest box wall / h, clamped to [0, 4]
//   15 own predicted displacement along the gravity axis / h
// RAW: FP32 features to feat[p][16]; otherwise the network's input row
// bf16((f - mean) * inv_std) (norm = mean[16], inv_std[16]) to xbf[p][16].
template <bool RAW>
__global__ void __launch_bounds__(kBlock, kMinBlocksFeatures)
    k_features(const DevParams P, const NbrView V, const PassArgs a, float* __restrict__ feat,
               __nv_bfloat16* __restrict__ xbf, const float* __restrict__ norm, int limit) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  double err = 0.0;
  if (p < P.n) {
    float4 xp, dp;
    ld_pd(a.pd, p, xp, dp);
    // Only what varies per pair stays in the loop: the sum of t^3
    // (t = h^2 - r^2), the sums of c d with c = (h - r)^2 / r and of c^2 r^2,
    // the neighbour offsets and displacements; the kernel norms and the mass
    // multiply the sums once afterwards, as in the density pass.  The t^3
    // sum is Kahan-compensated per batch of four neighbours, as there.
    float st = 0.0f, comp = 0.0f;
    float sgx = 0.f, sgy = 0.f, sgz = 0.f, sC = 0.f;
    float ox = 0.f, oy = 0.f, oz = 0.f, ux = 0.f, uy = 0.f, uz = 0.f, rmin2 = P.h2;
    int cnt = 0;
    for_each_batch_pd<kNbrBatch>(V, a.pd, p, [&](const float4 (&xq)[kNbrBatch],
                                                 const float4 (&dq)[kNbrBatch], int nvalid) {
      float yb = 0.0f;
#pragma unroll
      for (int u = 0; u < kNbrBatch; ++u) {
        if (u < nvalid) {
          const Pair g = pair_geom(xp, dp, xq[u], dq[u]);
          const float t = fmaxf(P.h2 - g.r2, 0.0f);
          yb = fmaf(__fmul_rn(t, t), t, yb);
          float r, rinv;
          floored_r(P, g.r2, r, rinv);
          const float hm = fmaxf(P.h - r, 0.0f);
          const float c = __fmul_rn(__fmul_rn(hm, hm), rinv);
          sgx = fmaf(c, g.dx, sgx);
          sgy = fmaf(c, g.dy, sgy);
          sgz = fmaf(c, g.dz, sgz);
          sC = fmaf(__fmul_rn(c, c), g.r2, sC);
          ox -= g.dx;
          oy -= g.dy;
          oz -= g.dz;
          ux += dq[u].x;
          uy += dq[u].y;
          uz += dq[u].z;
          rmin2 = fminf(rmin2, g.r2);
          ++cnt;
        }
      }
      const float y = yb - comp;
      const float s = st + y;
      comp = (s - st) - y;
      st = s;
    });
    // sum_q (d_q - d_p) from sum_q d_q
    ux = fmaf(-(float)cnt, dp.x, ux);
    uy = fmaf(-(float)cnt, dp.y, uy);
    uz = fmaf(-(float)cnt, dp.z, uz);
    sgx *= P.DWn_m;
    sgy *= P.DWn_m;
    sgz *= P.DWn_m;
    sC *= P.DWn_m * P.DWn_m;
    const float rho = fmaf(P.Wn_m, st - comp, P.W0m);
    a.rho[p] = rho;
    const float C = (float)fmax(__ddiv_rn((double)rho, P.rho0_d) - 1.0, 0.0);
    const float s_pairs = sC * P.inv_rho0_sq;
    sC = __fadd_rn(sC, norm2(sgx, sgy, sgz));
    sC *= P.inv_rho0_sq;
    const float lam = -C / (sC + P.lambda_eps);
    const double xs = xstar_d(xp.x, dp.x), ys = xstar_d(xp.y, dp.y), zs = xstar_d(xp.z, dp.z);
    a.nr_out[p] = make_nr(P, xs, ys, zs, lam);
    err = fmax((double)rho / (double)P.rho0 - 1.0, 0.0);
    if (p < limit) {
      const float inv_h = 1.0f / P.h;
      const float s_self = __fmul_rn(norm2(sgx, sgy, sgz), P.inv_rho0_sq);
      const float inv_cnt = cnt > 0 ? 1.0f / (float)cnt : 0.0f;
      const float sc = inv_h * inv_cnt;
      float sdf = 4.0f;
      if (P.has_sdf && xs > P.ob_min[0] && xs < P.ob_max[0] && ys > P.ob_min[1] &&
          ys < P.ob_max[1] && zs > P.ob_min[2] && zs < P.ob_max[2]) {
        const float xt = (float)((xs - P.ob_min[0]) / (double)P.ob_len[0]);
        const float yt = (float)((ys - P.ob_min[1]) / (double)P.ob_len[1]);
        const float zt = (float)((zs - P.ob_min[2]) / (double)P.ob_len[2]);
        sdf = fminf(fmaxf(sdf_sample(P, xt, yt, zt) * P.model_to_world * inv_h, -4.0f), 4.0f);
      }
      const double wall =
          fmin(fmin(xs - P.bmin[0], P.bmax[0] - xs),
               fmin(fmin(ys - P.bmin[1], P.bmax[1] - ys), fmin(zs - P.bmin[2], P.bmax[2] - zs)));
      const float fw = fminf(fmaxf((float)(wall / P.hd), 0.0f), 4.0f);
      const float vg = (P.gaxis == 0 ? dp.x : (P.gaxis == 1 ? dp.y : dp.z)) * inv_h;
      const float f[16] = {fmaf(rho, P.inv_rho0, -1.0f), C, lam, s_pairs, s_self, (float)cnt,
                           ox * sc, oy * sc, oz * sc, ux * sc, uy * sc, uz * sc,
                           sdf, sqrtf(rmin2) * inv_h, fw, vg};
      if (RAW) {
        float4* out = reinterpret_cast<float4*>(feat + (size_t)p * 16);
#pragma unroll
        for (int k = 0; k < 4; ++k)
          out[k] = make_float4(f[4 * k], f[4 * k + 1], f[4 * k + 2], f[4 * k + 3]);
      } else {
        uint32_t w[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const float lo = (f[2 * k] - __ldg(norm + 2 * k)) * __ldg(norm + 16 + 2 * k);
          const float hi = (f[2 * k + 1] - __ldg(norm + 2 * k + 1)) * __ldg(norm + 17 + 2 * k);
          const __nv_bfloat162 b2 = __floats2bfloat162_rn(lo, hi);
          w[k] = *reinterpret_cast<const uint32_t*>(&b2);
        }
        uint4* out = reinterpret_cast<uint4*>(xbf + (size_t)p * 16);
        out[0] = make_uint4(w[0], w[1], w[2], w[3]);
        out[1] = make_uint4(w[4], w[5], w[6], w[7]);
      }
    }
  }
  block_resid(err, a.resid);
}

// target[p] += s * lambda_p (lambda in d.w of the records) for p < limit:
// the stiffness-weighted multiplier sum of a plain solve, the warm-start
// network's training target.
__global__ void k_accum_lambda(const uint4* __restrict__ rec, float s, float* __restrict__ target,
                               int limit) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < limit) target[p] = fmaf(s, __uint_as_float(rec[p].w), target[p]);
}

template <int MODE, int SCORR_N, bool SDF>
__global__ void __launch_bounds__(kBlock, kMinBlocksPosition)
    k_position(const DevParams P, const NbrView V, const PassArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  const uint4 rp = ld_nr(a.nr, p);
  const float lp = nr_w(rp);
  float4 xp, dp;  // own particle record, loaded ahead of the neighbour loop
  if (MODE == 0) ld_pd(a.pd, p, xp, dp);
  // sums of c d with c = (lambda_p + lambda_q + s_corr) (h - r)^2 / r and d
  // the pair difference, both in fixed-point units; the spiky norm, the mass
  // and 2^-2k multiply them once afterwards.  Every term carries d, so the batch's
  // padding slots (q = p, d = 0) add nothing and are not masked.
  float ax = 0.f, ay = 0.f, az = 0.f;
  for_each_neighbor_nr<kNbrBatch, true>(V, a.nr, p, [&](int, const uint4 rq) {
    const float fx = (float)(int)(rp.x - rq.x);
    const float fy = (float)(int)(rp.y - rq.y);
    const float fz = (float)(int)(rp.z - rq.z);
    // in fixed-point units: c_f = s (h_f - r_f)^2 / r_f = 2^k c
    float r2c, rinv;
    floored_r_fx(P, norm2(fx, fy, fz), r2c, rinv);
    const float hm = fx_hm(P, r2c, rinv);
    float s = lp + nr_w(rq);
    if (SCORR_N != 0) {
      // W(r) / W(dq) = u^3 with u = (h^2 - r^2) / (h^2 - dq^2), u <= 1.05
      const float u = fmaxf(fmaf(-P.scorr_u_fx, r2c, P.scorr_uh2), 0.0f);
      if (SCORR_N == 4) {
        const float u2 = u * u;
        const float u4 = u2 * u2;
        s = fmaf(-P.scorr_k, u4 * u4 * u4, s);
      } else {
        const float ratio = u * u * u;
        float sc = -P.scorr_k;
        for (int e = 0; e < P.scorr_n; ++e) sc = __fmul_rn(sc, ratio);
        s = __fadd_rn(s, sc);
      }
    }
    const float c = __fmul_rn(__fmul_rn(__fmul_rn(s, hm), hm), rinv);
    ax = fmaf(c, fx, ax);
    ay = fmaf(c, fy, ay);
    az = fmaf(c, fz, az);
  });
  const float s = a.stiffness * P.inv_rho0 * (P.DWn_m * P.fx_inv2);
  const float dpx = ax * s, dpy = ay * s, dpz = az * s;
  if (MODE == 1) {
    a.dp[p] = make_float4(dpx, dpy, dpz, 0.0f);
    return;
  }
  double xs = __dadd_rn(xstar_d(xp.x, dp.x), (double)dpx);
  double ys = __dadd_rn(xstar_d(xp.y, dp.y), (double)dpy);
  double zs = __dadd_rn(xstar_d(xp.z, dp.z), (double)dpz);
  xs = clamp_axis(xs, P.bmin[0], P.bmax[0], P.bmax_eps[0]);
  ys = clamp_axis(ys, P.bmin[1], P.bmax[1], P.bmax_eps[1]);
  zs = clamp_axis(zs, P.bmin[2], P.bmax[2], P.bmax_eps[2]);
  if (SDF) sdf_collide(P, xs, ys, zs);
  const double ex = __dsub_rn(xs, (double)xp.x), ey = __dsub_rn(ys, (double)xp.y),
               ez = __dsub_rn(zs, (double)xp.z);
  const float rho_p = a.rho[p];
  const float4 dn = make_float4(__double2float_rn(ex), __double2float_rn(ey),
                                __double2float_rn(ez), rho_p);
  st_pd(a.pd_out, p, xp, dn);
  // the record carries the canonical x* = x + d of what was just stored
  a.nr_out[p] = make_nr(P, xstar_d(xp.x, dn.x), xstar_d(xp.y, dn.y), xstar_d(xp.z, dn.z), rho_p);
  if (a.lam_acc) a.lam_acc[p] = fmaf(a.stiffness, lp, a.acc_add ? a.lam_acc[p] : 0.0f);
  if (a.last) {
    // UpdateVelocities, particles.c:814-837
    float vx = __double2float_rn(__ddiv_rn(ex, P.dt_d));
    float vy = __double2float_rn(__ddiv_rn(ey, P.dt_d));
    float vz = __double2float_rn(__ddiv_rn(ez, P.dt_d));
    vx = fminf(fmaxf(vx, -P.v_max), P.v_max);
    vy = fminf(fmaxf(vy, -P.v_max), P.v_max);
    vz = fminf(fmaxf(vz, -P.v_max), P.v_max);
    a.vel_out[p] = make_float4(vx, vy, vz, 0.0f);
  }
}

template <bool SDF>
__global__ void __launch_bounds__(kBlock) k_apply_dp(const DevParams P, const PassArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  float4 xp, dp;
  ld_rw(a.pd_out, p, xp, dp);
  const float4 dd = __ldg(a.dp + p);
  double xs = __dadd_rn(xstar_d(xp.x, dp.x), (double)dd.x);
  double ys = __dadd_rn(xstar_d(xp.y, dp.y), (double)dd.y);
  double zs = __dadd_rn(xstar_d(xp.z, dp.z), (double)dd.z);
  xs = clamp_axis(xs, P.bmin[0], P.bmax[0], P.bmax_eps[0]);
  ys = clamp_axis(ys, P.bmin[1], P.bmax[1], P.bmax_eps[1]);
  zs = clamp_axis(zs, P.bmin[2], P.bmax[2], P.bmax_eps[2]);
  if (SDF) sdf_collide(P, xs, ys, zs);
  a.pd_out[p].d = make_float4(__double2float_rn(__dsub_rn(xs, (double)xp.x)),
                              __double2float_rn(__dsub_rn(ys, (double)xp.y)),
                              __double2float_rn(__dsub_rn(zs, (double)xp.z)), dp.w);
}

__global__ void __launch_bounds__(kBlock) k_pack_nv(int n, const uint4* __restrict__ nr,
                                                    const float4* __restrict__ e,
                                                    NV* __restrict__ nv) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) st_nv(nv, p, ld_nr(nr, p), __ldg(e + p));
}

__global__ void __launch_bounds__(kBlock, kMinBlocksColor)
    k_color(const DevParams P, const NbrView V, const PassArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  const uint4 rp = ld_nr(a.nr, p);
  // sums of (h^2 - r^2)^2 r / (r rho_q) d, d in fixed-point units; the
  // poly6-gradient norm, m, h and 2^-k multiply them once (every term carries
  // d, so the padding slots add nothing)
  float cx = 0.f, cy = 0.f, cz = 0.f;
  for_each_neighbor_nr<kNbrBatch, true>(V, a.nr, p, [&](int, const uint4 rq) {
    const float fx = (float)(int)(rp.x - rq.x);
    const float fy = (float)(int)(rp.y - rq.y);
    const float fz = (float)(int)(rp.z - rq.z);
    // r and 1/r in fixed-point units (their product is unit-free)
    float r2c, rinv;
    floored_r_fx(P, norm2(fx, fy, fz), r2c, rinv);
    const float t = fmaxf(fmaf(-P.fx_inv2, r2c, P.h2), 0.0f);
    const float c = __fmul_rn(__fmul_rn(__fmul_rn(t, t), fx_r(r2c, rinv)),
                              __fmul_rn(rinv, rcp_fast(nr_w(rq))));
    cx = fmaf(c, fx, cx);
    cy = fmaf(c, fy, cy);
    cz = fmaf(c, fz, cz);
  });
  const float s = P.h * (P.DWPn * P.m * P.fx_inv);
  const float4 col = make_float4(s * cx, s * cy, s * cz, 0.0f);
  a.color[p] = col;
  if (a.nv_out) st_nv(a.nv_out, p, rp, col);
}

// Akinci cohesion spline (particles.c:54-65) without its norm: with
// y = ((h - r) r)^3, 2y - h^6/64 for r <= h/2, y up to h, 0 beyond (h6_64 =
// h^6/64); selects, no branches.
__device__ __forceinline__ float cohesion_unnormed(const DevParams& P, float r, float h6_64) {
  const float hr = (P.h - r) * r;
  const float y = hr * hr * hr;
  float c = r <= 0.5f * P.h ? fmaf(2.0f, y, -h6_64) : y;
  return r > P.h ? 0.0f : c;
}

__global__ void __launch_bounds__(kBlock, kMinBlocksTension)
    k_tension(const DevParams P, const NbrView V, const PassArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  uint4 recp;
  float4 cp;
  ld_nv(a.nv, p, recp, cp);
  const float rp = nr_w(recp);
  const float kcoh = -20.0f * P.gamma * P.m * P.m;
  const float kcur = -P.gamma * P.m;
  // colour of each neighbour fetched with its record; the self terms of the
  // padding slots vanish (d = 0, c_p - c_q = 0)
  // the spline's norm and 2^-k for d in fixed-point units (exact)
  const float kcoh_fx = kcoh * P.C_norm * P.fx_inv;
  const float h3 = P.h * P.h * P.h;
  const float h6_64 = h3 * h3 * (1.0f / 64.0f);
  const float two_rho0 = 2.0f * P.rho0;
  // kcur (c_p - c_q) = kcur c_p - kcur c_q
  const float kpx = kcur * cp.x, kpy = kcur * cp.y, kpz = kcur * cp.z;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  for_each_neighbor_nv<kNbrBatch, true>(V, a.nv, p, [&](int, const uint4 rq, const float4 cq) {
    const float dx = (float)(int)(recp.x - rq.x);
    const float dy = (float)(int)(recp.y - rq.y);
    const float dz = (float)(int)(recp.z - rq.z);
    const float r2 = __fmul_rn(norm2(dx, dy, dz), P.fx_inv2);
    float r, rinv;
    floored_r(P, r2, r, rinv);
    const float coh = kcoh_fx * cohesion_unnormed(P, r, h6_64) * rinv;
    const float K = two_rho0 * rcp_fast(rp + nr_w(rq));
    fx = fmaf(K, fmaf(coh, dx, fmaf(-kcur, cq.x, kpx)), fx);
    fy = fmaf(K, fmaf(coh, dy, fmaf(-kcur, cq.y, kpy)), fy);
    fz = fmaf(K, fmaf(coh, dz, fmaf(-kcur, cq.z, kpz)), fz);
  });
  float4 v = a.vel[p];
  const float s = P.dt / rp;
  v.x = fmaf(s, fx, v.x);
  v.y = fmaf(s, fy, v.y);
  v.z = fmaf(s, fz, v.z);
  a.vel[p] = v;
  if (a.nv_out) st_nv(a.nv_out, p, recp, v);
}

__global__ void __launch_bounds__(kBlock, kMinBlocksXsph)
    k_xsph(const DevParams P, const NbrView V, const PassArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  uint4 rp;
  float4 vp;
  ld_nv(a.nv, p, rp, vp);
  // sums of (v_q - v_p) t^3 / rho_q; the poly6 norm, m and c multiply them
  // once (the padding slots' v_q - v_p is 0)
  float sx = 0.f, sy = 0.f, sz = 0.f;
  for_each_neighbor_nv<kNbrBatch, true>(V, a.nv, p, [&](int, const uint4 rq, const float4 vq) {
    const Pair g = pair_nr(P, rp, rq);
    // particles.c:439 evaluates x^2 + y^2 * z^2 (kept unless xsph_exact)
    const float rr =
        P.xsph_exact ? g.r2
                     : fmaf(g.dx, g.dx, __fmul_rn(__fmul_rn(__fmul_rn(g.dy, g.dy), g.dz), g.dz));
    const float t = fmaxf(P.h2 - rr, 0.0f);
    const float w = __fmul_rn(__fmul_rn(__fmul_rn(t, t), t), rcp_fast(nr_w(rq)));
    sx = fmaf(vq.x - vp.x, w, sx);
    sy = fmaf(vq.y - vp.y, w, sy);
    sz = fmaf(vq.z - vp.z, w, sz);
  });
  const float cw = P.c_xsph * P.Wn_m;
  const float4 vn = make_float4(fmaf(cw, sx, vp.x), fmaf(cw, sy, vp.y), fmaf(cw, sz, vp.z), 0.0f);
  a.vel_out[p] = vn;
  if (a.nv_out) st_nv(a.nv_out, p, rp, vn);
  if (a.write_pos) {
    float4 xp, dp;
    ld_pd(a.pd, p, xp, dp);
    st_pd(a.pd_out, p,
          make_float4(__double2float_rn(xstar_d(xp.x, dp.x)),
                      __double2float_rn(xstar_d(xp.y, dp.y)),
                      __double2float_rn(xstar_d(xp.z, dp.z)), 0.0f),
          make_float4(0.f, 0.f, 0.f, nr_w(rp)));
  }
}

// With nr_out, also the records {X, |omega|} the confinement pass gathers
// (one 16-byte load per neighbour instead of a record and omega[q]).
__global__ void __launch_bounds__(kBlock, kMinBlocksVorticity)
    k_vorticity(const DevParams P, const NbrView V, const PassArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  uint4 rp;
  float4 vp;
  ld_nv(a.nv, p, rp, vp);
  // sums of (v_q - v_p) x c d with c = (h - r)^2 / r and d in fixed-point
  // units (r too); the spiky norm and 2^-2k multiply them once (the padding slots'
  // v_q - v_p and d are 0)
  float wx = 0.f, wy = 0.f, wz = 0.f;
  for_each_neighbor_nv<kNbrBatch, true>(V, a.nv, p, [&](int, const uint4 rq, const float4 vq) {
    const float dx = (float)(int)(rp.x - rq.x);
    const float dy = (float)(int)(rp.y - rq.y);
    const float dz = (float)(int)(rp.z - rq.z);
    float r2c, rinv;
    floored_r_fx(P, norm2(dx, dy, dz), r2c, rinv);
    const float hm = fx_hm(P, r2c, rinv);
    const float c = __fmul_rn(__fmul_rn(hm, hm), rinv);
    const float gx = __fmul_rn(c, dx), gy = __fmul_rn(c, dy), gz = __fmul_rn(c, dz);
    const float ux = vq.x - vp.x, uy = vq.y - vp.y, uz = vq.z - vp.z;
    wx = __fadd_rn(wx, fmaf(uy, gz, -__fmul_rn(uz, gy)));
    wy = __fadd_rn(wy, fmaf(uz, gx, -__fmul_rn(ux, gz)));
    wz = __fadd_rn(wz, fmaf(ux, gy, -__fmul_rn(uy, gx)));
  });
  const float sw = P.DWn * P.fx_inv2;
  wx *= sw;
  wy *= sw;
  wz *= sw;
  const float wm = sqrtf(norm2(wx, wy, wz));
  a.omega[p] = make_float4(wx, wy, wz, wm);
  if (a.nr_out) a.nr_out[p] = make_uint4(rp.x, rp.y, rp.z, __float_as_uint(wm));
}

// OW: a.nr carries |omega| as its payload (the vorticity pass's records);
// otherwise |omega_q| comes from omega[q].w.
template <bool OW>
__global__ void __launch_bounds__(kBlock, kMinBlocksConfinement)
    k_confinement(const DevParams P, const NbrView V, const PassArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  const uint4 rp = ld_nr(a.nr, p);
  // sums of |omega_q| (h - r)^2 / r d, d and r in fixed-point units; the
  // spiky norm and 2^-2k multiply them once (the padding slots' d is 0)
  float ex = 0.f, ey = 0.f, ez = 0.f;
  for_each_neighbor_nr<kNbrBatch, true>(V, a.nr, p, [&](int q, const uint4 rq) {
    const float dx = (float)(int)(rp.x - rq.x);
    const float dy = (float)(int)(rp.y - rq.y);
    const float dz = (float)(int)(rp.z - rq.z);
    float r2c, rinv;
    floored_r_fx(P, norm2(dx, dy, dz), r2c, rinv);
    const float hm = fx_hm(P, r2c, rinv);
    const float wq = OW ? nr_w(rq) : __ldg(a.omega + q).w;
    const float c = __fmul_rn(__fmul_rn(__fmul_rn(hm, hm), rinv), wq);
    ex = fmaf(c, dx, ex);
    ey = fmaf(c, dy, ey);
    ez = fmaf(c, dz, ez);
  });
  const float se = P.DWn * P.fx_inv2;
  ex *= se;
  ey *= se;
  ez *= se;
  const float em = fmaxf(sqrtf(norm2(ex, ey, ez)), P.rmin);
  const float nx = ex / em, ny = ey / em, nz = ez / em;
  const float4 w = __ldg(a.omega + p);
  const float s = P.dt * P.vort_eps / P.m;
  float4 v = a.vel[p];
  v.x = fmaf(s, fmaf(ny, w.z, -__fmul_rn(nz, w.y)), v.x);
  v.y = fmaf(s, fmaf(nz, w.x, -__fmul_rn(nx, w.z)), v.y);
  v.z = fmaf(s, fmaf(nx, w.y, -__fmul_rn(ny, w.x)), v.z);
  a.vel[p] = v;
  if (a.write_pos) {
    float4 xp, dp;
    ld_pd(a.pd, p, xp, dp);
    st_pd(a.pd_out, p,
          make_float4(__double2float_rn(xstar_d(xp.x, dp.x)),
                      __double2float_rn(xstar_d(xp.y, dp.y)),
                      __double2float_rn(xstar_d(xp.z, dp.z)), 0.0f),
          make_float4(0.f, 0.f, 0.f, OW ? 0.0f : nr_w(rp)));
  }
}

__global__ void __launch_bounds__(kBlock) k_gravity(const DevParams P, float4* vel) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  float4 v = vel[p];
  if (P.gaxis == 0) v.x = __fadd_rn(v.x, P.gdt_f);
  else if (P.gaxis == 1) v.y = __fadd_rn(v.y, P.gdt_f);
  else v.z = __fadd_rn(v.z, P.gdt_f);
  vel[p] = v;
}

__global__ void __launch_bounds__(kBlock)
    k_predict(const DevParams P, PD* pd, const float4* __restrict__ vel) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  const float4 x = pd[p].x, v = vel[p];
  double xs = __dadd_rn((double)x.x, __dmul_rn((double)v.x, P.dt_d));
  double ys = __dadd_rn((double)x.y, __dmul_rn((double)v.y, P.dt_d));
  double zs = __dadd_rn((double)x.z, __dmul_rn((double)v.z, P.dt_d));
  xs = clamp_axis(xs, P.bmin[0], P.bmax[0], P.bmax_eps[0]);
  ys = clamp_axis(ys, P.bmin[1], P.bmax[1], P.bmax_eps[1]);
  zs = clamp_axis(zs, P.bmin[2], P.bmax[2], P.bmax_eps[2]);
  const float w = pd[p].d.w;
  pd[p].d = make_float4(__double2float_rn(__dsub_rn(xs, (double)x.x)),
                        __double2float_rn(__dsub_rn(ys, (double)x.y)),
                        __double2float_rn(__dsub_rn(zs, (double)x.z)), w);
}

__global__ void __launch_bounds__(kBlock)
    k_update_velocities(const DevParams P, const PD* __restrict__ pd,
                        float4* __restrict__ vel, const float* __restrict__ w_src,
                        uint4* __restrict__ nr) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  if (nr) nr[p].w = __float_as_uint(w_src[p]);
  const float4 d = pd[p].d;
  float vx = __double2float_rn(__ddiv_rn((double)d.x, P.dt_d));
  float vy = __double2float_rn(__ddiv_rn((double)d.y, P.dt_d));
  float vz = __double2float_rn(__ddiv_rn((double)d.z, P.dt_d));
  vx = fminf(fmaxf(vx, -P.v_max), P.v_max);
  vy = fminf(fmaxf(vy, -P.v_max), P.v_max);
  vz = fminf(fmaxf(vz, -P.v_max), P.v_max);
  vel[p] = make_float4(vx, vy, vz, 0.0f);
}

__global__ void __launch_bounds__(kBlock)
    k_update_positions(const DevParams P, PD* pd) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  const float4 x = pd[p].x;
  const float4 d = pd[p].d;
  const float nx = __double2float_rn(xstar_d(x.x, d.x));
  const float ny = __double2float_rn(xstar_d(x.y, d.y));
  const float nz = __double2float_rn(xstar_d(x.z, d.z));
  pd[p].x = make_float4(nx, ny, nz, 0.0f);
  // keep x* unchanged: d' = x* - x_new (exactly representable residue)
  pd[p].d = make_float4(__double2float_rn(__dsub_rn(xstar_d(x.x, d.x), (double)nx)),
                        __double2float_rn(__dsub_rn(xstar_d(x.y, d.y), (double)ny)),
                        __double2float_rn(__dsub_rn(xstar_d(x.z, d.z), (double)nz)), d.w);
}

__global__ void __launch_bounds__(kBlock)
    k_pack_w(const DevParams P, PD* pd, uint4* nr, const float* __restrict__ src) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  const float w = src[p];
  if (pd) pd[p].d.w = w;
  if (nr) nr[p].w = __float_as_uint(w);
}

// 16-byte records from the particle records: canonical x* = x + d and the
// payload src[p] (d.w without src).
__global__ void __launch_bounds__(kBlock)
    k_make_nr(const DevParams P, const PD* __restrict__ pd, const float* __restrict__ src,
              uint4* __restrict__ nr) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  const float4 x = pd[p].x, d = pd[p].d;
  nr[p] = make_nr(P, xstar_d(x.x, d.x), xstar_d(x.y, d.y), xstar_d(x.z, d.z),
                  src ? src[p] : d.w);
}

__global__ void __launch_bounds__(kBlock)
    k_collisions_double(const DevParams P, double* x, double* y, double* z, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a = x[i], b = y[i], c = z[i];
  if (sdf_collide(P, a, b, c)) {
    x[i] = a;
    y[i] = b;
    z[i] = c;
  }
}

}  // namespace

void launch_density_lambda(const DevParams& P, const NbrView& V, const PassArgs& a, int mode,
                           bool residual, cudaStream_t st) {
  const int g = grid_for(P.n);
  if (mode == 0) {
    if (residual) k_density_lambda<0, true><<<g, kBlock, 0, st>>>(P, V, a);
    else k_density_lambda<0, false><<<g, kBlock, 0, st>>>(P, V, a);
  } else if (mode == 1) {
    if (residual) k_density_lambda<1, true><<<g, kBlock, 0, st>>>(P, V, a);
    else k_density_lambda<1, false><<<g, kBlock, 0, st>>>(P, V, a);
  } else {
    k_density_lambda<2, false><<<g, kBlock, 0, st>>>(P, V, a);
  }
}

void launch_features(const DevParams& P, const NbrView& V, const PassArgs& a, float* feat,
                     int limit, cudaStream_t st) {
  k_features<true><<<grid_for(P.n), kBlock, 0, st>>>(P, V, a, feat, nullptr, nullptr, limit);
}

void launch_features_bf16(const DevParams& P, const NbrView& V, const PassArgs& a,
                          __nv_bfloat16* xbf, const float* norm, cudaStream_t st) {
  k_features<false><<<grid_for(P.n), kBlock, 0, st>>>(P, V, a, nullptr, xbf, norm, P.n);
}

void launch_accum_lambda(const uint4* rec, float s, float* target, int limit, cudaStream_t st) {
  if (limit > 0) k_accum_lambda<<<(limit + kBlock - 1) / kBlock, kBlock, 0, st>>>(rec, s, target, limit);
}

void launch_position(const DevParams& P, const NbrView& V, const PassArgs& a, int mode,
                     cudaStream_t st) {
  const int g = grid_for(P.n);
  const int sn = P.scorr_k != 0.0f ? (P.scorr_n == 4 ? 4 : -1) : 0;
  const bool sdf = P.has_sdf != 0;
#define SPHPC_POS(M, N, S) k_position<M, N, S><<<g, kBlock, 0, st>>>(P, V, a)
  if (mode == 0) {
    if (sn == 0) { if (sdf) SPHPC_POS(0, 0, true); else SPHPC_POS(0, 0, false); }
    else if (sn == 4) { if (sdf) SPHPC_POS(0, 4, true); else SPHPC_POS(0, 4, false); }
    else { if (sdf) SPHPC_POS(0, -1, true); else SPHPC_POS(0, -1, false); }
  } else {
    if (sn == 0) SPHPC_POS(1, 0, false);
    else if (sn == 4) SPHPC_POS(1, 4, false);
    else SPHPC_POS(1, -1, false);
  }
#undef SPHPC_POS
}

void launch_apply_dp(const DevParams& P, const PassArgs& a, cudaStream_t st) {
  if (P.has_sdf) k_apply_dp<true><<<grid_for(P.n), kBlock, 0, st>>>(P, a);
  else k_apply_dp<false><<<grid_for(P.n), kBlock, 0, st>>>(P, a);
}

void launch_pack_nv(int n, const uint4* nr, const float4* e, NV* nv, cudaStream_t st) {
  if (n > 0) k_pack_nv<<<grid_for(n), kBlock, 0, st>>>(n, nr, e, nv);
}
void launch_color(const DevParams& P, const NbrView& V, const PassArgs& a, cudaStream_t st) {
  k_color<<<grid_for(P.n), kBlock, 0, st>>>(P, V, a);
}
void launch_tension(const DevParams& P, const NbrView& V, const PassArgs& a, cudaStream_t st) {
  k_tension<<<grid_for(P.n), kBlock, 0, st>>>(P, V, a);
}
void launch_xsph(const DevParams& P, const NbrView& V, const PassArgs& a, cudaStream_t st) {
  k_xsph<<<grid_for(P.n), kBlock, 0, st>>>(P, V, a);
}
void launch_vorticity(const DevParams& P, const NbrView& V, const PassArgs& a, cudaStream_t st) {
  k_vorticity<<<grid_for(P.n), kBlock, 0, st>>>(P, V, a);
}
void launch_confinement(const DevParams& P, const NbrView& V, const PassArgs& a, bool omega_in_nr,
                        cudaStream_t st) {
  if (omega_in_nr) k_confinement<true><<<grid_for(P.n), kBlock, 0, st>>>(P, V, a);
  else k_confinement<false><<<grid_for(P.n), kBlock, 0, st>>>(P, V, a);
}
void launch_gravity(const DevParams& P, float4* vel, cudaStream_t st) {
  k_gravity<<<grid_for(P.n), kBlock, 0, st>>>(P, vel);
}
void launch_predict(const DevParams& P, PD* pd, const float4* vel, cudaStream_t st) {
  k_predict<<<grid_for(P.n), kBlock, 0, st>>>(P, pd, vel);
}
void launch_update_velocities(const DevParams& P, const PD* pd, float4* vel, cudaStream_t st,
                              const float* w_src, uint4* nr) {
  k_update_velocities<<<grid_for(P.n), kBlock, 0, st>>>(P, pd, vel, w_src, nr);
}
void launch_update_positions(const DevParams& P, PD* pd, cudaStream_t st) {
  k_update_positions<<<grid_for(P.n), kBlock, 0, st>>>(P, pd);
}
void launch_pack_w(const DevParams& P, PD* pd, uint4* nr, const float* src, cudaStream_t st) {
  k_pack_w<<<grid_for(P.n), kBlock, 0, st>>>(P, pd, nr, src);
}
void launch_make_nr(const DevParams& P, const PD* pd, const float* src, uint4* nr,
                    cudaStream_t st) {
  k_make_nr<<<grid_for(P.n), kBlock, 0, st>>>(P, pd, src, nr);
}
void launch_collisions_double(const DevParams& P, double* x, double* y, double* z, int n,
                              cudaStream_t st) {
  k_collisions_double<<<grid_for(n), kBlock, 0, st>>>(P, x, y, z, n);
}

}  // namespace sphpc
