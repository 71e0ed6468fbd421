// grid.cu -- uniform-grid hashing, particle reorder, cell-start table and the
// neighbour build of the PBF pipeline.
#include <cstdlib>
#include <cstring>

#include "kernels.cuh"

namespace sphpc {

namespace {

// Canonical predicted position of one particle.  predict: ApplyGravity then
// PredictPositions (particles.c:516-527, 766-782) evaluated in FP64 exactly
// as the reference does, then the box clamp (particles.c:842-867); the
// displacement d = x* - x is rounded to FP32 and x* := fl64(x + d).
__device__ __forceinline__ void canonical_xstar(const DevParams& P, const float4 x,
                                                const float4 v, const float4 dgiven,
                                                bool predict, float4& d, double& xs,
                                                double& ys, double& zs) {
  if (predict) {
    double vx = (double)v.x, vy = (double)v.y, vz = (double)v.z;
    if (P.gaxis == 0) vx = __dadd_rn(vx, P.gdt_d);
    else if (P.gaxis == 1) vy = __dadd_rn(vy, P.gdt_d);
    else vz = __dadd_rn(vz, P.gdt_d);
    xs = __dadd_rn((double)x.x, __dmul_rn(vx, P.dt_d));
    ys = __dadd_rn((double)x.y, __dmul_rn(vy, P.dt_d));
    zs = __dadd_rn((double)x.z, __dmul_rn(vz, P.dt_d));
    xs = clamp_axis(xs, P.bmin[0], P.bmax[0], P.bmax_eps[0]);
    ys = clamp_axis(ys, P.bmin[1], P.bmax[1], P.bmax_eps[1]);
    zs = clamp_axis(zs, P.bmin[2], P.bmax[2], P.bmax_eps[2]);
    d = make_float4(__double2float_rn(__dsub_rn(xs, (double)x.x)),
                    __double2float_rn(__dsub_rn(ys, (double)x.y)),
                    __double2float_rn(__dsub_rn(zs, (double)x.z)), 0.0f);
  } else {
    d = dgiven;
  }
  xs = xstar_d(x.x, d.x);
  ys = xstar_d(x.y, d.y);
  zs = xstar_d(x.z, d.z);
}

__device__ __forceinline__ void grid_cell(const DevParams& P, double xs, double ys, double zs,
                                          int& cx, int& cy, int& cz) {
  cx = grid_coord(xs, P.hd);
  cy = grid_coord(ys, P.hd);
  cz = grid_coord(zs, P.hd);
}

// HashVal, neighbors.c:94-95 (unsigned arithmetic)
__device__ __forceinline__ uint32_t cell_key(const DevParams& P, int cx, int cy, int cz) {
  return (uint32_t)P.nx * (uint32_t)P.ny * (uint32_t)cz +
         ((uint32_t)cy * (uint32_t)P.nx + (uint32_t)cx);
}

__device__ __forceinline__ uint32_t pack_cell(const DevParams& P, int cx, int cy, int cz) {
  return (uint32_t)cx | ((uint32_t)cy << P.bx) | ((uint32_t)cz << (P.bx + P.by));
}

__global__ void __launch_bounds__(kBlock)
    k_hash(const DevParams P, const PD* __restrict__ pd, const float4* __restrict__ vel,
           const uint32_t* __restrict__ ids,
           uint32_t* __restrict__ keys_by_id, uint32_t* __restrict__ loc_by_id,
           uint32_t* __restrict__ hist, int passes, int predict, uint32_t* __restrict__ err) {
  __shared__ uint32_t s_hist[kMaxPasses * kRadix];
  for (int i = threadIdx.x; i < kMaxPasses * kRadix; i += blockDim.x) s_hist[i] = 0;
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < P.n) {
    float4 x, dg;
    ld_pd(pd, i, x, dg);
    const float4 v = predict ? __ldg(vel + i) : make_float4(0.f, 0.f, 0.f, 0.f);
    float4 d;
    double xs, ys, zs;
    canonical_xstar(P, x, v, dg, predict != 0, d, xs, ys, zs);
    int cx, cy, cz;
    grid_cell(P, xs, ys, zs, cx, cy, cz);
    uint32_t key = cell_key(P, cx, cy, cz);
    if (key >= P.ncells || cx >= P.nx || cy >= P.ny || cz >= P.nz) {
      atomicOr(err, kErrCellRange);
      key = P.ncells - 1;
    }
    const uint32_t id = __ldg(ids + i);
    keys_by_id[id] = key;
    loc_by_id[id] = (uint32_t)i;
    count_key_digits(s_hist, key, passes);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < passes * kRadix; k += blockDim.x)
    if (s_hist[k]) atomicAdd(hist + k, s_hist[k]);
}

__global__ void __launch_bounds__(kBlock)
    k_reorder(const DevParams P, const uint32_t* __restrict__ sorted_ids,
              const uint32_t* __restrict__ loc_by_id, const PD* __restrict__ pd_in,
              const float4* __restrict__ vel_in, PD* __restrict__ pd_out,
              float4* __restrict__ vel_out, float4* __restrict__ xsa, uint4* __restrict__ nr_out,
              uint32_t* __restrict__ cellp, int predict, int move_vel, ReorderExtra ex) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= P.n) return;
  const uint32_t id = __ldg(sorted_ids + j);
  const uint32_t src = __ldg(loc_by_id + id);
  float4 x, dg;
  ld_pd(pd_in, (int)src, x, dg);
  float4 v = (predict || move_vel) ? __ldg(vel_in + src) : make_float4(0.f, 0.f, 0.f, 0.f);
  float4 d;
  double xs, ys, zs;
  canonical_xstar(P, x, v, dg, predict != 0, d, xs, ys, zs);
  int cx, cy, cz;
  grid_cell(P, xs, ys, zs, cx, cy, cz);
  cx = min(cx, P.nx - 1);
  cy = min(cy, P.ny - 1);
  cz = min(cz, P.nz - 1);
  d.w = predict ? 0.0f : dg.w;
  st_pd(pd_out, j, x, d);
  xsa[j] = make_float4((float)xs, (float)ys, (float)zs, 0.0f);
  nr_out[j] = make_nr(P, xs, ys, zs, d.w);
  cellp[j] = pack_cell(P, cx, cy, cz);
  if (move_vel) {
    if (predict) {
      // the velocity after ApplyGravity, as the reference holds it
      if (P.gaxis == 0) v.x = __fadd_rn(v.x, P.gdt_f);
      else if (P.gaxis == 1) v.y = __fadd_rn(v.y, P.gdt_f);
      else v.z = __fadd_rn(v.z, P.gdt_f);
    }
    vel_out[j] = v;
  }
#pragma unroll
  for (int k = 0; k < 6; ++k)
    if (ex.in4[k]) ex.out4[k][j] = __ldg(ex.in4[k] + src);
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (ex.in1[k]) ex.out1[k][j] = __ldg(ex.in1[k] + src);
  if (ex.nr_carry) ex.nr_carry[j] = make_nr(P, xs, ys, zs, __ldg(ex.carry_src + src));
}

constexpr int kSmallGap = 32;
constexpr int64_t kGapChunk = 4096;  // worklist entries cover at most this many cells

__device__ __forceinline__ void push_gap(int64_t lo, int64_t hi, uint32_t val, uint4* gaps,
                                         uint32_t* gap_count) {
  const int64_t pieces = (hi - lo + kGapChunk) / kGapChunk;
  const uint32_t g = atomicAdd(gap_count, (uint32_t)pieces);
  for (int64_t k = 0; k < pieces; ++k) {
    const int64_t a = lo + k * kGapChunk;
    const int64_t b = min(hi, a + kGapChunk - 1);
    gaps[g + k] = make_uint4((uint32_t)a, (uint32_t)b, val, 0u);
  }
}

// start[c] = lower_bound(keys, c): the first slot j of every non-empty key
// writes j into the cells (key[j-1], key[j]]; long runs of empty cells go to
// a worklist filled by k_fill_gaps.
__global__ void __launch_bounds__(kBlock)
    k_cell_starts(const uint32_t* __restrict__ keys, int n, uint32_t ncells,
                  uint32_t* __restrict__ cstart, uint4* __restrict__ gaps,
                  uint32_t* __restrict__ gap_count, uint32_t* __restrict__ err) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int64_t k = (int64_t)__ldg(keys + j);
  const int64_t kp = j > 0 ? (int64_t)__ldg(keys + j - 1) : -1;
  if (k >= (int64_t)ncells) {
    atomicOr(err, kErrCellRange);
    return;
  }
  if (k != kp) {
    const int64_t lo = kp + 1, hi = k;  // inclusive
    if (hi - lo + 1 <= kSmallGap) {
      for (int64_t c = lo; c <= hi; ++c) cstart[c] = (uint32_t)j;
    } else {
      push_gap(lo, hi, (uint32_t)j, gaps, gap_count);
    }
  }
  if (j == n - 1) {
    const int64_t lo = k + 1, hi = (int64_t)ncells;  // includes the sentinel cstart[C]
    if (hi - lo + 1 <= kSmallGap) {
      for (int64_t c = lo; c <= hi; ++c) cstart[c] = (uint32_t)n;
    } else {
      push_gap(lo, hi, (uint32_t)n, gaps, gap_count);
    }
  }
}

__global__ void __launch_bounds__(kBlock)
    k_fill_gaps(const uint4* __restrict__ gaps, const uint32_t* __restrict__ gap_count,
                uint32_t* __restrict__ cstart) {
  const uint32_t ng = *gap_count;
  for (uint32_t g = blockIdx.x; g < ng; g += gridDim.x) {
    const uint4 e = gaps[g];
    for (uint64_t c = (uint64_t)e.x + threadIdx.x; c <= (uint64_t)e.y; c += blockDim.x)
      cstart[c] = e.z;
  }
}

// FillNeighbors' validity test and HashVal coordinate of one shifted axis
// value (neighbors.c:252-263).
__device__ __forceinline__ bool shifted_coord(double x, double h, int nmax, int& g) {
  const double f = floor(__ddiv_rn(x, h));
  if (f > (double)(nmax - 1) || x < 0.0) return false;
  g = (int)(unsigned)f;
  return true;
}

__device__ __forceinline__ bool axis_regular(double x, double h, int c, int nmax) {
  int g;
  const bool vm = shifted_coord(__dadd_rn(x, -h), h, nmax, g);
  const bool okm = vm ? (g == c - 1) : (c == 0);
  const bool vp = shifted_coord(__dadd_rn(x, h), h, nmax, g);
  const bool okp = vp ? (g == c + 1) : (c == nmax - 1);
  return okm && okp;
}

struct BuildCtx {
  float4 xf;              // x* as FP32 (candidate pre-test)
  float4 xp, dp;          // exact representation x + d
  double xs, ys, zs;      // canonical double x*
  float h2lo, h2hi;
  double h2d;
};

// r^2 < h^2 exactly as neighbors.c:278-285 evaluates it on the canonical
// double positions.  The FP32 absolute positions decide every pair whose r^2
// lies outside the band [P.bld_h2lo, P.bld_h2hi] = h^2 (1 -+ 2^-10); the FP64
// test decides the rest.  The host opens the band to every pair when FP32
// rounding of the grid's largest coordinate could move r^2 by that much
// (sphpc_neighbor_pretest_fp32_safe: beyond about 2^12 h).
__device__ __forceinline__ bool exact_neighbor(const BuildCtx& c, const PD* __restrict__ pd,
                                            int j) {
  float4 xq, dq;
  ld_pd(pd, j, xq, dq);
  const double ddx = __dsub_rn(c.xs, xstar_d(xq.x, dq.x));
  const double ddy = __dsub_rn(c.ys, xstar_d(xq.y, dq.y));
  const double ddz = __dsub_rn(c.zs, xstar_d(xq.z, dq.z));
  const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)),
                              __dmul_rn(ddz, ddz));
  return r2 < c.h2d;
}

__device__ __forceinline__ bool is_neighbor(const BuildCtx& c, const PD* __restrict__ pd,
                                            const float4* __restrict__ xsa, int j) {
  const float4 q = __ldg(xsa + j);
  const float fx = c.xf.x - q.x, fy = c.xf.y - q.y, fz = c.xf.z - q.z;
  const float r2f = fx * fx + fy * fy + fz * fz;
  if (r2f < c.h2lo) return true;
  if (r2f > c.h2hi) return false;
  return exact_neighbor(c, pd, j);
}

// FillNeighbors' 27-cell walk (neighbors.c:247-295) verbatim, for a
// particle whose neighbour cells are not cx-1..cx+1 (FP64 rounding at a cell
// face): its bucket goes to out[count * stride]; returns the count.
__device__ __forceinline__ int walk_27_cells(const DevParams& P, const NbrView& V, const BuildCtx& c,
                                          const PD* __restrict__ pd,
                                          const float4* __restrict__ xsa, int p,
                                          uint32_t* __restrict__ out, size_t stride) {
  int count = 0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        int gx, gy, gz;
        if (!shifted_coord(__dadd_rn(c.xs, (double)dx * P.hd), P.hd, P.nx, gx)) continue;
        if (!shifted_coord(__dadd_rn(c.ys, (double)dy * P.hd), P.hd, P.ny, gy)) continue;
        if (!shifted_coord(__dadd_rn(c.zs, (double)dz * P.hd), P.hd, P.nz, gz)) continue;
        const uint32_t key = (uint32_t)P.nx * (uint32_t)P.ny * (uint32_t)gz +
                             ((uint32_t)gy * (uint32_t)P.nx + (uint32_t)gx);
        if (key >= P.ncells) continue;
        const int b = (int)__ldg(V.cstart + key);
        const int e = (int)__ldg(V.cstart + key + 1);
        for (int j = b; j < e && count < kMaxNeighbors; ++j) {
          if (j != p && is_neighbor(c, pd, xsa, j)) out[(size_t)(count++) * stride] = (uint32_t)j;
        }
      }
  return count;
}

constexpr int kBuildBlock = 128;

// FillNeighbors, neighbors.c:217-298: one thread per particle, bucket entries
// written as they are found into column nbr[count][p] (L2 merges the partial
// lines of a warp's columns).
__global__ void __launch_bounds__(kBuildBlock, 10)
    k_build_neighbors(const DevParams P, const NbrView V, const PD* __restrict__ pd,
                      const float4* __restrict__ xsa, const uint32_t* __restrict__ cellp,
                      uint32_t* __restrict__ nbr, uint8_t* __restrict__ ncount) {
  const int p = blockIdx.x * kBuildBlock + threadIdx.x;
  if (p >= P.n) return;
  BuildCtx c;
  ld_pd(pd, p, c.xp, c.dp);
  c.xf = __ldg(xsa + p);
  c.xs = xstar_d(c.xp.x, c.dp.x);
  c.ys = xstar_d(c.xp.y, c.dp.y);
  c.zs = xstar_d(c.xp.z, c.dp.z);
  c.h2lo = P.bld_h2lo;
  c.h2hi = P.bld_h2hi;
  c.h2d = P.h2d;
  int cx, cy, cz;
  unpack_cell(V, __ldg(cellp + p), cx, cy, cz);
  const bool regular = axis_regular(c.xs, P.hd, cx, P.nx) &&
                       axis_regular(c.ys, P.hd, cy, P.ny) &&
                       axis_regular(c.zs, P.hd, cz, P.nz);
  uint32_t* out = nbr + p;
  const size_t stride = (size_t)P.n;
  int count = 0;
  if (regular) {
    // rows (dz, dy) of cells cx-1..cx+1 are contiguous slot ranges
    const int xlo = cx - (cx > 0);
    const int xhi = cx + (cx < P.nx - 1);
    for (int dz = -1; dz <= 1; ++dz) {
      const int z = cz + dz;
      if ((unsigned)z >= (unsigned)P.nz) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int y = cy + dy;
        if ((unsigned)y >= (unsigned)P.ny) continue;
        const uint32_t rk = (uint32_t)z * P.nxny + (uint32_t)y * (uint32_t)P.nx;
        const int b = (int)__ldg(V.cstart + rk + xlo);
        const int e = (int)__ldg(V.cstart + rk + xhi + 1);
        // self can only appear in the particle's own row
        const bool self_row = dz == 0 && dy == 0;
        int j = b;
        for (; j + 4 <= e; j += 4) {
          // hit and band masks of four candidates without branches; the exact
          // test only for the rare in-band bits, then the hits in order
          uint32_t hit = 0u, band = 0u;
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const float4 q = __ldg(xsa + j + u);
            const float fx = c.xf.x - q.x, fy = c.xf.y - q.y, fz = c.xf.z - q.z;
            const float r2 = fx * fx + fy * fy + fz * fz;
            hit |= (uint32_t)(r2 <= c.h2hi) << u;
            band |= (uint32_t)(r2 >= c.h2lo) << u;
          }
          if (self_row && (unsigned)(p - j) < 4u) hit &= ~(1u << (p - j));
          band &= hit;
          if (band) {
#pragma unroll
            for (int u = 0; u < 4; ++u)
              if (((band >> u) & 1u) && !exact_neighbor(c, pd, j + u)) hit &= ~(1u << u);
          }
          while (hit) {
            const int u = __ffs(hit) - 1;
            hit &= hit - 1u;
            out[(size_t)count * stride] = (uint32_t)(j + u);
            if (++count == kMaxNeighbors) goto done;
          }
        }
        for (; j < e; ++j) {
          const float4 q = __ldg(xsa + j);
          const float fx = c.xf.x - q.x, fy = c.xf.y - q.y, fz = c.xf.z - q.z;
          const float r2 = fx * fx + fy * fy + fz * fz;
          if (r2 > c.h2hi || (self_row && j == p)) continue;
          if (r2 >= c.h2lo && !exact_neighbor(c, pd, j)) continue;
          out[(size_t)count * stride] = (uint32_t)j;
          if (++count == kMaxNeighbors) goto done;
        }
      }
    }
  } else {
    count = walk_27_cells(P, V, c, pd, xsa, p, out, stride);
  }
done:
  ncount[p] = (uint8_t)count;
}

// ---------------------------------------------------------------------------
// Staged neighbour build (FillNeighbors, neighbors.c:217-298): one thread per
// particle walks its 9 (dz, dy) slot rows as k_build_neighbors does, but
// appends every candidate without branches to its own column of a
// shared-memory staging area (store the slot, advance the count on a hit;
// the particle itself is skipped by splitting its own row), and the block
// writes the buckets out at the end as whole columns of nbr[60][n]: for each
// entry index, a warp's 32 consecutive slots are one 128-byte line.
// ---------------------------------------------------------------------------
constexpr int kStagedBlock = 128;

__device__ __forceinline__ void staged_range(const BuildCtx& c, const PD* __restrict__ pd,
                                             const float4* __restrict__ xsa, int ja, int jb,
                                             uint32_t* __restrict__ stg, int& cnt) {
  int j = ja;
  for (; j + 4 <= jb && cnt <= kMaxNeighbors - 4; j += 4) {
    float4 q[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) q[u] = __ldg(xsa + j + u);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const float fx = c.xf.x - q[u].x, fy = c.xf.y - q[u].y, fz = c.xf.z - q[u].z;
      const float r2 = fx * fx + fy * fy + fz * fz;
      bool hit = r2 <= c.h2hi;
      if (hit && r2 >= c.h2lo) hit = exact_neighbor(c, pd, j + u);
      stg[cnt * kStagedBlock] = (uint32_t)(j + u);
      cnt += hit ? 1 : 0;
    }
  }
  for (; j < jb && cnt < kMaxNeighbors; ++j) {
    const float4 q = __ldg(xsa + j);
    const float fx = c.xf.x - q.x, fy = c.xf.y - q.y, fz = c.xf.z - q.z;
    const float r2 = fx * fx + fy * fy + fz * fz;
    bool hit = r2 <= c.h2hi;
    if (hit && r2 >= c.h2lo) hit = exact_neighbor(c, pd, j);
    stg[cnt * kStagedBlock] = (uint32_t)j;
    cnt += hit ? 1 : 0;
  }
}

__global__ void __launch_bounds__(kStagedBlock)
    k_build_staged(const DevParams P, const NbrView V, const PD* __restrict__ pd,
                   const float4* __restrict__ xsa, const uint32_t* __restrict__ cellp,
                   uint32_t* __restrict__ nbr, uint8_t* __restrict__ ncount) {
  __shared__ uint32_t s_stage[kMaxNeighbors * kStagedBlock];
  const int p = blockIdx.x * kStagedBlock + threadIdx.x;
  if (p >= P.n) return;
  uint32_t* stg = s_stage + threadIdx.x;
  const size_t stride = (size_t)P.n;
  BuildCtx c;
  ld_pd(pd, p, c.xp, c.dp);
  c.xf = __ldg(xsa + p);
  c.xs = xstar_d(c.xp.x, c.dp.x);
  c.ys = xstar_d(c.xp.y, c.dp.y);
  c.zs = xstar_d(c.xp.z, c.dp.z);
  c.h2lo = P.bld_h2lo;
  c.h2hi = P.bld_h2hi;
  c.h2d = P.h2d;
  int cx, cy, cz;
  unpack_cell(V, __ldg(cellp + p), cx, cy, cz);
  const bool regular = axis_regular(c.xs, P.hd, cx, P.nx) &&
                       axis_regular(c.ys, P.hd, cy, P.ny) &&
                       axis_regular(c.zs, P.hd, cz, P.nz);
  int count = 0;
  if (regular) {
    const int xlo = cx - (cx > 0);
    const int xhi = cx + (cx < P.nx - 1);
    for (int dz = -1; dz <= 1 && count < kMaxNeighbors; ++dz) {
      const int z = cz + dz;
      if ((unsigned)z >= (unsigned)P.nz) continue;
      for (int dy = -1; dy <= 1 && count < kMaxNeighbors; ++dy) {
        const int y = cy + dy;
        if ((unsigned)y >= (unsigned)P.ny) continue;
        const uint32_t rk = (uint32_t)z * P.nxny + (uint32_t)y * (uint32_t)P.nx;
        const int b = (int)__ldg(V.cstart + rk + xlo);
        const int e = (int)__ldg(V.cstart + rk + xhi + 1);
        if (dz == 0 && dy == 0) {
          staged_range(c, pd, xsa, b, p, stg, count);
          staged_range(c, pd, xsa, p + 1, e, stg, count);
        } else {
          staged_range(c, pd, xsa, b, e, stg, count);
        }
      }
    }
    for (int t = 0; t < count; ++t) nbr[(size_t)t * stride + p] = stg[t * kStagedBlock];
  } else {
    count = walk_27_cells(P, V, c, pd, xsa, p, nbr + p, stride);
  }
  ncount[p] = (uint8_t)count;
}

// ---------------------------------------------------------------------------
// Cell-cooperative neighbour build (FillNeighbors, neighbors.c:217-298).
//
// Regular particles of one cell share their candidate list: the 9 (dz, dy)
// rows of cells cx-1..cx+1, each a contiguous slot range, concatenated in the
// reference's order (dz, then dy, then dx and ascending sorted index).  One
// warp takes a window of 32 slots; for each run of particles of the same cell
// in the window (m particles), every particle gets L = 32 / m lanes and each
// lane tests a contiguous part of the list, so all lanes of the warp step
// through the same candidates in lockstep (one broadcast load serves the m
// particles) with no divergence between cells.  Hits are appended without
// branches to the lane's column of a shared-memory staging area; the parts'
// counts are prefix-summed within each particle, which puts the hits in the
// reference's order and truncates at 60 exactly as the per-candidate walk
// does; the buckets are then written as whole columns of nbr[60][n].
// Particles whose neighbour cells are not cx-1..cx+1 take the verbatim
// 27-cell walk on their own lane.
// ---------------------------------------------------------------------------
constexpr int kCoopWarps = 4;
constexpr int kRows = 9;

struct CoopRow {
  int b, e, off;  // slot range [b, e) at offset off of the concatenated list
};

// Tests slots [ja, jb) against the lane's particle, appending the hits (in
// slot order) to the lane's staging column stg[t * 32 + lane], t < 60.
__device__ __forceinline__ void coop_range(const BuildCtx& c, const PD* __restrict__ pd,
                                           const float4* __restrict__ xsa, int ja, int jb,
                                           uint32_t* __restrict__ stg, int lane, int& cnt) {
  int j = ja;
  // batches of four while four more entries fit below the cap
  for (; j + 4 <= jb && cnt <= kMaxNeighbors - 4; j += 4) {
    float4 q[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) q[u] = __ldg(xsa + j + u);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const float fx = c.xf.x - q[u].x, fy = c.xf.y - q[u].y, fz = c.xf.z - q[u].z;
      const float r2 = fx * fx + fy * fy + fz * fz;
      bool hit = r2 <= c.h2hi;
      if (hit && r2 >= c.h2lo) hit = exact_neighbor(c, pd, j + u);
      stg[cnt * 32 + lane] = (uint32_t)(j + u);
      cnt += hit ? 1 : 0;
    }
  }
  for (; j < jb && cnt < kMaxNeighbors; ++j) {
    const float4 q = __ldg(xsa + j);
    const float fx = c.xf.x - q.x, fy = c.xf.y - q.y, fz = c.xf.z - q.z;
    const float r2 = fx * fx + fy * fy + fz * fz;
    bool hit = r2 <= c.h2hi;
    if (hit && r2 >= c.h2lo) hit = exact_neighbor(c, pd, j);
    stg[cnt * 32 + lane] = (uint32_t)j;
    cnt += hit ? 1 : 0;
  }
}

// The lane's part [a, b) of the concatenated candidate list of particle p;
// the particle itself (in row 4, the (0, 0) row) is skipped.
__device__ __forceinline__ void coop_walk(const BuildCtx& c, const CoopRow* rows, int a, int b,
                                          int p, const PD* __restrict__ pd,
                                          const float4* __restrict__ xsa,
                                          uint32_t* __restrict__ stg, int lane, int& cnt) {
  int r = 0;
  while (r < kRows - 1 && rows[r + 1].off <= a) ++r;
  for (; a < b && r < kRows && cnt < kMaxNeighbors; ++r) {
    const CoopRow R = rows[r];
    const int end = min(b, R.off + (R.e - R.b));
    if (end <= a) continue;
    const int ja = R.b + (a - R.off), jb = R.b + (end - R.off);
    if (r == 4) {
      coop_range(c, pd, xsa, ja, min(jb, p), stg, lane, cnt);
      coop_range(c, pd, xsa, max(ja, p + 1), jb, stg, lane, cnt);
    } else {
      coop_range(c, pd, xsa, ja, jb, stg, lane, cnt);
    }
    a = end;
  }
}

__global__ void __launch_bounds__(kCoopWarps * 32)
    k_build_coop(const DevParams P, const NbrView V, const PD* __restrict__ pd,
                 const float4* __restrict__ xsa, const uint32_t* __restrict__ cellp,
                 uint32_t* __restrict__ nbr, uint8_t* __restrict__ ncount) {
  __shared__ uint32_t s_stage[kCoopWarps][kMaxNeighbors * 32];
  __shared__ CoopRow s_rows[kCoopWarps][kRows];
  __shared__ int s_off[kCoopWarps][32];
  constexpr uint32_t kAll = 0xffffffffu;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int win = (blockIdx.x * kCoopWarps + w) * 32;
  if (win >= P.n) return;  // the whole warp
  uint32_t* stg = s_stage[w];
  CoopRow* rows = s_rows[w];
  int* offs = s_off[w];
  const size_t stride = (size_t)P.n;

  // the lane's own slot: position, cell, and whether its neighbour cells are
  // cx-1..cx+1 on every axis
  const int s = win + lane;
  const bool valid = s < P.n;
  BuildCtx c;
  c.h2lo = P.bld_h2lo;
  c.h2hi = P.bld_h2hi;
  c.h2d = P.h2d;
  uint32_t cp = kAll;
  bool regular = false;
  if (valid) {
    ld_pd(pd, s, c.xp, c.dp);
    c.xf = __ldg(xsa + s);
    c.xs = xstar_d(c.xp.x, c.dp.x);
    c.ys = xstar_d(c.xp.y, c.dp.y);
    c.zs = xstar_d(c.xp.z, c.dp.z);
    cp = __ldg(cellp + s);
    int cx, cy, cz;
    unpack_cell(V, cp, cx, cy, cz);
    regular = axis_regular(c.xs, P.hd, cx, P.nx) && axis_regular(c.ys, P.hd, cy, P.ny) &&
              axis_regular(c.zs, P.hd, cz, P.nz);
  } else {
    c.xf = make_float4(0.f, 0.f, 0.f, 0.f);
    c.xs = c.ys = c.zs = 0.0;
  }
  const uint32_t vmask = __ballot_sync(kAll, valid);
  const int nv = __popc(vmask);  // valid lanes are a prefix of the warp
  const uint32_t cp_prev = __shfl_up_sync(kAll, cp, 1);
  uint32_t heads = __ballot_sync(kAll, valid && (lane == 0 || cp != cp_prev));

  while (heads) {
    const int r0 = __ffs(heads) - 1;
    heads &= heads - 1;
    const int r1 = heads ? __ffs(heads) - 1 : nv;
    const int m = r1 - r0;
    // the 9 rows of the run's cell and their offsets in the list
    const uint32_t rcp = __shfl_sync(kAll, cp, r0);
    int rb = 0, re = 0;
    if (lane < kRows) {
      int cx, cy, cz;
      unpack_cell(V, rcp, cx, cy, cz);
      const int z = cz + lane / 3 - 1, y = cy + lane % 3 - 1;
      if ((unsigned)z < (unsigned)P.nz && (unsigned)y < (unsigned)P.ny) {
        const uint32_t rk = (uint32_t)z * P.nxny + (uint32_t)y * (uint32_t)P.nx;
        const int xlo = cx - (cx > 0);
        const int xhi = cx + (cx < P.nx - 1);
        rb = (int)__ldg(V.cstart + rk + xlo);
        re = (int)__ldg(V.cstart + rk + xhi + 1);
      }
    }
    const int len = re - rb;
    int incl = len;
#pragma unroll
    for (int o = 1; o < 16; o <<= 1) {
      const int y = __shfl_up_sync(kAll, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane < kRows) rows[lane] = CoopRow{rb, re, incl - len};
    const int T = __shfl_sync(kAll, incl, kRows - 1);
    __syncwarp();

    // L lanes per particle; lane (i, k) tests part k of particle i's list
    const int L = 32 / m;
    const int i = lane / L, k = lane - (lane / L) * L;
    const bool act = i < m;
    const int src = r0 + (act ? i : 0);
    BuildCtx pc;
    pc.h2lo = c.h2lo;
    pc.h2hi = c.h2hi;
    pc.h2d = c.h2d;
    pc.xf.x = __shfl_sync(kAll, c.xf.x, src);
    pc.xf.y = __shfl_sync(kAll, c.xf.y, src);
    pc.xf.z = __shfl_sync(kAll, c.xf.z, src);
    pc.xs = __shfl_sync(kAll, c.xs, src);
    pc.ys = __shfl_sync(kAll, c.ys, src);
    pc.zs = __shfl_sync(kAll, c.zs, src);
    const bool preg = __shfl_sync(kAll, regular ? 1 : 0, src) != 0;
    const int pp = win + src;
    int cnt = 0;
    if (act && preg) {
      const int a = (int)((long long)T * k / L);
      const int b = (int)((long long)T * (k + 1) / L);
      coop_walk(pc, rows, a, b, pp, pd, xsa, stg, lane, cnt);
    }
    // where each part's hits start in its particle's bucket
    int incl2 = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kAll, incl2, o);
      if (lane >= o) incl2 += y;
    }
    const int before = __shfl_sync(kAll, incl2, act && i > 0 ? i * L - 1 : 0);
    const int base = act && i > 0 ? before : 0;
    const int last = __shfl_sync(kAll, incl2, act ? i * L + L - 1 : 0);
    offs[lane] = incl2 - cnt - base;
    const int pcount = act ? min(last - base, kMaxNeighbors) : 0;
    __syncwarp();
    // write-out: lane -> particle i2 = lane % m, entry e0 + lane / m
    const int maxc = __reduce_max_sync(kAll, (unsigned)pcount);
    const int i2 = lane % m;
    const int cnt2 = __shfl_sync(kAll, pcount, i2 * L);
    const bool wl = lane < m * L;
    for (int e0 = 0; e0 < maxc; e0 += L) {
      const int e = e0 + lane / m;
      if (wl && e < cnt2) {
        int lo = 0, hi = L - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (offs[i2 * L + mid] <= e) lo = mid;
          else hi = mid - 1;
        }
        const int kl = i2 * L + lo;
        nbr[(size_t)e * stride + (size_t)(win + r0 + i2)] = stg[(e - offs[kl]) * 32 + kl];
      }
    }
    if (act && k == 0 && preg) ncount[pp] = (uint8_t)pcount;
    __syncwarp();  // the staging area and rows belong to the next run
  }
  if (valid && !regular) {
    const int cnt = walk_27_cells(P, V, c, pd, xsa, s, nbr + s, stride);
    ncount[s] = (uint8_t)cnt;
  }
}

__global__ void __launch_bounds__(kBlock)
    k_export_buckets(const NbrView V, const uint32_t* __restrict__ ids,
                     uint32_t* __restrict__ nbr, int32_t* __restrict__ count) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= V.n) return;
  const uint32_t idp = __ldg(ids + p);
  uint32_t* out = nbr + (size_t)idp * kMaxNeighbors;
  int cnt = 0;
  for_each_neighbor(V, p, [&](int q) {
    if (cnt < kMaxNeighbors) out[cnt] = __ldg(ids + q);
    ++cnt;
  });
  for (int j = cnt; j < kMaxNeighbors; ++j) out[j] = 0u;
  count[idp] = cnt;
}

}  // namespace

void launch_hash(const DevParams& P, const PD* pd, const float4* vel, const uint32_t* ids,
                 uint32_t* keys_by_id, uint32_t* loc_by_id, uint32_t* hist, int passes,
                 bool predict, uint32_t* err, cudaStream_t st) {
  k_hash<<<grid_for(P.n), kBlock, 0, st>>>(P, pd, vel, ids, keys_by_id, loc_by_id, hist,
                                           passes, predict ? 1 : 0, err);
}

void launch_reorder(const DevParams& P, const uint32_t* sorted_ids, const uint32_t* loc_by_id,
                    const PD* pd_in, const float4* vel_in, PD* pd_out, float4* vel_out,
                    float4* xsa, uint4* nr_out, uint32_t* cellp, bool predict, bool move_vel,
                    const ReorderExtra* extra, cudaStream_t st) {
  ReorderExtra ex = {};
  if (extra) ex = *extra;
  k_reorder<<<grid_for(P.n), kBlock, 0, st>>>(P, sorted_ids, loc_by_id, pd_in, vel_in, pd_out,
                                              vel_out, xsa, nr_out, cellp, predict ? 1 : 0,
                                              move_vel ? 1 : 0, ex);
}

void launch_cell_starts(const uint32_t* keys_sorted, int n, uint32_t ncells, uint32_t* cstart,
                        uint4* gaps, uint32_t* gap_count, uint32_t* err, cudaStream_t st) {
  if (n == 0) {
    cudaMemsetAsync(cstart, 0, sizeof(uint32_t) * ((size_t)ncells + 1), st);
    return;
  }
  cudaMemsetAsync(gap_count, 0, sizeof(uint32_t), st);
  k_cell_starts<<<grid_for(n), kBlock, 0, st>>>(keys_sorted, n, ncells, cstart, gaps,
                                                 gap_count, err);
  k_fill_gaps<<<148 * 16, kBlock, 0, st>>>(gaps, gap_count, cstart);
}

void launch_build_neighbors(const DevParams& P, const NbrView& V, const PD* pd,
                            const float4* xsa, const uint32_t* cellp, uint32_t* nbr,
                            uint8_t* ncount, cudaStream_t st) {
  static const int build_kind = [] {
    const char* e = getenv("SPHPC_NEIGHBOR_BUILD");
    if (e && strcmp(e, "lane") == 0) return 1;
    if (e && strcmp(e, "staged") == 0) return 2;
    return 0;
  }();
  if (build_kind == 2) {
    k_build_staged<<<grid_for(P.n, kStagedBlock), kStagedBlock, 0, st>>>(P, V, pd, xsa, cellp,
                                                                          nbr, ncount);
    return;
  }
  if (build_kind == 1) {
    k_build_neighbors<<<grid_for(P.n, kBuildBlock), kBuildBlock, 0, st>>>(P, V, pd, xsa, cellp,
                                                                           nbr, ncount);
    return;
  }
  const int warps = (P.n + 31) / 32;
  k_build_coop<<<(warps + kCoopWarps - 1) / kCoopWarps, kCoopWarps * 32, 0, st>>>(
      P, V, pd, xsa, cellp, nbr, ncount);
}

void launch_export_buckets(const NbrView& V, const uint32_t* ids, uint32_t* nbr, int32_t* count,
                           cudaStream_t st) {
  k_export_buckets<<<grid_for(V.n), kBlock, 0, st>>>(V, ids, nbr, count);
}

}  // namespace sphpc
