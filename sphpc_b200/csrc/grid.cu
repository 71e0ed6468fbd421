// grid.cu -- uniform-grid hashing, particle reorder, cell-start table and the
// neighbour build of the PBF pipeline.
#include "kernels.cuh"

namespace sphpc {

namespace {

// x* as absolute FP32 for the neighbour build's candidate test, in pair
// blocks: slots 2b and 2b+1 share the 32 bytes {x0, x1, y0, y1, z0, z1, 0,
// 0} at float4 index 2b, so that the coordinates of a slot pair load as the
// 64-bit operands of the packed FP32x2 arithmetic of sm_100.
__device__ __forceinline__ void xsa_store(float4* xsa, int j, float x, float y, float z) {
  float* f = reinterpret_cast<float*>(xsa + (j & ~1)) + (j & 1);
  f[0] = x;
  f[2] = y;
  f[4] = z;
  f[6] = 0.0f;
}

__device__ __forceinline__ float4 xsa_load(const float4* __restrict__ xsa, int j) {
  const float* f = reinterpret_cast<const float*>(xsa + (j & ~1)) + (j & 1);
  return make_float4(__ldg(f), __ldg(f + 2), __ldg(f + 4), 0.0f);
}

// The pair block of even slot j as three 64-bit pairs {x_j, x_j+1}, {y..},
// {z..}: one 256-bit read-only load (sm_100).
__device__ __forceinline__ void ld_pair(const float4* __restrict__ xsa, int j, uint64_t& xx,
                                        uint64_t& yy, uint64_t& zz) {
  asm("{\n\t.reg .b64 pad;\n\t"
      "ld.global.nc.v4.u64 {%0,%1,%2,pad}, [%3];\n\t}"
      : "=l"(xx), "=l"(yy), "=l"(zz)
      : "l"(xsa + j));
}

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
  xsa_store(xsa, j, (float)xs, (float)ys, (float)zs);
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

// cstart[lo..hi] = v, inline for a short run of cells, else as worklist
// pieces for k_fill_gaps.
__device__ __forceinline__ void set_cells(int64_t lo, int64_t hi, uint32_t v,
                                          uint32_t* __restrict__ cstart, uint4* gaps,
                                          uint32_t* gap_count) {
  if (hi - lo + 1 <= kSmallGap) {
    for (int64_t c = lo; c <= hi; ++c) cstart[c] = v;
  } else {
    push_gap(lo, hi, v, gaps, gap_count);
  }
}

// start[c] = lower_bound(keys, c): the first slot j of every non-empty key
// writes j into the cells (key[j-1], key[j]]; long runs of empty cells go to
// a worklist filled by k_fill_gaps.  A thread takes four consecutive slots
// (one 128-bit load of keys and the key before them).
constexpr int kStartsPerThread = 4;
__global__ void __launch_bounds__(kBlock)
    k_cell_starts(const uint32_t* __restrict__ keys, int n, uint32_t ncells,
                  uint32_t* __restrict__ cstart, uint4* __restrict__ gaps,
                  uint32_t* __restrict__ gap_count, uint32_t* __restrict__ err) {
  const int j0 = (blockIdx.x * blockDim.x + threadIdx.x) * kStartsPerThread;
  if (j0 >= n) return;
  uint32_t k[kStartsPerThread];
  if (j0 + kStartsPerThread <= n) {
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(keys + j0));
    k[0] = v.x;
    k[1] = v.y;
    k[2] = v.z;
    k[3] = v.w;
  } else {
#pragma unroll
    for (int u = 0; u < kStartsPerThread; ++u) k[u] = j0 + u < n ? __ldg(keys + j0 + u) : 0u;
  }
  int64_t kp = j0 > 0 ? (int64_t)__ldg(keys + j0 - 1) : -1;
#pragma unroll
  for (int u = 0; u < kStartsPerThread; ++u) {
    const int j = j0 + u;
    if (j >= n) break;
    const int64_t kk = (int64_t)k[u];
    if (kk >= (int64_t)ncells) {
      atomicOr(err, kErrCellRange);
      return;
    }
    if (kk != kp) set_cells(kp + 1, kk, (uint32_t)j, cstart, gaps, gap_count);
    kp = kk;
    // after the last key: every cell up to the sentinel cstart[C] starts at n
    if (j == n - 1) set_cells(kk + 1, (int64_t)ncells, (uint32_t)n, cstart, gaps, gap_count);
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
  const float4 q = xsa_load(xsa, j);
  const float fx = c.xf.x - q.x, fy = c.xf.y - q.y, fz = c.xf.z - q.z;
  const float r2f = norm2(fx, fy, fz);
  if (r2f < c.h2lo) return true;
  if (r2f > c.h2hi) return false;
  return exact_neighbor(c, pd, j);
}

// Address of list entry t of particle p in the four-entry blocks nbr4[15][n].
__device__ __forceinline__ size_t nbr_index(int n, int p, int t) {
  return (((size_t)(t >> 2) * n + p) << 2) + (t & 3);
}

// FillNeighbors' 27-cell walk (neighbors.c:247-295) verbatim, for a
// particle whose neighbour cells are not cx-1..cx+1 (FP64 rounding at a cell
// face): its bucket goes to list entries 0..count-1 of p in nbr, the last
// block's entries past the count are set to p; returns the count.
__device__ __forceinline__ int walk_27_cells(const DevParams& P, const NbrView& V, const BuildCtx& c,
                                          const PD* __restrict__ pd,
                                          const float4* __restrict__ xsa, int p,
                                          uint32_t* __restrict__ nbr) {
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
          if (j != p && is_neighbor(c, pd, xsa, j)) nbr[nbr_index(V.n, p, count++)] = (uint32_t)j;
        }
      }
  for (int t = count; t & 3; ++t) nbr[nbr_index(V.n, p, t)] = (uint32_t)p;
  return count;
}

// ---------------------------------------------------------------------------
// Staged neighbour build (FillNeighbors, neighbors.c:217-298): one thread per
// particle walks its 9 (dz, dy) slot rows in the reference's order (rows of
// cells cx-1..cx+1 are contiguous slot ranges, cells in dx order, particles
// in ascending original index), appending every candidate without branches
// to its own column of a shared-memory staging area -- store the entry,
// advance the count on a hit; the particle itself is skipped by splitting
// its own row -- and writes its bucket out at the end as four-entry blocks
// of nbr4[15][n] (for each block index, a warp's 32 consecutive slots are
// four whole 128-byte lines), the last block's entries past the count set to
// p.  A staged entry is 2 bytes, (row << 12) | offset in the
// row, with the row starts kept in shared memory, so a thread holds 156
// bytes of shared memory and the candidate loop only the particle's FP32
// position: enough blocks stay resident to hide the candidate loads.  The
// candidates of a row are tested two at a time with the packed FP32x2
// arithmetic of sm_100 (staged_range).  A particle with a row of more than
// 4095 candidates takes the verbatim 27-cell walk.
// ---------------------------------------------------------------------------
constexpr int kStagedBlock = 128;
constexpr int kRowBits = 12;
constexpr int kRowMax = (1 << kRowBits) - 1;

// Exact FP64 test of neighbors.c:278-285 for particle p and candidate j
// (rare: only pairs whose FP32 r^2 lies in the band); reloads both records.
__device__ __forceinline__ bool staged_exact(const DevParams& P, const PD* __restrict__ pd, int p,
                                          int j) {
  float4 xp, dpp, xq, dq;
  ld_pd(pd, p, xp, dpp);
  ld_pd(pd, j, xq, dq);
  const double ddx = __dsub_rn(xstar_d(xp.x, dpp.x), xstar_d(xq.x, dq.x));
  const double ddy = __dsub_rn(xstar_d(xp.y, dpp.y), xstar_d(xq.y, dq.y));
  const double ddz = __dsub_rn(xstar_d(xp.z, dpp.z), xstar_d(xq.z, dq.z));
  const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)),
                              __dmul_rn(ddz, ddz));
  return r2 < P.h2d;
}

// Test and append of one candidate slot j with FP32 r^2 = r2 (the exact
// FP64 test decides inside the band): the entry is stored at the thread's
// next staging slot and the count advances on a hit.
__device__ __forceinline__ void staged_one(const DevParams& P, const PD* __restrict__ pd, int p,
                                           int j, float r2, uint32_t entry,
                                           uint16_t* __restrict__ stg, int& cnt) {
  bool hit = r2 <= P.bld_h2hi;
  if (hit && r2 >= P.bld_h2lo) hit = staged_exact(P, pd, p, j);
  stg[cnt * kStagedBlock] = (uint16_t)entry;
  cnt += hit ? 1 : 0;
}

// Test and append of the four candidates j .. j+3 with FP32 r^2 = r2[u]:
// one branch for the group, taken only when a candidate lies in the band
// (the exact FP64 test then decides those), then four branch-free appends.
__device__ __forceinline__ void staged_four(const DevParams& P, const PD* __restrict__ pd, int p,
                                            int j, const float (&r2)[4], uint32_t entry,
                                            uint16_t* __restrict__ stg, int& cnt) {
  bool hit[4];
  bool band = false;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    hit[u] = r2[u] <= P.bld_h2hi;
    band |= hit[u] && r2[u] >= P.bld_h2lo;
  }
  if (band) {
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (hit[u] && r2[u] >= P.bld_h2lo) hit[u] = staged_exact(P, pd, p, j + u);
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    stg[cnt * kStagedBlock] = (uint16_t)(entry + u);
    cnt += hit[u] ? 1 : 0;
  }
}

// r^2 of one slot from the FP32 positions (the ragged ends of a range).
__device__ __forceinline__ float staged_r2(const float4* __restrict__ xsa, int j, float px,
                                           float py, float pz) {
  const float4 q = xsa_load(xsa, j);
  const float fx = px - q.x, fy = py - q.y, fz = pz - q.z;
  return norm2(fx, fy, fz);
}

// Appends the candidates of slots [ja, jb) of row r (starting at slot rb),
// entries (r << kRowBits) | (j - rb).  The slots of an even-aligned pair are
// tested together with packed FP32x2 arithmetic (each lane rounds as the
// scalar form would: x_p - x_q, then (dx^2 + dy^2) + dz^2 by fused
// multiply-adds), two pairs per batch while four more entries fit below the
// cap; an odd first or last slot is tested alone.
__device__ __forceinline__ void staged_range(const DevParams& P, const PD* __restrict__ pd,
                                             const float4* __restrict__ xsa, uint64_t pxx,
                                             uint64_t pyy, uint64_t pzz, float px, float py,
                                             float pz, int p, int r, int rb, int ja, int jb,
                                             uint16_t* __restrict__ stg, int& cnt) {
  const uint32_t tag = (uint32_t)r << kRowBits;
  int j = ja;
  if ((j & 1) && j < jb && cnt < kMaxNeighbors) {
    staged_one(P, pd, p, j, staged_r2(xsa, j, px, py, pz), tag | (uint32_t)(j - rb), stg, cnt);
    ++j;
  }
  for (; j + 4 <= jb && cnt <= kMaxNeighbors - 4; j += 4) {
    // pair blocks of slots j, j+1 and j+2, j+3
    uint64_t x0, y0, z0, x1, y1, z1;
    ld_pair(xsa, j, x0, y0, z0);
    ld_pair(xsa, j + 2, x1, y1, z1);
    uint64_t d = f2_sub(pxx, x0);
    uint64_t s0 = f2_mul(d, d);
    d = f2_sub(pyy, y0);
    s0 = f2_fma(d, d, s0);
    d = f2_sub(pzz, z0);
    s0 = f2_fma(d, d, s0);
    d = f2_sub(pxx, x1);
    uint64_t s1 = f2_mul(d, d);
    d = f2_sub(pyy, y1);
    s1 = f2_fma(d, d, s1);
    d = f2_sub(pzz, z1);
    s1 = f2_fma(d, d, s1);
    const float r2[4] = {f2_lo(s0), f2_hi(s0), f2_lo(s1), f2_hi(s1)};
    staged_four(P, pd, p, j, r2, tag | (uint32_t)(j - rb), stg, cnt);
  }
  for (; j + 2 <= jb && cnt <= kMaxNeighbors - 2; j += 2) {
    uint64_t x0, y0, z0;
    ld_pair(xsa, j, x0, y0, z0);
    uint64_t d = f2_sub(pxx, x0);
    uint64_t s0 = f2_mul(d, d);
    d = f2_sub(pyy, y0);
    s0 = f2_fma(d, d, s0);
    d = f2_sub(pzz, z0);
    s0 = f2_fma(d, d, s0);
    const uint32_t e = tag | (uint32_t)(j - rb);
    staged_one(P, pd, p, j, f2_lo(s0), e, stg, cnt);
    staged_one(P, pd, p, j + 1, f2_hi(s0), e + 1, stg, cnt);
  }
  for (; j < jb && cnt < kMaxNeighbors; ++j)
    staged_one(P, pd, p, j, staged_r2(xsa, j, px, py, pz), tag | (uint32_t)(j - rb), stg, cnt);
}

// 9 blocks of 128 threads per SM: 56 registers (8 bytes spilled since the
// four-entry write-out, no slower at 16.7M particles than without; a tighter
// cap spills more and gains nothing).
__global__ void __launch_bounds__(kStagedBlock, 9)
    k_build_staged(const DevParams P, const NbrView V, const PD* __restrict__ pd,
                   const float4* __restrict__ xsa, const uint32_t* __restrict__ cellp,
                   uint32_t* __restrict__ nbr, uint8_t* __restrict__ ncount) {
  __shared__ uint16_t s_stage[kMaxNeighbors * kStagedBlock];
  __shared__ int s_rowb[9 * kStagedBlock];
  const int p = blockIdx.x * kStagedBlock + threadIdx.x;
  if (p >= P.n) return;
  uint16_t* stg = s_stage + threadIdx.x;
  int* rowb = s_rowb + threadIdx.x;
  BuildCtx c;
  ld_pd(pd, p, c.xp, c.dp);
  c.xs = xstar_d(c.xp.x, c.dp.x);
  c.ys = xstar_d(c.xp.y, c.dp.y);
  c.zs = xstar_d(c.xp.z, c.dp.z);
  int cx, cy, cz;
  unpack_cell(V, __ldg(cellp + p), cx, cy, cz);
  bool regular = axis_regular(c.xs, P.hd, cx, P.nx) && axis_regular(c.ys, P.hd, cy, P.ny) &&
                 axis_regular(c.zs, P.hd, cz, P.nz);
  // the 9 rows' slot ranges (empty outside the grid)
  const int xlo = cx - (cx > 0);
  const int xhi = cx + (cx < P.nx - 1);
  if (regular) {
    for (int r = 0; r < 9; ++r) {
      const int z = cz + r / 3 - 1, y = cy + r % 3 - 1;
      int b = 0, e = 0;
      if ((unsigned)z < (unsigned)P.nz && (unsigned)y < (unsigned)P.ny) {
        const uint32_t rk = (uint32_t)z * P.nxny + (uint32_t)y * (uint32_t)P.nx;
        b = (int)__ldg(V.cstart + rk + xlo);
        e = (int)__ldg(V.cstart + rk + xhi + 1);
      }
      if (e - b > kRowMax) regular = false;  // the row offset would not fit
      rowb[r * kStagedBlock] = b;
    }
  }
  int count = 0;
  if (regular) {
    const float4 xf = xsa_load(xsa, p);
    const uint64_t pxx = f2_dup(xf.x), pyy = f2_dup(xf.y), pzz = f2_dup(xf.z);
    for (int r = 0; r < 9 && count < kMaxNeighbors; ++r) {
      const int z = cz + r / 3 - 1, y = cy + r % 3 - 1;
      if ((unsigned)z >= (unsigned)P.nz || (unsigned)y >= (unsigned)P.ny) continue;
      const uint32_t rk = (uint32_t)z * P.nxny + (uint32_t)y * (uint32_t)P.nx;
      const int b = rowb[r * kStagedBlock];
      const int e = (int)__ldg(V.cstart + rk + xhi + 1);
      if (r == 4) {
        staged_range(P, pd, xsa, pxx, pyy, pzz, xf.x, xf.y, xf.z, p, r, b, b, p, stg, count);
        staged_range(P, pd, xsa, pxx, pyy, pzz, xf.x, xf.y, xf.z, p, r, b, p + 1, e, stg, count);
      } else {
        staged_range(P, pd, xsa, pxx, pyy, pzz, xf.x, xf.y, xf.z, p, r, b, b, e, stg, count);
      }
    }
    // one 16-byte block of four entries per store; the last block's entries
    // past the count are p
    uint4* out = reinterpret_cast<uint4*>(nbr) + p;
    auto entry = [&](int t) {
      const uint32_t en = stg[t * kStagedBlock];
      return t < count ? (uint32_t)(rowb[(en >> kRowBits) * kStagedBlock] + (int)(en & kRowMax))
                       : (uint32_t)p;
    };
#pragma unroll 1
    for (int t0 = 0; t0 < count; t0 += 4, out += P.n)
      *out = make_uint4(entry(t0), entry(t0 + 1), entry(t0 + 2), entry(t0 + 3));
  } else {
    c.xf = xsa_load(xsa, p);
    c.h2lo = P.bld_h2lo;
    c.h2hi = P.bld_h2hi;
    c.h2d = P.h2d;
    count = walk_27_cells(P, V, c, pd, xsa, p, nbr);
  }
  ncount[p] = (uint8_t)count;
}

__global__ void __launch_bounds__(kBlock)
    k_export_buckets(const NbrView V, const uint32_t* __restrict__ ids,
                     uint32_t* __restrict__ nbr, int32_t* __restrict__ count,
                     uint32_t* __restrict__ err) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= V.n) return;
  // the list's last block must hold p past the count (the batched visits
  // read those entries as the pair (p, p))
  const int c0 = (int)__ldg(V.ncount + p);
  for (int t = c0; t & 3; ++t)
    if (nbr_entry(V, p, t) != (uint32_t)p) atomicOr(err, kErrNbrTail);
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
  const int threads = (n + kStartsPerThread - 1) / kStartsPerThread;
  k_cell_starts<<<grid_for(threads), kBlock, 0, st>>>(keys_sorted, n, ncells, cstart, gaps,
                                                       gap_count, err);
  k_fill_gaps<<<148 * 16, kBlock, 0, st>>>(gaps, gap_count, cstart);
}

void launch_build_neighbors(const DevParams& P, const NbrView& V, const PD* pd,
                            const float4* xsa, const uint32_t* cellp, uint32_t* nbr,
                            uint8_t* ncount, cudaStream_t st) {
  k_build_staged<<<grid_for(P.n, kStagedBlock), kStagedBlock, 0, st>>>(P, V, pd, xsa, cellp, nbr,
                                                                        ncount);
}

void launch_export_buckets(const NbrView& V, const uint32_t* ids, uint32_t* nbr, int32_t* count,
                           uint32_t* err, cudaStream_t st) {
  k_export_buckets<<<grid_for(V.n), kBlock, 0, st>>>(V, ids, nbr, count, err);
}

}  // namespace sphpc
