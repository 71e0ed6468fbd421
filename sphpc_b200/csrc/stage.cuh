// stage.cuh -- shared-memory staging of a CTA's neighbourhood records.
//
// A CTA owns kStageThreads consecutive slots.  Slots are sorted by cell key
// (z, then y, then x), so its particles lie in one to three (cy, cz) rows of
// cells, and every neighbour of a regular particle lies in the rows (cy+dy,
// cz+dz), dy, dz in {-1, 0, 1}, within one cell of the CTA's x extent.  Those
// rows are contiguous slot ranges; the CTA merges them, copies their records
// into shared memory with coalesced 256-bit loads, and each thread then reads
// its neighbours' records from shared memory instead of scattering 32-byte
// requests through L1.  A neighbour outside the staged ranges (a particle
// whose neighbour cells FP64 rounding moved, or a CTA whose rows do not fit)
// is read from global memory.
#pragma once
#include "sphpc_dev.cuh"

namespace sphpc {

constexpr int kStageThreads = 128;
constexpr int kStageRecords = 1536;     // 48 KB of 32-byte records
constexpr int kStageMaxRanges = 27;     // 3 source rows x 9 neighbour rows

struct StageShared {
  int nranges;                          // 0: staging disabled for this CTA
  int rs[kStageMaxRanges];              // range start slot
  int re[kStageMaxRanges];              // range end slot (exclusive)
  int ro[kStageMaxRanges];              // offset of the range in recs[]
};

// Thread 0: the merged slot ranges of the CTA's neighbour rows.
__device__ __forceinline__ void stage_plan(const NbrView& V, const uint32_t* __restrict__ cellp,
                                           int p0, int p1, StageShared& S) {
  int cx0, cy0, cz0, cx1, cy1, cz1;
  unpack_cell(V, __ldg(cellp + p0), cx0, cy0, cz0);
  unpack_cell(V, __ldg(cellp + p1), cx1, cy1, cz1);
  const int row0 = cz0 * V.ny + cy0, row1 = cz1 * V.ny + cy1;
  S.nranges = 0;
  if (row1 - row0 > 2) return;
  int rs[kStageMaxRanges], re[kStageMaxRanges], m = 0;
  for (int row = row0; row <= row1; ++row) {
    const int cy = row % V.ny, cz = row / V.ny;
    const int xa = row == row0 ? cx0 : 0;
    const int xb = row == row1 ? cx1 : V.nx - 1;
    const int xlo = max(xa - 1, 0), xhi = min(xb + 1, V.nx - 1);
    for (int dz = -1; dz <= 1; ++dz) {
      const int z = cz + dz;
      if ((unsigned)z >= (unsigned)V.nz) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int y = cy + dy;
        if ((unsigned)y >= (unsigned)V.ny) continue;
        const uint32_t rk = (uint32_t)z * V.nxny + (uint32_t)y * (uint32_t)V.nx;
        const int b = (int)__ldg(V.cstart + rk + xlo);
        const int e = (int)__ldg(V.cstart + rk + xhi + 1);
        if (e <= b) continue;
        // insertion by start
        int k = m++;
        while (k > 0 && rs[k - 1] > b) {
          rs[k] = rs[k - 1];
          re[k] = re[k - 1];
          --k;
        }
        rs[k] = b;
        re[k] = e;
      }
    }
  }
  // merge overlapping / touching ranges
  int nr = 0, total = 0;
  for (int k = 0; k < m; ++k) {
    if (nr > 0 && rs[k] <= S.re[nr - 1]) {
      if (re[k] > S.re[nr - 1]) S.re[nr - 1] = re[k];
    } else {
      S.rs[nr] = rs[k];
      S.re[nr] = re[k];
      ++nr;
    }
  }
  for (int k = 0; k < nr; ++k) {
    S.ro[k] = total;
    total += S.re[k] - S.rs[k];
  }
  S.nranges = total <= kStageRecords ? nr : 0;
}

// Whole CTA: plan and copy.  Every thread of the CTA must call it.
__device__ __forceinline__ void stage_load(const NbrView& V, const uint32_t* __restrict__ cellp,
                                           const PD* __restrict__ pd, StageShared& S,
                                           PD* recs) {
  const int p0 = blockIdx.x * kStageThreads;
  const int p1 = min(p0 + kStageThreads, V.n) - 1;
  if (threadIdx.x == 0) stage_plan(V, cellp, p0, p1, S);
  __syncthreads();
  const int nr = S.nranges;
  for (int k = 0; k < nr; ++k) {
    const int b = S.rs[k], len = S.re[k] - b, o = S.ro[k];
    for (int i = threadIdx.x; i < len; i += kStageThreads) {
      float4 x, d;
      ld_pd(pd, b + i, x, d);
      recs[o + i].x = x;
      recs[o + i].d = d;
    }
  }
  __syncthreads();
}

// Per thread: a cursor over the staged ranges.  Buckets are in ascending
// slot order (rows in key order, slots ascending within a row), so the
// cursor normally only moves forward; it also moves back for the rare bucket
// that revisits a cell.
struct StageCursor {
  int r = 0;
  __device__ __forceinline__ void get(const StageShared& S, const PD* recs,
                                      const PD* __restrict__ pd, int q, float4& x, float4& d) {
    const int nr = S.nranges;
    while (r > 0 && q < S.re[r - 1]) --r;   // back while q lies before the previous end
    while (r < nr && q >= S.re[r]) ++r;     // forward past ranges that end at or before q
    if (r < nr && q >= S.rs[r]) {
      const PD& rec = recs[S.ro[r] + q - S.rs[r]];
      x = rec.x;
      d = rec.d;
    } else {
      ld_pd(pd, q, x, d);
    }
  }
};

}  // namespace sphpc
