// radix_sort.cuh -- stable LSD radix sort of u32 keys with u32 values.
//
// Replaces thrust::sort_by_key (thrust_c.cu:86-91).  One "onesweep" kernel
// per 8-bit digit: every tile of 4096 pairs ranks its keys stably inside the
// tile (warp match + per-warp digit counters, in input order), publishes its
// per-digit counts, resolves the per-digit prefix of all earlier tiles with a
// decoupled look-back, stages the tile in shared memory in digit order and
// writes each digit run contiguously.  HBM traffic per digit pass is one read
// and one write of the pairs (16 B per pair); the digit histograms of all
// passes come from one extra read of the keys (or from the hash kernel that
// produced them).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sphpc {

constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 pairs
constexpr int kMaxPasses = 4;

constexpr uint32_t kLbAgg = 1u << 30;   // look-back: tile aggregate available
constexpr uint32_t kLbInc = 2u << 30;   // look-back: inclusive prefix available
constexpr uint32_t kLbValue = (1u << 30) - 1u;
constexpr int kSpinLimit = 1 << 22;     // bounded waits: ~0.1-1 s, then error
constexpr int kLookBack = 4;            // look-back flags read per poll

// Scratch needed by one sort of n pairs with `passes` digit passes.
struct SortScratch {
  uint32_t* keys_alt;     // n
  uint32_t* vals_alt;     // n
  uint32_t* hist;         // kMaxPasses * kRadix  (counts, then exclusive offsets)
  uint32_t* lookback;     // kMaxPasses * tiles * kRadix
  uint32_t* counters;     // kMaxPasses tile counters
  uint32_t* err;          // error bits
};

inline int sort_tiles(int n) { return (n + kSortTile - 1) / kSortTile; }

// Bytes of scratch excluding the two alternate buffers.
inline size_t sort_aux_words(int n) {
  return (size_t)kMaxPasses * kRadix + (size_t)kMaxPasses * sort_tiles(n) * kRadix +
         kMaxPasses;
}

// Host: enqueue the whole sort on `stream`.  Sorts (keys, vals) by the low
// 8*passes bits of the keys.  With vals_iota the input values are taken to be
// 0..n-1 and vals is only an output buffer.  If hist_ready is true,
// scratch.hist already holds the digit counts of all passes (from a fused
// producer).  An odd pass count leaves the result in the scratch alternates:
// copy_back copies it into keys/vals, otherwise keys_res/vals_res say where
// it is.
cudaError_t radix_sort_pairs(uint32_t* keys, uint32_t* vals, int n, int passes,
                             const SortScratch& s, cudaStream_t stream, bool hist_ready,
                             bool vals_iota, bool copy_back, uint32_t** keys_res,
                             uint32_t** vals_res);

// Histogram of all `passes` digits, accumulated into hist (must be zeroed).
void launch_digit_histogram(const uint32_t* keys, int n, int passes, uint32_t* hist,
                            cudaStream_t stream);

// Device helper for fused producers: count the digits of one key into
// shared-memory histograms s_hist[passes][kRadix].
__device__ __forceinline__ void count_key_digits(uint32_t* s_hist, uint32_t key, int passes) {
  for (int p = 0; p < passes; ++p)
    atomicAdd(&s_hist[p * kRadix + ((key >> (p * kRadixBits)) & (kRadix - 1))], 1u);
}

// Failure-detection check of the look-back wait: one onesweep CTA waits on a
// flag that no CTA ever writes, with a poll limit of spin_limit; returns the
// error bits it raised (kErrSortSpin when the bounded wait gave up).
cudaError_t lookback_wait_probe(int spin_limit, uint32_t* err_bits);

// lower_bound / upper_bound of every c in [0, count) over sorted keys
// (FindLowerBounds / FindUpperBounds, thrust_c.cu:93-120).
cudaError_t launch_bounds(const uint32_t* keys, int n, int count, uint32_t* out, bool upper,
                          cudaStream_t stream);

}  // namespace sphpc
