// radix_sort.cu -- onesweep LSD radix sort and the cell-bounds seam kernels.
#include "radix_sort.cuh"

#include <vector>

namespace sphpc {

namespace {

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.volatile.global.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

__device__ __forceinline__ void st_volatile(uint32_t* p, uint32_t v) {
  asm volatile("st.volatile.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__global__ void __launch_bounds__(256) k_digit_histogram(const uint32_t* __restrict__ keys,
                                                         int n, int passes,
                                                         uint32_t* __restrict__ hist) {
  __shared__ uint32_t s_hist[kMaxPasses * kRadix];
  for (int i = threadIdx.x; i < kMaxPasses * kRadix; i += blockDim.x) s_hist[i] = 0;
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    count_key_digits(s_hist, __ldg(keys + i), passes);
  __syncthreads();
  for (int i = threadIdx.x; i < passes * kRadix; i += blockDim.x)
    if (s_hist[i]) atomicAdd(hist + i, s_hist[i]);
}

// Exclusive scan of each pass's 256 digit counts (one block, 256 threads).
__global__ void __launch_bounds__(256) k_scan_digits(uint32_t* __restrict__ hist, int passes) {
  __shared__ uint32_t s_warp[kRadix / 32];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (int p = 0; p < passes; ++p) {
    const uint32_t v = hist[p * kRadix + t];
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    uint32_t wsum = 0;
    for (int w = 0; w < warp; ++w) wsum += s_warp[w];
    hist[p * kRadix + t] = wsum + x - v;
    __syncthreads();
  }
}

// One digit pass.  vals_in == nullptr means the values are the input
// indices (iota), which is how SortHash calls SortByKey (neighbors.c:123).
// Five blocks per SM (48 registers, no spills; 43 KB of shared memory
// each) rather than the two that the compiler's own choice of 128
// registers leaves room for: the passes wait on loads and on the
// look-back, so resident warps are what hides it.  The values are loaded
// only when the tile is staged, which is what lets the ranking fit.
__global__ void __launch_bounds__(kSortThreads, 5)
    k_onesweep(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
               uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, int n,
               int shift, const uint32_t* __restrict__ digit_offset,
               uint32_t* __restrict__ lookback, uint32_t* __restrict__ tile_counter,
               uint32_t* __restrict__ err, int spin_limit) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_whist[kSortWarps][kRadix + 1];
  __shared__ uint32_t s_dstart[kRadix];
  __shared__ uint32_t s_gbase[kRadix];
  __shared__ uint32_t s_wsum[kRadix / 32];
  __shared__ uint32_t s_keys[kSortTile];
  __shared__ uint32_t s_vals[kSortTile];

  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (t == 0) s_tile = atomicAdd(tile_counter, 1u);
  for (int i = t; i < kSortWarps * (kRadix + 1); i += kSortThreads)
    (&s_whist[0][0])[i] = 0;
  __syncthreads();
  const uint32_t tile = s_tile;
  // n <= kLbValue < 2^30, so every index fits 32 bits
  const int tile_base = (int)tile * kSortTile;
  const int wbase = tile_base + warp * 32 * kSortItems;

  // the values are loaded only when the tile is staged, so that the ranking
  // holds two arrays of registers, not three
  uint32_t key[kSortItems], rank[kSortItems];
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) {
    const int idx = wbase + i * 32 + lane;
    key[i] = idx < n ? __ldg(keys_in + idx) : 0xffffffffu;
  }
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) {
    const int idx = wbase + i * 32 + lane;
    const uint32_t d = idx < n ? ((key[i] >> shift) & (kRadix - 1)) : (uint32_t)kRadix;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const int leader = __ffs(peers) - 1;
    uint32_t prev = 0;
    if (lane == leader) {
      prev = s_whist[warp][d];
      s_whist[warp][d] = prev + __popc(peers);
    }
    prev = __shfl_sync(0xffffffffu, prev, leader);
    rank[i] = prev + __popc(peers & lt);
    __syncwarp();
  }
  __syncthreads();

  // Per digit: exclusive prefix over warps, the tile count, look-back.
  {
    const int d = t;  // kSortThreads == kRadix
    uint32_t sum = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t c = s_whist[w][d];
      s_whist[w][d] = sum;
      sum += c;
    }
    const uint32_t cnt = sum;
    uint32_t* my = lookback + (size_t)tile * kRadix + d;
    if (tile == 0) {
      st_volatile(my, kLbInc | cnt);
    } else {
      st_volatile(my, kLbAgg | cnt);
    }
    uint32_t excl = 0;
    if (tile > 0) {
      // kLookBack predecessors' flags per poll, consumed in order down to the
      // first inclusive one; a poll that finds the nearest one not yet
      // published waits and polls again from there
      int64_t pt = (int64_t)tile - 1;
      int spins = 0;
      for (;;) {
        uint32_t v[kLookBack];
#pragma unroll
        for (int k = 0; k < kLookBack; ++k)
          v[k] = pt - k >= 0 ? ld_volatile(lookback + (size_t)(pt - k) * kRadix + d) : 0u;
        int k = 0;
        bool done = false;
#pragma unroll
        for (; k < kLookBack; ++k) {
          if ((v[k] & (kLbAgg | kLbInc)) == 0) break;
          excl += v[k] & kLbValue;
          if (v[k] & kLbInc) {
            done = true;
            break;
          }
        }
        if (done) break;
        pt -= k;
        if (k == 0) {
          if (++spins > spin_limit) {
            atomicOr(err, 2u);  // kErrSortSpin
            break;
          }
          __nanosleep(32);
        }
      }
      st_volatile(my, kLbInc | (excl + cnt));
    }
    s_gbase[d] = __ldg(digit_offset + d) + excl;
    // tile-local exclusive scan of cnt over digits
    uint32_t x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_wsum[warp] = x;
    __syncthreads();
    uint32_t wsum = 0;
    for (int w = 0; w < warp; ++w) wsum += s_wsum[w];
    s_dstart[d] = wsum + x - cnt;
  }
  __syncthreads();

  // Stage the tile in digit order.
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) {
    const int idx = wbase + i * 32 + lane;
    if (idx < n) {
      const uint32_t d = (key[i] >> shift) & (kRadix - 1);
      const uint32_t lp = s_dstart[d] + s_whist[warp][d] + rank[i];
      s_keys[lp] = key[i];
      s_vals[lp] = vals_in ? __ldg(vals_in + idx) : (uint32_t)idx;
    }
  }
  __syncthreads();
  const int valid = min(kSortTile, n - tile_base);
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) {
    const int k = t + i * kSortThreads;
    if (k < valid) {
      const uint32_t kk = s_keys[k];
      const uint32_t d = (kk >> shift) & (kRadix - 1);
      const uint32_t g = s_gbase[d] + (uint32_t)k - s_dstart[d];
      if (g < (uint32_t)n) {
        keys_out[g] = kk;
        vals_out[g] = s_vals[k];
      } else {
        atomicOr(err, 4u);  // inconsistent digit counts: never write out of range
      }
    }
  }
}

__global__ void k_bounds(const uint32_t* __restrict__ keys, int n, int count,
                         uint32_t* __restrict__ out, int upper) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < count;
       c += gridDim.x * blockDim.x) {
    int lo = 0, hi = n;
    const uint32_t v = (uint32_t)c;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      const uint32_t k = __ldg(keys + mid);
      const bool go_right = upper ? (k <= v) : (k < v);
      if (go_right) lo = mid + 1; else hi = mid;
    }
    out[c] = (uint32_t)lo;
  }
}

}  // namespace

void launch_digit_histogram(const uint32_t* keys, int n, int passes, uint32_t* hist,
                            cudaStream_t stream) {
  if (n <= 0) return;
  int blocks = (n + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_digit_histogram<<<blocks, 256, 0, stream>>>(keys, n, passes, hist);
}

cudaError_t radix_sort_pairs(uint32_t* keys, uint32_t* vals, int n, int passes,
                             const SortScratch& s, cudaStream_t stream, bool hist_ready,
                             bool vals_iota, bool copy_back, uint32_t** keys_res,
                             uint32_t** vals_res) {
  if (passes < 1 || passes > kMaxPasses) return cudaErrorInvalidValue;
  if (n < 0 || (uint64_t)n > kLbValue || vals == nullptr) return cudaErrorInvalidValue;
  cudaError_t e;
  if (n <= 1) {
    if (n == 1 && vals_iota) {
      e = cudaMemsetAsync(vals, 0, sizeof(uint32_t), stream);
      if (e != cudaSuccess) return e;
    }
    if (keys_res) *keys_res = keys;
    if (vals_res) *vals_res = vals;
    return cudaSuccess;
  }
  const int tiles = sort_tiles(n);
  if (!hist_ready) {
    e = cudaMemsetAsync(s.hist, 0, sizeof(uint32_t) * kMaxPasses * kRadix, stream);
    if (e != cudaSuccess) return e;
    launch_digit_histogram(keys, n, passes, s.hist, stream);
  }
  e = cudaMemsetAsync(s.lookback, 0, sizeof(uint32_t) * (size_t)passes * tiles * kRadix,
                      stream);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(s.counters, 0, sizeof(uint32_t) * kMaxPasses, stream);
  if (e != cudaSuccess) return e;
  k_scan_digits<<<1, kRadix, 0, stream>>>(s.hist, passes);
  // Pass p reads the previous output and writes buffer set (p & 1):
  // set 0 = scratch alternates, set 1 = the caller's arrays.
  uint32_t* const bk[2] = {s.keys_alt, keys};
  uint32_t* const bv[2] = {s.vals_alt, vals};
  const uint32_t* kin = keys;
  const uint32_t* vin = vals_iota ? nullptr : vals;
  for (int p = 0; p < passes; ++p) {
    uint32_t* kout = bk[p & 1];
    uint32_t* vout = bv[p & 1];
    k_onesweep<<<tiles, kSortThreads, 0, stream>>>(
        kin, vin, kout, vout, n, p * kRadixBits, s.hist + p * kRadix,
        s.lookback + (size_t)p * tiles * kRadix, s.counters + p, s.err, kSpinLimit);
    kin = kout;
    vin = vout;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  uint32_t* kres = const_cast<uint32_t*>(kin);
  uint32_t* vres = const_cast<uint32_t*>(vin);
  if (copy_back && kres != keys) {
    e = cudaMemcpyAsync(keys, kres, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, stream);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(vals, vres, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, stream);
    if (e != cudaSuccess) return e;
    kres = keys;
    vres = vals;
  }
  if (keys_res) *keys_res = kres;
  if (vals_res) *vals_res = vres;
  return cudaSuccess;
}

cudaError_t lookback_wait_probe(int spin_limit, uint32_t* err_bits) {
  // Two tiles of keys; the tile counter starts at 1, so the one CTA
  // launched ranks tile 1 and looks back at tile 0, whose flag no CTA ever
  // writes.  Its wait gives up after spin_limit polls and sets kErrSortSpin;
  // the digit offsets are those of all 2 tiles, so every scatter the CTA
  // then makes stays below n.
  const int n = 2 * kSortTile;
  std::vector<uint32_t> hk(n);
  uint32_t hist[kRadix] = {};
  for (int i = 0; i < n; ++i) {
    hk[i] = (uint32_t)i * 2654435761u;
    ++hist[hk[i] & (kRadix - 1)];
  }
  uint32_t offs[kRadix];
  uint32_t acc = 0;
  for (int d = 0; d < kRadix; ++d) {
    offs[d] = acc;
    acc += hist[d];
  }
  uint32_t* buf = nullptr;
  const size_t words = 4 * (size_t)n + kRadix + 2 * kRadix + 2;
  cudaError_t e = cudaMalloc(&buf, words * sizeof(uint32_t));
  if (e != cudaSuccess) return e;
  uint32_t* keys = buf;
  uint32_t* vals = buf + n;
  uint32_t* kout = buf + 2 * (size_t)n;
  uint32_t* vout = buf + 3 * (size_t)n;
  uint32_t* doff = buf + 4 * (size_t)n;
  uint32_t* lookback = doff + kRadix;
  uint32_t* counter = lookback + 2 * kRadix;
  uint32_t* err = counter + 1;
  const uint32_t one = 1u;
  e = cudaMemset(buf, 0, words * sizeof(uint32_t));
  if (e == cudaSuccess)
    e = cudaMemcpy(keys, hk.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(doff, offs, sizeof(offs), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(counter, &one, sizeof(one), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_onesweep<<<1, kSortThreads>>>(keys, vals, kout, vout, n, 0, doff, lookback, counter, err,
                                    spin_limit);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(err_bits, err, sizeof(uint32_t), cudaMemcpyDeviceToHost);
  cudaFree(buf);
  return e;
}

cudaError_t launch_bounds(const uint32_t* keys, int n, int count, uint32_t* out, bool upper,
                          cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  int blocks = (count + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_bounds<<<blocks, 256, 0, stream>>>(keys, n, count, out, upper ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace sphpc
