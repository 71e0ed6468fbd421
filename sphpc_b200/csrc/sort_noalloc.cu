// sort_noalloc.cu -- SortByKeyNoAlloc: the stable key/value sort of SortByKey
// for callers that must not allocate device memory.
//
// SortByKey grows a cached scratch buffer with cudaMalloc the first time it
// sees a larger count.  Some callers cannot let a library do that: hosts that
// own every byte of device memory through their own pool and forbid
// allocations behind their back, and time-critical loops in which a
// cudaMalloc (which can synchronise the device or fail under memory
// pressure) is not acceptable.  This entry point instead keeps its scratch in
// the fixed array below, so it calls no cudaMalloc, cudaFree or allocating
// library routine; the price is a maximum count and one shared scratch area
// per GPU.
#include <cstring>
#include <mutex>

#include "host_internal.h"
#include "radix_sort.cuh"

namespace sphpc {

// Largest count SortByKeyNoAlloc accepts: 262,144 key/value pairs.
constexpr int kNoAllocMaxPairs = 1 << 18;

// Words of scratch: two alternate buffers of kNoAllocMaxPairs plus the
// digit histograms, look-back flags, tile counters and error word of
// radix_sort_pairs (about 2.4 MB).  Every GPU that loads the library holds
// this array until the process exits.
constexpr size_t kNoAllocWords =
    2 * (size_t)kNoAllocMaxPairs + ((size_t)kMaxPasses * kRadix +
                                    (size_t)kMaxPasses * ((kNoAllocMaxPairs + kSortTile - 1) /
                                                          kSortTile) * kRadix +
                                    kMaxPasses) + 8;

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;

// The looked-up address of each device, with the unique id of the context it
// belongs to: a cudaDeviceReset ends the device's primary context, the next
// runtime call makes a new one and loads the module again, and the array may
// then sit at another address.
struct ScratchSlot {
  uint32_t* ptr = nullptr;
  unsigned long long ctx_id = 0;
  bool ctx_known = false;
};
ScratchSlot g_scratch[kMaxDevices];

// cuCtxGetCurrent / cuCtxGetId from the driver, fetched through the runtime
// (the library links only the static runtime).
using CtxGetCurrentFn = int (*)(void**);
using CtxGetIdFn = int (*)(void*, unsigned long long*);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;
bool g_ctx_fns_tried = false;

// Unique id of the current context; false when the driver cannot say (then
// the address is looked up again on every call).
bool current_ctx_id(unsigned long long* id) {
  if (!g_ctx_fns_tried) {
    g_ctx_fns_tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
  }
  if (!g_ctx_get_current || !g_ctx_get_id) return false;
  void* ctx = nullptr;
  if (g_ctx_get_current(&ctx) != 0 || !ctx) return false;
  return g_ctx_get_id(ctx, id) == 0;
}

// Device address of g_noalloc_scratch on the current device.  In host code
// the array's name is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress, with the device current: once per device, and again
// whenever the device's context has changed since (after a cudaDeviceReset).
int scratch_address(uint32_t** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error(SPHPC_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return set_error(SPHPC_EINVAL, "SortByKeyNoAlloc: device %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_setup_mu);
  ScratchSlot& slot = g_scratch[dev];
  // no current context yet (before the first runtime call on this thread,
  // or right after a reset) counts as unknown: cudaGetSymbolAddress below
  // makes the primary context current, and the next call records its id
  unsigned long long id = 0;
  const bool known = current_ctx_id(&id);
  if (!slot.ptr || !known || !slot.ctx_known || slot.ctx_id != id) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return set_error(SPHPC_ECUDA, "cudaGetSymbolAddress(g_noalloc_scratch): %s",
                       cudaGetErrorString(e));
    slot.ptr = static_cast<uint32_t*>(p);
    slot.ctx_id = id;
    slot.ctx_known = known;
  }
  *out = slot.ptr;
  return SPHPC_OK;
}

}  // namespace
}  // namespace sphpc

using namespace sphpc;

extern "C" int SortByKeyNoAlloc(unsigned int* const keys, unsigned int* const values,
                                const int count, const void* const cuda_stream) {
  if (count < 0 || (count > 0 && (!keys || !values)))
    return set_error(SPHPC_EINVAL, "SortByKeyNoAlloc: bad arguments");
  if (count > kNoAllocMaxPairs)
    return set_error(SPHPC_EINVAL,
                     "SortByKeyNoAlloc: count %d exceeds the fixed scratch limit of %d pairs "
                     "(use SortByKey, which allocates its scratch)",
                     count, kNoAllocMaxPairs);
  if (count <= 1) return SPHPC_OK;
  uint32_t* base = nullptr;
  const int rc = scratch_address(&base);
  if (rc) return rc;
  SortScratch s;
  s.keys_alt = base;
  s.vals_alt = base + kNoAllocMaxPairs;
  uint32_t* aux = base + 2 * (size_t)kNoAllocMaxPairs;
  s.hist = aux;
  s.counters = aux + (size_t)kMaxPasses * kRadix;
  s.err = aux + (size_t)kMaxPasses * kRadix + kMaxPasses;
  s.lookback = aux + (size_t)kMaxPasses * kRadix + kMaxPasses + 4;
  cudaStream_t st = (cudaStream_t)cuda_stream;
  // The array keeps the previous call's contents: the error word must start
  // at zero (histograms, look-back flags and tile counters are cleared by
  // radix_sort_pairs itself).
  cudaError_t e = cudaMemsetAsync(s.err, 0, sizeof(uint32_t), st);
  if (e != cudaSuccess)
    return set_error(SPHPC_ECUDA, "SortByKeyNoAlloc: %s", cudaGetErrorString(e));
  e = radix_sort_pairs(keys, values, count, kMaxPasses, s, st, false, false, true, nullptr,
                       nullptr);
  if (e != cudaSuccess)
    return set_error(SPHPC_ECUDA, "SortByKeyNoAlloc: %s", cudaGetErrorString(e));
  uint32_t herr = 0;
  e = cudaMemcpyAsync(&herr, s.err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess)
    return set_error(SPHPC_ECUDA, "SortByKeyNoAlloc: %s", cudaGetErrorString(e));
  if (herr)
    return set_error(SPHPC_EKERNEL, "SortByKeyNoAlloc: sort reported error bits 0x%x", herr);
  return SPHPC_OK;
}
