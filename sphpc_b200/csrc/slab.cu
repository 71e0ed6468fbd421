// slab.cu -- device side of the slab decomposition along x (the reference's
// Simulation/src/communication.c:222-753 and geometry.c:102-166).
//
// The reference exchanges a halo of width h before the neighbour search and
// refreshes the halo's scalars and tuples after every pass (2I + 5 MPI round
// trips per step, UpdateHaloScalar / UpdateHaloTuple).  Here one exchange per
// step carries everything the step needs: every rank works on its own
// particles plus copies of its neighbours' particles within a halo width R
// that covers every neighbour hop of the step (2I in the constraint solve, 2
// for surface tension, 1 for XSPH, 2 for vorticity confinement, one h each,
// plus the motion of a step).  The halo's own results go stale from the
// outside in, never further than those hops, so the owned particles' results
// are those of the undivided domain; ownership moves to the neighbour when a
// particle's position leaves the slab (ExchangeOOB), in the same message.
//
// A record carries a particle between ranks: {x, y, z, gid} and
// {vx, vy, vz, flags}, 32 bytes (flags bit 0: the receiver owns it).
#include "kernels.cuh"

namespace sphpc {

namespace {

__device__ __forceinline__ void put_record(SlabRecord* buf, uint32_t* counter, uint32_t cap,
                                           const float4 x, uint32_t gid, const float4 v,
                                           uint32_t flags) {
  const uint32_t k = atomicAdd(counter, 1u);
  if (k < cap) {
    buf[k].a = make_float4(x.x, x.y, x.z, __uint_as_float(gid));
    buf[k].b = make_float4(v.x, v.y, v.z, __uint_as_float(flags));
  }
}

// Classifies every particle of the working set by its step-start position
// x (ExchangeOOB's CopyIfLessThan / CopyIfGreaterThan, communication.c:
// 465-491, and ExchangeHalo's edge selection, :232-247):
//   owned, lo <= x < hi: kept as owned; a copy to the left neighbour when
//     x < lo + R, to the right one when x >= hi - R;
//   owned, x < lo (x >= hi): ownership to the left (right) neighbour, kept
//     here as a halo copy when within R of the slab;
//   halo: dropped (its owner sends a fresh copy).
// A side without a neighbour owns everything beyond it.
__global__ void __launch_bounds__(256)
    k_slab_pack(int n, const uint32_t* __restrict__ ids, const uint32_t* __restrict__ gid,
                const uint8_t* __restrict__ owned, const PD* __restrict__ pd,
                const float4* __restrict__ vel, double lo, double hi, double R, int has_left,
                int has_right, SlabRecord* keep, SlabRecord* send_l, SlabRecord* send_r,
                uint32_t* __restrict__ counters, uint32_t cap_keep, uint32_t cap_send) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t i = __ldg(ids + j);
  if (!__ldg(owned + i)) return;
  float4 x, d;
  ld_pd(pd, j, x, d);
  const double xs = xstar_d(x.x, d.x);
  const float4 xf = make_float4((float)xs, (float)xstar_d(x.y, d.y), (float)xstar_d(x.z, d.z), 0.f);
  const float4 v = __ldg(vel + j);
  const uint32_t g = __ldg(gid + i);
  const bool go_left = has_left && xs < lo;
  const bool go_right = has_right && xs >= hi;
  if (go_left || go_right) {
    put_record(go_left ? send_l : send_r, counters + (go_left ? 1 : 2), cap_send, xf, g, v, 1u);
    const double depth = go_left ? lo - xs : xs - hi;
    if (depth < R) put_record(keep, counters, cap_keep, xf, g, v, 0u);
    return;
  }
  put_record(keep, counters, cap_keep, xf, g, v, 1u);
  if (has_left && xs < lo + R) put_record(send_l, counters + 1, cap_send, xf, g, v, 0u);
  if (has_right && xs >= hi - R) put_record(send_r, counters + 2, cap_send, xf, g, v, 0u);
}

__device__ __forceinline__ const SlabRecord& record_at(const SlabParts& s, uint32_t k) {
  if (k < s.n0) return s.p0[k];
  k -= s.n0;
  if (k < s.n1) return s.p1[k];
  return s.p2[k - s.n1];
}

__global__ void __launch_bounds__(256) k_slab_keys(SlabParts s, uint32_t* __restrict__ keys) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= s.n0 + s.n1 + s.n2) return;
  keys[k] = __float_as_uint(record_at(s, k).a.w);
}

// Slot s of the new working set takes the record of rank s in gid order
// (the host order of the set is gid order, so the neighbour buckets list
// each cell's particles in gid order as the undivided domain does).
__global__ void __launch_bounds__(256)
    k_slab_load(SlabParts s, const uint32_t* __restrict__ perm, PD* __restrict__ pd,
                float4* __restrict__ vel, uint32_t* __restrict__ gid, uint8_t* __restrict__ owned,
                uint32_t* __restrict__ ids) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= s.n0 + s.n1 + s.n2) return;
  const SlabRecord& r = record_at(s, __ldg(perm + k));
  st_pd(pd, (int)k, make_float4(r.a.x, r.a.y, r.a.z, 0.f), make_float4(0.f, 0.f, 0.f, 0.f));
  vel[k] = make_float4(r.b.x, r.b.y, r.b.z, 0.f);
  gid[k] = __float_as_uint(r.a.w);
  owned[k] = (uint8_t)(__float_as_uint(r.b.w) & 1u);
  ids[k] = k;
}

__global__ void __launch_bounds__(256)
    k_slab_owned(int n, const uint32_t* __restrict__ ids, const uint32_t* __restrict__ gid,
                 const uint8_t* __restrict__ owned, const PD* __restrict__ pd,
                 const float4* __restrict__ vel, SlabRecord* out, uint32_t* counter,
                 uint32_t cap) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t i = __ldg(ids + j);
  if (!__ldg(owned + i)) return;
  float4 x, d;
  ld_pd(pd, j, x, d);
  const float4 xf = make_float4((float)xstar_d(x.x, d.x), (float)xstar_d(x.y, d.y),
                                (float)xstar_d(x.z, d.z), 0.f);
  put_record(out, counter, cap, xf, __ldg(gid + i), __ldg(vel + j), 1u);
}

// gid = first + host index; owned when the position lies in the slab (a
// side without a neighbour owns everything beyond it).
__global__ void k_slab_init(int n, const uint32_t* __restrict__ ids, const PD* __restrict__ pd,
                            uint32_t first, double lo, double hi, int has_left, int has_right,
                            uint32_t* gid, uint8_t* owned) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t i = __ldg(ids + j);
  float4 x, d;
  ld_pd(pd, j, x, d);
  const double xs = xstar_d(x.x, d.x);
  gid[i] = first + i;
  owned[i] = (uint8_t)((!has_left || xs >= lo) && (!has_right || xs < hi));
}

}  // namespace

void launch_slab_init(int n, const uint32_t* ids, const PD* pd, uint32_t first_gid, double lo,
                      double hi, bool has_left, bool has_right, uint32_t* gid, uint8_t* owned,
                      cudaStream_t st) {
  if (n <= 0) return;
  k_slab_init<<<grid_for(n), kBlock, 0, st>>>(n, ids, pd, first_gid, lo, hi, has_left ? 1 : 0,
                                              has_right ? 1 : 0, gid, owned);
}

void launch_slab_pack(int n, const uint32_t* ids, const uint32_t* gid, const uint8_t* owned,
                      const PD* pd, const float4* vel, double lo, double hi, double R,
                      bool has_left, bool has_right, SlabRecord* keep, SlabRecord* send_l,
                      SlabRecord* send_r, uint32_t* counters, uint32_t cap_keep,
                      uint32_t cap_send, cudaStream_t st) {
  if (n <= 0) return;
  k_slab_pack<<<grid_for(n), 256, 0, st>>>(n, ids, gid, owned, pd, vel, lo, hi, R,
                                           has_left ? 1 : 0, has_right ? 1 : 0, keep, send_l,
                                           send_r, counters, cap_keep, cap_send);
}

void launch_slab_keys(const SlabParts& s, uint32_t* keys, cudaStream_t st) {
  const int m = (int)(s.n0 + s.n1 + s.n2);
  if (m <= 0) return;
  k_slab_keys<<<grid_for(m), 256, 0, st>>>(s, keys);
}

void launch_slab_load(const SlabParts& s, const uint32_t* perm, PD* pd, float4* vel,
                      uint32_t* gid, uint8_t* owned, uint32_t* ids, cudaStream_t st) {
  const int m = (int)(s.n0 + s.n1 + s.n2);
  if (m <= 0) return;
  k_slab_load<<<grid_for(m), 256, 0, st>>>(s, perm, pd, vel, gid, owned, ids);
}

void launch_slab_owned(int n, const uint32_t* ids, const uint32_t* gid, const uint8_t* owned,
                       const PD* pd, const float4* vel, SlabRecord* out, uint32_t* counter,
                       uint32_t cap, cudaStream_t st) {
  if (n <= 0) return;
  k_slab_owned<<<grid_for(n), 256, 0, st>>>(n, ids, gid, owned, pd, vel, out, counter, cap);
}

}  // namespace sphpc
