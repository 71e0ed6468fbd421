// kernels.cuh -- host-side launch wrappers of the PBF pipeline kernels.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "radix_sort.cuh"
#include "sphpc_dev.cuh"

namespace sphpc {

constexpr int kBlock = 256;

inline int grid_for(int n, int block = kBlock) { return n > 0 ? (n + block - 1) / block : 1; }

// ---- hash / sort / cells / reorder / neighbour build (grid.cu) ----

// Fused ApplyGravity + PredictPositions + HashParticles (particles.c:516-527,
// 748-784, neighbors.c:101-125) for the whole-step driver: from x and v in
// slot order, computes the canonical x*, its cell key, and scatters the key
// and the slot into original-index order.  When `predict` is false the
// current x* (pos + disp) is hashed instead.  Accumulates the radix digit
// histograms of all `passes` into hist.
void launch_hash(const DevParams& P, const PD* pd, const float4* vel, const uint32_t* ids,
                 uint32_t* keys_by_id, uint32_t* loc_by_id, uint32_t* hist, int passes,
                 bool predict, uint32_t* err, cudaStream_t st);

// Reorder gather: new slot j takes particle sorted_ids[j] from its old slot.
// predict: recompute x* from x and v (+gravity) as launch_hash did, else
// gather d.  Writes the records, x* as FP32 (xsa) and cellp (packed cell of
// x*).  Optional extra float4 / float fields are gathered too (nullptr to
// skip).
struct ReorderExtra {
  const float4* in4[6];
  float4* out4[6];
  const float* in1[4];
  float* out1[4];
  // carried warm start: records {x*, carry_src[old slot]} into nr_carry
  const float* carry_src;
  uint4* nr_carry;
};
void launch_reorder(const DevParams& P, const uint32_t* sorted_ids, const uint32_t* loc_by_id,
                    const PD* pd_in, const float4* vel_in, PD* pd_out, float4* vel_out,
                    float4* xsa, uint4* nr_out, uint32_t* cellp, bool predict, bool move_vel,
                    const ReorderExtra* extra, cudaStream_t st);

// Cell start table cstart[0..C] from sorted keys (lower bounds; cstart[C]=n).
// gaps: worklist scratch of >= n + 2 + C/4096 + 2 uint4 entries; gap_count:
// one u32.
void launch_cell_starts(const uint32_t* keys_sorted, int n, uint32_t ncells, uint32_t* cstart,
                        uint4* gaps, uint32_t* gap_count, uint32_t* err, cudaStream_t st);

// Neighbour build (FillNeighbors, neighbors.c:217-298): per particle, its
// bucket of neighbour slots (four-entry blocks nbr4[j / 4][p], entries past
// the count in the last block set to p) and its size ncount[p].
void launch_build_neighbors(const DevParams& P, const NbrView& V, const PD* pd,
                            const float4* xsa, const uint32_t* cellp, uint32_t* nbr,
                            uint8_t* ncount, cudaStream_t st);

// Export the buckets in original-index space: nbr[id*60 + j], count[id];
// raises kErrNbrTail in err if a list's last block does not hold p past the
// count.
void launch_export_buckets(const NbrView& V, const uint32_t* ids, uint32_t* nbr, int32_t* count,
                           uint32_t* err, cudaStream_t st);

// ---- PBF passes (pbf.cu) ----

struct PassArgs {
  const PD* pd;        // particle records {x, d} (own reads only)
  PD* pd_out;          // particle records written by the pass (never pd)
  const uint4* nr;     // 16-byte neighbour records read by the pass
  uint4* nr_out;       // neighbour records written by the pass (never nr)
  float4* vel;
  float4* vel_out;
  float* rho;
  float* lam;
  float4* dp;          // UpdateDPs output (per-function path)
  float4* color;
  float4* omega;
  double* resid;       // [0] max density error bits (as u64), [1] sum
  float stiffness;     // UpdateDPs stiffness for this substep
  int last;            // fused position pass: also UpdateVelocities
  int write_pos;       // post pass: also UpdatePositions
  float* lam_acc;      // position pass: multiplier applied so far this step,
                       // sum of stiffness * lambda_p (null: not kept)
  int acc_add;         // 1: add to lam_acc, 0: start it with this pass
  const NV* nv;        // post passes: {record, colour or velocity} gathered
  NV* nv_out;          // post passes: {record, colour or velocity} for the next pass
};

// Density (+lambda) pass: ComputeDensities (particles.c:461-514) and
// ComputeLambda (:588-666).  mode 0: both (records with lambda in d.w to
// pd_out, lam[] if set), mode 1: density only, mode 2: lambda only (reads
// rho[]).
void launch_density_lambda(const DevParams& P, const NbrView& V, const PassArgs& a, int mode,
                           bool residual, cudaStream_t st);
// First density/lambda pass of a step (mode 0 with residual) that also writes
// the warm-start network's 16 features of particles p < limit to feat[p][16].
void launch_features(const DevParams& P, const NbrView& V, const PassArgs& a, float* feat,
                     int limit, cudaStream_t st);
// The same pass writing the network's normalised BF16 input rows
// bf16((f - norm[0:16]) * norm[16:32]) to xbf[p][16] for every particle.
void launch_features_bf16(const DevParams& P, const NbrView& V, const PassArgs& a,
                          __nv_bfloat16* xbf, const float* norm, cudaStream_t st);
// target[p] += s * lambda_p (lambda in rec[p].d.w), p < limit.
void launch_accum_lambda(const uint4* rec, float s, float* target, int limit, cudaStream_t st);
// Position pass: UpdateDPs (:668-746) with lambda from d.w; mode 0 fuses
// UpdatePositionStars (:529-564, clamp + SDF collision) and, if a.last,
// UpdateVelocities (:787-838); mode 1 writes dp[] only.
void launch_position(const DevParams& P, const NbrView& V, const PassArgs& a, int mode,
                     cudaStream_t st);
// UpdatePositionStars alone, in place on pd_out: d += dp, clamp, SDF.
void launch_apply_dp(const DevParams& P, const PassArgs& a, cudaStream_t st);
// nv[p] = {nr[p], e[p]}: the combined records of a post pass whose
// producer did not write them.
void launch_pack_nv(int n, const uint4* nr, const float4* e, NV* nv, cudaStream_t st);
// ComputeSurfaceTension colour pass (:94-140) and force pass (:142-204).
// The colour pass gathers nr (neighbour densities in w) and writes color[]
// and nv_out = {nr, colour}; the force pass gathers nv, updates vel in place
// and, if nv_out is set, writes {nr, new velocity} there.
void launch_color(const DevParams& P, const NbrView& V, const PassArgs& a, cudaStream_t st);
void launch_tension(const DevParams& P, const NbrView& V, const PassArgs& a, cudaStream_t st);
// ApplyViscosity (:383-459) as a Jacobi update of the velocities in nv into
// vel_out (and, if set, nv_out = {nr, new velocity}); with write_pos also
// UpdatePositions into pd_out.
void launch_xsph(const DevParams& P, const NbrView& V, const PassArgs& a, cudaStream_t st);
// ComputeVorticity (:207-283) from the velocities in nv;
// ApplyVorticityConfinement (:285-381) updates vel in place.
void launch_vorticity(const DevParams& P, const NbrView& V, const PassArgs& a, cudaStream_t st);
void launch_confinement(const DevParams& P, const NbrView& V, const PassArgs& a, bool omega_in_nr,
                        cudaStream_t st);
// Pointwise steps.
void launch_gravity(const DevParams& P, float4* vel, cudaStream_t st);
void launch_predict(const DevParams& P, PD* pd, const float4* vel, cudaStream_t st);
// With nr, also nr[p].w = w_src[p] (the records' payload for the post passes).
void launch_update_velocities(const DevParams& P, const PD* pd, float4* vel, cudaStream_t st,
                              const float* w_src = nullptr, uint4* nr = nullptr);
void launch_update_positions(const DevParams& P, PD* pd, cudaStream_t st);
// d.w and/or the record payload <- src[p] (a per-particle scalar for the
// neighbour passes; null pd or nr skips it).
void launch_pack_w(const DevParams& P, PD* pd, uint4* nr, const float* src, cudaStream_t st);
// Neighbour records from particle records: canonical x* and payload src[p]
// (d.w when src is null).
void launch_make_nr(const DevParams& P, const PD* pd, const float* src, uint4* nr,
                    cudaStream_t st);
// CalculateParticleCollisions seam on device double arrays.
void launch_collisions_double(const DevParams& P, double* x, double* y, double* z, int n,
                              cudaStream_t st);

// ---- slab decomposition along x (slab.cu) ----

// One particle between ranks: {x, y, z, gid bits}, {vx, vy, vz, flags bits}
// (flags bit 0: owned by the receiver).
struct __align__(32) SlabRecord {
  float4 a, b;
};
// Three record arrays read as one concatenation (kept, from the left, from
// the right).
struct SlabParts {
  const SlabRecord* p0;
  const SlabRecord* p1;
  const SlabRecord* p2;
  uint32_t n0, n1, n2;
};
// gid[i] = first + i for host index i; owned[i] when the particle's
// position lies in [lo, hi) (a side without a neighbour owns everything
// beyond it).
void launch_slab_init(int n, const uint32_t* ids, const PD* pd, uint32_t first_gid, double lo,
                      double hi, bool has_left, bool has_right, uint32_t* gid, uint8_t* owned,
                      cudaStream_t st);
// Sorts the owned particles of the working set (slot order, host index
// ids[j]) into kept / to-the-left / to-the-right records by their
// step-start position (counters[0..2], capacities cap_keep / cap_send:
// records past a capacity are counted, not written).
void launch_slab_pack(int n, const uint32_t* ids, const uint32_t* gid, const uint8_t* owned,
                      const PD* pd, const float4* vel, double lo, double hi, double R,
                      bool has_left, bool has_right, SlabRecord* keep, SlabRecord* send_l,
                      SlabRecord* send_r, uint32_t* counters, uint32_t cap_keep,
                      uint32_t cap_send, cudaStream_t st);
// keys[k] = gid of record k of the concatenation.
void launch_slab_keys(const SlabParts& s, uint32_t* keys, cudaStream_t st);
// Slot k (and host index k) of the new working set <- record perm[k].
void launch_slab_load(const SlabParts& s, const uint32_t* perm, PD* pd, float4* vel,
                      uint32_t* gid, uint8_t* owned, uint32_t* ids, cudaStream_t st);
// Records of the owned particles (unordered; *counter of them).
void launch_slab_owned(int n, const uint32_t* ids, const uint32_t* gid, const uint8_t* owned,
                       const PD* pd, const float4* vel, SlabRecord* out, uint32_t* counter,
                       uint32_t cap, cudaStream_t st);

}  // namespace sphpc
