/*
 * sphpc.h -- host C API of libsphpc_cuda.so, the B200 replacement for
 * SPHPC's per-step particle pipeline.
 *
 * The reference keeps its particle arrays on the GPU with OpenACC data
 * directives and calls its step functions on the "present" copies.  This
 * library does the same with an explicit mirror: AllocInitParticles (or
 * sphpc_enter_data) creates the device copy of a struct Particles, every
 * step function below works on that copy, and sphpc_update_host /
 * sphpc_update_device play the role of `#pragma acc update`.  The device
 * copy is FP32 in cell-sorted order; the host arrays stay FP64 in the
 * reference's original-index order.
 *
 * Every function returns 0 on success and a negative SPHPC_E* code on
 * failure (the reference exits the process instead); sphpc_last_error()
 * describes the last failure of the calling thread.  Nothing here falls
 * back to the CPU: without a usable CUDA device every device call fails
 * with SPHPC_ECUDA.
 */
#ifndef SPHPC_H_
#define SPHPC_H_

#include "sphpc_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define SPHPC_OK 0
#define SPHPC_EINVAL (-1)   /* bad argument or unsupported configuration */
#define SPHPC_EIO (-2)      /* file missing or malformed */
#define SPHPC_ECUDA (-3)    /* CUDA runtime error / no device */
#define SPHPC_ENOMEM (-4)   /* host or device allocation failed */
#define SPHPC_ENOTREADY (-5)/* object not initialised (no device copy) */
#define SPHPC_EKERNEL (-6)  /* a kernel reported an error (see message) */

const char *sphpc_last_error(void);
const char *sphpc_version(void);

/* ---------------- configuration ---------------- */

/* Reference values of every hard-coded constant. */
void sphpc_default_solver(struct SphpcSolver *solver);
/* Solver settings used by the next AllocInitParticles / sphpc_enter_data
 * (the configuration loaders set them too). */
void sphpc_set_default_solver(const struct SphpcSolver *solver);

/* ReadParameters, input_parser.h:16-20: reads ./sim-config.ini.  The
 * [Obstacle] section is optional here (required by the reference). */
int ReadParameters(struct Params *parameters, struct Particles *particles,
                   struct AABB *boundary_volume, struct AABB *initial_fluid_volume,
                   struct Obstacle *obstacle);

/* SetParameters, simulation.h:28-33 / simulation.c:130-178: ReadParameters
 * plus particle spacing, h = 2 spacing, dq = 0.1 h and kernel norms. */
int SetParameters(struct Params *params, struct Particles *particles,
                  struct Neighbors *neighbors, struct AABB *boundary_global,
                  struct AABB *water_volume_global, struct Obstacle *obstacle);

/* SetParameters for an INI file at `path`, also reading the optional
 * extension keys into `solver` (may be NULL). */
int sphpc_load_config(const char *path, struct Params *params, struct Particles *particles,
                      struct AABB *boundary_global, struct AABB *water_volume_global,
                      struct Obstacle *obstacle, struct SphpcSolver *solver);

/* SetParticleNumbers, geometry.h:21-24 (the communication argument of the
 * reference is accepted and ignored: single rank). */
int SetParticleNumbers(const struct AABB *fluid_global, struct Particles *particles,
                       struct Params *params, void *communication);

/* ConstructFluidVolume, geometry.h:16-18: cell-centred lattice plus the
 * solver's seeded jitter; sets local_count, global_count, fluid_volume. */
int ConstructFluidVolume(struct Particles *particles, struct Params *params,
                         const struct AABB *fluid);

/* ---------------- particles (particles.h:44-108) ---------------- */

/* Host arrays (max_local each), lattice, rest state, device copy. */
int AllocInitParticles(struct Particles *particles, struct Params *params,
                       struct AABB *fluid_volume_initial);
int FinalizeParticles(struct Particles *particles);

/* Device copy of host arrays that were filled by the caller (acc enter data
 * copyin); uses x, y, z, v, x_star (when non-NULL) and density. */
int sphpc_enter_data(struct Particles *particles, const struct Params *params);
int sphpc_exit_data(struct Particles *particles);
int sphpc_update_host(struct Particles *particles);    /* device -> host, all fields */
/* Selected fields only: bit k of field_mask is the k-th double array of
 * struct Particles (0 x_star ... 3 x, 4 y, 5 z ... 18 density, 19 lambda),
 * e.g. (1<<3)|(1<<4)|(1<<5)|(1<<18) for the output frame of
 * fileio_adios.c:73-76. */
int sphpc_update_host_fields(struct Particles *particles, unsigned int field_mask);
/* The same read-back, returning once it is enqueued: the fields are gathered
 * on the particle set's stream and copied to the host arrays on a copy
 * stream of the particle set, so the steps that follow run while the frame
 * crosses the link.  The host arrays hold the frame only after
 * sphpc_host_wait; every other transfer of the set (and the next
 * asynchronous read-back) waits for it first.  No counterpart in the
 * reference, whose acc update host waits for the copy. */
int sphpc_update_host_fields_async(struct Particles *particles, unsigned int field_mask);
int sphpc_host_wait(struct Particles *particles);
/* Host -> device of selected field groups (same bit numbering; a group
 * such as x/y/z is uploaded when all its bits are set; x/y/z are required). */
int sphpc_update_device_fields(struct Particles *particles, unsigned int field_mask);
int sphpc_update_device(struct Particles *particles);  /* host -> device, all fields */
/* Solver settings of this particle set (copied). */
int sphpc_set_solver(struct Particles *particles, const struct SphpcSolver *solver);
int sphpc_get_solver(const struct Particles *particles, struct SphpcSolver *solver);
/* CUDA stream (cudaStream_t) the particle set's kernels run on. */
int sphpc_set_stream(struct Particles *particles, void *cuda_stream);

int ApplyGravity(struct Particles *fluid_particles, const struct Params *params);
int PredictPositions(struct Particles *particles, const struct Params *params,
                     const struct AABB *boundary_global);
int ComputeDensities(struct Particles *fluid_particles, const struct Params *params,
                     const struct Neighbors *neighbors);
int ComputeLambda(struct Particles *fluid_particles, const struct Params *params,
                  const struct Neighbors *neighbors);
int UpdateDPs(struct Particles *fluid_particles, const struct Params *params,
              const struct Neighbors *neighbors, const int substep);
int UpdatePositionStars(struct Particles *particles, const struct AABB *boundary_global,
                        const struct Obstacle *obstacle, const struct Params *params);
int UpdateVelocities(struct Particles *fluid_particles, const struct Params *params);
int ComputeSurfaceTension(struct Particles *particles, const struct Params *params,
                          const struct Neighbors *neighbors);
int ApplyViscosity(struct Particles *fluid_particles, const struct Params *params,
                   const struct Neighbors *neighbors);
int ComputeVorticity(struct Particles *particles, const struct Params *params,
                     const struct Neighbors *neighbors);
int ApplyVorticityConfinement(struct Particles *fluid_particles, const struct Params *params,
                              const struct Neighbors *neighbors);
int UpdatePositions(struct Particles *fluid_particles);

/* ---------------- neighbours (neighbors.h:30-47) ---------------- */

int AllocInitNeighbors(struct Neighbors *neighbors, const struct Particles *particles,
                       const struct Params *params, const struct AABB *boundary_global);
int FinalizeNeighbors(struct Neighbors *neighbors);
/* HashParticles + SortHash + FindCellBounds + FillNeighbors on the device
 * copy of `particles` (also reorders the device copy by cell). */
int FindAllNeighbors(const struct Particles *particles, const struct Params *params,
                     struct Neighbors *neighbors);
/* The current neighbour buckets in the reference's layout and index space:
 * indices[id*60 + j] (original indices), counts[id]. */
int sphpc_get_neighbor_buckets(const struct Particles *particles, unsigned int *indices,
                               int *counts);
/* Sorted hash keys, sorted original ids (SortHash result) and the cell start
 * table (FindLowerBounds over all cells, plus the trailing count), as the
 * reference holds hash_values / particle_ids / start_indices. */
int sphpc_get_cell_data(const struct Particles *particles, unsigned int *hash_values,
                        unsigned int *particle_ids, unsigned int *start_indices);

/* No counterpart in the reference (whose FillNeighbors tests every pair in
 * FP64, neighbors.c:278-285).  1 if the neighbour build's FP32 candidate
 * pre-test decides r^2 < h^2 exactly as that FP64 test does for
 * coordinates of magnitude up to max_coord (it leaves pairs within
 * +-2^-10 h^2 of h^2 to the FP64 test); 0 otherwise, in which case the
 * build sends every candidate to the FP64 test.  The build applies it with
 * max_coord = h * max(hash_size_x, hash_size_y, hash_size_z). */
int sphpc_neighbor_pretest_fp32_safe(double max_coord, double h);

/* ---------------- slab decomposition along x (communication.c) ---------------- */

/* The reference splits the domain into x-slabs, one per MPI rank: it trades
 * particles that left a slab (ExchangeOOB, communication.c:453-585), copies
 * a halo of width h (ExchangeHalo, :222-321) and refreshes the halo's
 * scalars and tuples after every pass (UpdateHaloScalar / UpdateHaloTuple,
 * :587-753).  Here one exchange per step does all of it: each rank's
 * working set is its own particles plus copies of its neighbours' particles
 * within a halo width (sphpc_slab_halo_width) that covers every neighbour
 * hop of a step, so its own particles' results are those of the undivided
 * domain (bit for bit: the set is kept in global-id order, so buckets list
 * each cell's particles in the same order).  Records (32 bytes each:
 * {x, y, z, gid}, {vx, vy, vz, flags}) are device memory the caller moves
 * between ranks (NCCL send/recv, or a peer copy).  A slab steps with the
 * fixed iteration count (adaptive and warm_start off). */

/* Makes the device copy a slab [node_start_x, node_end_x) of a decomposed
 * domain (has_left / has_right: whether neighbours exist; a side without
 * one owns everything beyond it): global ids first_gid + host index, and
 * the particles inside owned.  Every rank may start from the whole scene;
 * the particles it does not own leave at the first sphpc_slab_pack. */
int sphpc_slab_init(struct Particles *particles, unsigned int first_gid, double node_start_x,
                    double node_end_x, int has_left, int has_right);
/* Halo width one exchange per step needs for these solver settings. */
int sphpc_slab_halo_width(const struct Params *params, const struct SphpcSolver *solver,
                          double *width);
/* Sorts the owned particles by their position at the start of the next
 * step against [node_start_x, node_end_x): records for the left and right
 * neighbours (has_left / has_right: whether they exist) into send_left /
 * send_right (device memory, send_capacity records each), the rest kept.
 * Returns the record counts. */
int sphpc_slab_pack(struct Particles *particles, double node_start_x, double node_end_x,
                    double halo_width, int has_left, int has_right, void *send_left,
                    void *send_right, int send_capacity, int *count_left, int *count_right);
/* Rebuilds the working set from the kept records and the neighbours'
 * (device memory) in global-id order; sets local_count. */
int sphpc_slab_unpack(struct Particles *particles, const void *recv_left, int count_left,
                      const void *recv_right, int count_right);
/* The owned particles' global ids, positions and velocities (host arrays,
 * in no particular order); *count of them. */
int sphpc_slab_owned(const struct Particles *particles, unsigned int *gids, double *xyz,
                     double *vel, int capacity, int *count);
/* BalanceNodes (geometry.c:102-166) given the neighbours' particle counts
 * and slab lengths: moves params->node_start_x / node_end_x by h towards an
 * even share of global_count. */
int sphpc_balance_nodes(int rank, int proc_count, int num_rank, int num_right,
                        double length_left, double length_right, int global_count,
                        struct Params *params);

/* ---------------- obstacle (obstacle.h:32-33) ---------------- */

/* Reads the SDFGen ASCII file named in obstacle->SDF_file_name
 * (obstacle.c:13-79), fixes world_bounds' aspect ratio and uploads the SDF. */
int AllocInitObstacle(struct Obstacle *obstacle);
int FinalizeObstacle(struct Obstacle *obstacle);
/* The file-reading half of AllocInitObstacle (host only, no device):
 * fills SDF_dim_*, origin, SDF_spacing, SDF_buffer (malloc'd) and the
 * world_bounds aspect fix. */
int sphpc_read_sdf(struct Obstacle *obstacle);

/* ---------------- whole step ---------------- */

/* `steps` repetitions of the loop body of main (simulation.c:56-116):
 * gravity, predict, neighbours, the constraint loop with SDF collisions,
 * velocities, surface tension, XSPH viscosity, vorticity confinement,
 * positions -- fused into the pipeline's kernels.  obstacle may be NULL. */
int sphpc_step(struct Particles *particles, const struct Params *params,
               struct Neighbors *neighbors, const struct AABB *boundary_global,
               const struct Obstacle *obstacle, int steps);

/* FP64 diagnostics of the device copy (density error from the last density
 * evaluation, energy, centre of mass, momentum). */
int sphpc_diagnostics(const struct Particles *particles, struct SphpcDiag *diag);
/* Iterations, convergence and residual of the last sphpc_step. */
int sphpc_step_info(const struct Particles *particles, struct SphpcStepInfo *info);
/* Kernel-reported error bits since the last call (0 = none); clears them. */
int sphpc_device_errors(const struct Particles *particles, unsigned int *bits);

/* ---------------- obstacle tooling ---------------- */

/* Signed distance field of a closed triangle mesh on the device, in the
 * sample layout of the SDFGen files AllocInitObstacle reads (obstacle.c:13-79):
 * phi[i + dims[0] * (j + dims[1] * k)] at origin + (i, j, k) * dx, negative
 * inside; |phi| is the exact distance to the nearest triangle, the sign the
 * generalized winding number.  vertices[3 * n_vertices], triangles[3 *
 * n_triangles] (vertex indices) and phi are host memory.  The reference has
 * no counterpart (it reads files made by an external tool). */
int sphpc_mesh_sdf(const float *vertices, int n_vertices, const int *triangles, int n_triangles,
                   const int *dims, const double *origin, double dx, float *phi);

/* Particle-to-level-set surface of a snapshot on a dense device grid (the
 * operations of PostProcessing/OpenVDB/src/ConstructSurface.cc:39-72, which
 * uses OpenVDB sparse grids on the CPU): voxel size radius / 2, spheres of
 * the given radius rasterised as min(|x - p| - radius) within a band of
 * half_width voxels + radius, then dilated by radius, smoothed (three passes
 * of a 3-tap mean per axis) and eroded by radius.  xyz[3 * np] interleaved
 * doubles (the sim-N.bin layout), phi[i + dims[0] * (j + dims[1] * k)] at
 * origin + (i, j, k) * radius / 2, negative inside; host memory. */
int sphpc_particle_surface(const double *xyz, int np, double radius, int half_width,
                           const int *dims, const double *origin, float *phi);

/* ---------------- snapshot output ---------------- */

/* fileio_MPI_IO.h:15-27: output/sim-N.bin under the working directory, the
 * particles' x, y, z as interleaved doubles in original particle order.
 * WriteParticles gathers on the device and returns once the copy to the
 * page-locked write_buffer is queued; a host thread writes the file.  The
 * next WriteParticles, sphpc_fileio_wait and FinalizeFileIO wait for it and
 * return its outcome. */
int AllocInitFileIO(struct FileIO *const file_io, const struct Particles *const particles,
                    const struct Params *params);
int WriteParticles(const struct Particles *const particles, const struct Params *const params,
                   struct FileIO *const file_io);
int sphpc_fileio_wait(struct FileIO *file_io);
int FinalizeFileIO(struct FileIO *const file_io);

/* ---------------- learned warm start ---------------- */

/* Forward pass of the warm-start network on n feature rows d_feat[n][16]
 * (device memory) into d_out[n] (device), with the FP32 parameter vector
 * params[9473] (W1[64][16] b1 W2[64][64] b2 W3[64][64] b3 w4[64] b4) and
 * normalisation norm[33] (mean[16] inv_std[16] out_scale) on the host.
 * No counterpart in the reference. */
int sphpc_mlp_forward(const float *d_feat, int n, const float *params, const float *norm,
                      float *d_out, void *cuda_stream);

/* Gradient of the batch loss L = 1/(2n) sum_p (u_p - t_p / out_scale)^2 (u the
 * network output before out_scale) over n rows d_feat[n][16], d_target[n]
 * (device memory), through the tensor-core training kernels: grad_out[9473]
 * and *loss_out on the host.  No counterpart in the reference. */
int sphpc_mlp_grad(const float *d_feat, const float *d_target, int n, const float *params,
                   const float *norm, float *grad_out, float *loss_out, void *cuda_stream);

/* The process's training set of (features, target) rows, resident on the
 * device that reserved it.  reserve grows it (keeping the rows), clear empties
 * it, free releases it; append copies rows from the host; read copies rows
 * [offset, offset + count) to the host; stats writes the normalisation
 * norm[33] (feature means, 1/standard deviations, target standard deviation).
 * No counterpart in the reference. */
int sphpc_mlp_dataset_reserve(long long capacity);
int sphpc_mlp_dataset_size(long long *n);
int sphpc_mlp_dataset_clear(void);
int sphpc_mlp_dataset_free(void);
int sphpc_mlp_dataset_append(const float *feat, const float *target, long long count);
int sphpc_mlp_dataset_read(long long offset, long long count, float *feat, float *target);
int sphpc_mlp_dataset_stats(float *norm);

/* AdamW (beta 0.9/0.999, eps 1e-8, decoupled weight decay on weights only)
 * on the training set: `steps` steps of `batch` rows, each pass over the set
 * in a fresh seeded permutation, learning rate from lr to lr_final on a half
 * cosine (equal: constant); params_out[9473] and loss_out[steps] (batch loss
 * before each update, may be NULL) on the host.  No counterpart in the
 * reference. */
int sphpc_mlp_train(const float *params_in, const float *norm, int steps, int batch, float lr,
                    float lr_final, float weight_decay, unsigned long long seed,
                    float *params_out, float *loss_out);

/* One time step like sphpc_step with the plain solver at a fixed
 * `iterations`, appending one training row per particle (as many as fit):
 * the 16 features of the predicted state and target sum_k s_k lambda_k, the
 * stiffness-weighted multiplier sum of the solve.  Returns the rows appended
 * (>= 0) or an error code.  No counterpart in the reference. */
int sphpc_mlp_collect(struct Particles *particles, const struct Params *params,
                      struct Neighbors *neighbors, const struct AABB *boundary_global,
                      const struct Obstacle *obstacle, int iterations);

/* Installs (or removes) the network the warm start of sphpc_step uses when
 * the solver's warm_start is set: params[9473], norm[33] as above. */
int sphpc_mlp_load(struct Particles *particles, const float *params, const float *norm);
int sphpc_mlp_unload(struct Particles *particles);

/* Features [N][16] (by particle id, host memory) of the current device state;
 * call after FindAllNeighbors.  Overwrites no particle state. */
int sphpc_mlp_features(struct Particles *particles, const struct Params *params,
                       const struct AABB *boundary_global, const struct Obstacle *obstacle,
                       float *features);

/* Per-stage CUDA-event timing of the particle set's launches.  The last
 * entry sphpc_profile_read returns is "kernel_launches": the number of
 * kernels the particle set has launched in total (its launches field). */
int sphpc_profile(struct Particles *particles, int enable);
int sphpc_profile_read(const struct Particles *particles, struct SphpcKernelTime *out,
                       int max_entries, int *n_entries);

#ifdef __cplusplus
}
#endif

#endif
