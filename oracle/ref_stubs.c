/*
 * ref_stubs.c -- the device-library seam of the reference, restated on the
 * host so that the reference's own Simulation/src/particles.c and
 * Simulation/src/neighbors.c run unmodified on the CPU.
 *
 * TEST INFRASTRUCTURE ONLY: linked into oracle/_ref/libsphpc_ref.so, the
 * reference-built checker.  Nothing here is part of the product.
 *
 *   SortByKey / FindLowerBounds / FindUpperBounds  (thrust_c.cu:86-120)
 *   CalculateParticleCollisions                    (obstacle_cuda.cu:118-131)
 *   acc_get_cuda_stream                            (OpenACC runtime)
 *   ConstructFluidVolume                           (geometry.c, link only)
 */
#include <stddef.h>
#include <stdint.h>

#include "obstacle.h"
#include "pbf_oracle.h"

struct Particles;
struct Params;
struct AABB;

/* geometry.c:19-74 is not compiled (it needs MPI); AllocInitParticles
 * (particles.c:1032) references it but the harness never calls
 * AllocInitParticles -- it fills the arrays itself (ref_driver.c). */
void ConstructFluidVolume(struct Particles *const particles, struct Params *const params,
                          const struct AABB *const fluid) {
  (void)particles;
  (void)params;
  (void)fluid;
}

void *acc_get_cuda_stream(int async) {
  (void)async;
  return NULL;
}

void SortByKey(unsigned int *const keys, unsigned int *const values,
               const int count, const void *const cuda_stream) {
  (void)cuda_stream;
  oracle_sort_by_key(keys, values, count);
}

void FindLowerBounds(const unsigned int *const hash_values,
                     const int value_count, const int search_count,
                     unsigned int *const start_indices,
                     const void *const cuda_stream) {
  (void)cuda_stream;
  oracle_lower_bounds(hash_values, value_count, search_count, start_indices);
}

void FindUpperBounds(const unsigned int *const hash_values,
                     const int value_count, const int search_count,
                     unsigned int *const end_indices,
                     const void *const cuda_stream) {
  (void)cuda_stream;
  oracle_upper_bounds(hash_values, value_count, search_count, end_indices);
}

/* The reference kernel samples a CUDA texture; on the host the obstacle's
 * SDF_buffer (host copy, obstacle.c:44) is sampled by the oracle's tex3D
 * restatement. */
void CalculateParticleCollisions(double *x, double *y, double *z,
                                 const int particle_count,
                                 const struct Obstacle obstacle) {
  if (!obstacle.SDF_buffer) return;
  OracleParams p;
  p.sdf = obstacle.SDF_buffer;
  p.sdim[0] = obstacle.SDF_dim_x;
  p.sdim[1] = obstacle.SDF_dim_y;
  p.sdim[2] = obstacle.SDF_dim_z;
  p.sdf_spacing = obstacle.SDF_spacing;
  p.ob_min[0] = obstacle.world_bounds.min_x;
  p.ob_min[1] = obstacle.world_bounds.min_y;
  p.ob_min[2] = obstacle.world_bounds.min_z;
  p.ob_max[0] = obstacle.world_bounds.max_x;
  p.ob_max[1] = obstacle.world_bounds.max_y;
  p.ob_max[2] = obstacle.world_bounds.max_z;
  oracle_particle_collisions(&p, x, y, z, particle_count);
}
