/*
 * sphpc_device.h -- the reference's device-library seam, re-implemented with
 * this library's own sm_100a kernels (no Thrust, no texture objects).  Same
 * names and argument lists as the functions the reference's C code calls
 * through `#pragma acc host_data use_device`; all pointers are device
 * pointers, cuda_stream is a cudaStream_t (NULL = legacy default stream).
 */
#ifndef SPHPC_DEVICE_H_
#define SPHPC_DEVICE_H_

#include "sphpc_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* thrust_c.h:41-44 (thrust_c.cu:86-91): stable sort of (keys, values) by
 * key.  Scratch memory is allocated by the library and cached. */
int SortByKey(unsigned int *const keys, unsigned int *const values, const int count,
              const void *const cuda_stream);

/* thrust_c.h:46-50 (thrust_c.cu:93-105): start_indices[c] =
 * lower_bound(hash_values[0..value_count), c) for c in [0, search_count). */
int FindLowerBounds(const unsigned int *const hash_values, const int value_count,
                    const int search_count, unsigned int *const start_indices,
                    const void *const cuda_stream);

/* thrust_c.h:59-63 (thrust_c.cu:107-120): upper_bound, same layout. */
int FindUpperBounds(const unsigned int *const hash_values, const int value_count,
                    const int search_count, unsigned int *const end_indices,
                    const void *const cuda_stream);

/* obstacle_cuda.h:23-27 (obstacle_cuda.cu:118-131): pushes every particle
 * whose double position lies inside the obstacle out along the SDF normal.
 * The obstacle must have been uploaded (AllocInitObstacle / _CUDA).  Runs on
 * the legacy default stream, as the reference's launch does. */
int CalculateParticleCollisions(double *x, double *y, double *z, const int particle_count,
                                const struct Obstacle obstacle);

/* obstacle_cuda.h:19-21: device copy of obstacle->SDF_buffer. */
int AllocInitObstacle_CUDA(struct Obstacle *obstacle);
int FinalizeObstacle_CUDA(struct Obstacle_CUDA *obstacle_cuda);

#ifdef __cplusplus
}
#endif

#endif
