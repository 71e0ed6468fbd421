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

/* No counterpart in the reference.  The same stable sort as SortByKey for
 * callers that must not allocate device memory (a host that owns all device
 * memory through its own pool, or a time-critical loop where a cudaMalloc,
 * which can synchronise the device or fail under memory pressure, is not
 * acceptable).  Its scratch is a fixed array of about 2.4 MB inside the
 * library, held by every GPU that loads the library until the process exits,
 * so count is limited to 262,144 pairs (larger counts return SPHPC_EINVAL).
 * It calls no cudaMalloc or cudaFree.  The first call on a device, and the
 * first after the device's context has been replaced (cudaDeviceReset),
 * looks up the array's device address (cudaGetSymbolAddress).  All calls on
 * a device share the one array: calls that overlap on the GPU (from several
 * host threads or streams) race and must be serialised by the caller.  Each
 * call waits on the host until its sort has finished on cuda_stream (it
 * reads back the sort's error word). */
int SortByKeyNoAlloc(unsigned int *const keys, unsigned int *const values, const int count,
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

/* No counterpart in the reference (its Thrust seam has no waits,
 * thrust_c.cu:86-91).  Failure-detection checks of the library's bounded
 * device waits: each runs one block that waits, with the given poll limit,
 * on a flag nothing ever sets -- a radix-sort look-back flag of an earlier
 * tile (SortByKey's onesweep passes wait up to 2^22 polls), or a
 * tensor-core completion mbarrier (the warm-start network's kernels wait up
 * to 2^20 polls).  The wait gives up, the kernel records an error bit and
 * returns, and the call returns SPHPC_EKERNEL with *error_bits set (2 for
 * the sort, 16 for the mbarrier); SPHPC_OK would mean the wait ended by
 * itself.  The device stays usable afterwards. */
int sphpc_check_sort_wait(int spin_limit, unsigned int *error_bits);
int sphpc_check_mbarrier_wait(int poll_limit, unsigned int *error_bits);

/* No counterpart in the reference.  Failure injection for the allocation
 * error paths: after `after` more device allocations of a particle set have
 * succeeded, the next one fails with SPHPC_ENOMEM (without calling
 * cudaMalloc) and the injection switches itself off; -1 switches it off. */
int sphpc_fail_device_alloc(int after);

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
