// host_internal.h -- shared host-side helpers of libsphpc_cuda.so.
#pragma once
#include <cstdint>
#include <string>

#include "../../include/sphpc.h"

// Return the CUDA call's error as SPHPC_ECUDA with its text and location.
#define SPHPC_CK(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return ::sphpc::set_error(SPHPC_ECUDA, "%s: %s (%s:%d)", #call,                  \
                                cudaGetErrorString(e_), __FILE__, __LINE__);            \
  } while (0)

// Return a non-zero status code unchanged.
#define SPHPC_RC(expr)      \
  do {                      \
    const int rc_ = (expr); \
    if (rc_) return rc_;    \
  } while (0)

namespace sphpc {

// Records a formatted error message for sphpc_last_error() and returns code.
int set_error(int code, const char* fmt, ...);
void clear_error();

// Default solver settings registered by the last configuration load
// (AllocInitParticles uses them when the particle set has none yet).
void set_current_solver(const SphpcSolver& s);
SphpcSolver current_solver();

// Sum of the poly6 kernel over a perfect cubic lattice of the given spacing
// (self included): rest density / particle mass for a lattice at rest.
double lattice_poly6_sum(double h, double W_norm, double spacing);

// SplitMix64-based counter uniform in [0,1) keyed by (seed, index, axis)
// (Steele, Lea, Flood, "Fast splittable pseudorandom number generators",
// OOPSLA 2014).
double counter_uniform01(uint64_t seed, uint64_t index, uint32_t axis);

// Launches, on the particle set's stream, the gather of its positions x, y, z
// as interleaved doubles d_out[3 * id + k] in original particle order;
// returns the particle count and the stream.
int sim_interleave_positions(const struct Particles* particles, double* d_out, int* n,
                             void** stream);

// Kernel norms of SetParameters (simulation.c:173-177).
void set_kernel_norms(Params* p);

}  // namespace sphpc
