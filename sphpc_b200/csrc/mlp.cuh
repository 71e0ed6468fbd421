// mlp.cuh -- learned warm start of the constraint solve (device state).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "sphpc_dev.cuh"

namespace sphpc {

struct MlpState {
  bool ready = false;
};

inline void mlp_release(MlpState& m) { m.ready = false; }

// Writes pd_out = {x, (d, lambda0)} for every particle from the network's
// prediction; returns a negative code when the network is not loaded.
int mlp_warm_start(MlpState& m, const DevParams& P, const NbrView& V, const PD* pd,
                   PD* pd_out, const float4* vel, const uint8_t* ncount, cudaStream_t st);

}  // namespace sphpc
