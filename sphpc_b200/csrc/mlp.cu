// mlp.cu -- learned warm start (not built yet: reports "not loaded").
#include "host_internal.h"
#include "mlp.cuh"

namespace sphpc {

int mlp_warm_start(MlpState& m, const DevParams&, const NbrView&, const PD*, PD*,
                   const float4*, const uint8_t*, cudaStream_t) {
  (void)m;
  return set_error(SPHPC_ENOTREADY, "warm start: no network loaded");
}

}  // namespace sphpc
