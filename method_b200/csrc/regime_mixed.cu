// The mixed form of the fused REGIME tile: the stiff fluxes split and
// reconstructed in FP32 (the mixed form's flux arithmetic, FMA allowed), E,
// q, K's differences, the diffusion vectors and the state update in FP64.
#include <cuda_runtime.h>

#include "launch.h"
#include "regime_tile.cuh"

namespace mth {

cudaError_t launch_regime_tile_mixed(const Grid& g, int order, const double* cons,
                                     const double* prims, double* target, double dt,
                                     cudaStream_t st, bool ext_only) {
  return launch_regime_tile_order<float>(g, order, cons, prims, target, dt, st, ext_only);
}

}  // namespace mth
