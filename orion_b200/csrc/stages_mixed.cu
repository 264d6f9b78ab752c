// Mixed-precision stage launchers: FP32 storage and arithmetic for the flux,
// viscous and sweep stages (FP64 metrics, Q update and norms).  Compiled with
// contraction and approximate FP32 division / square root.
#include "stages.cuh"

namespace orion {
const StageOps& mixed_ops() {
  static const StageOps ops = make_ops<float, float>();
  return ops;
}
}  // namespace orion
