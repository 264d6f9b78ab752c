// Plain FP64 stage launchers.  Compiled with --fmad=false and IEEE division /
// square root so every stage repeats the reference's arithmetic operation by
// operation.
#include "stages.cuh"

namespace orion {
const StageOps& plain_ops() {
  static const StageOps ops = make_ops<double, double>();
  return ops;
}
}  // namespace orion
