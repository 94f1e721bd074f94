// ne2b_step_k10.cu — step kernel instances: int32 fixed-point ring, without the AdEx path.
#include "ne2b_step.cuh"

namespace ne2b {
template struct StepKind<true, false>;
}  // namespace ne2b
