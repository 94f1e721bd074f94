// ne2b_step_k11.cu — step kernel instances: int32 fixed-point ring, with the AdEx path.
#include "ne2b_step.cuh"

namespace ne2b {
template struct StepKind<true, true>;
}  // namespace ne2b
