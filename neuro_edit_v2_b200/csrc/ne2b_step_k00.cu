// ne2b_step_k00.cu — step kernel instances: f32 ring, without the AdEx path.
#include "ne2b_step.cuh"

namespace ne2b {
template struct StepKind<false, false>;
}  // namespace ne2b
