// ne2b_step_k01.cu — step kernel instances: f32 ring, with the AdEx path.
#include "ne2b_step.cuh"

namespace ne2b {
template struct StepKind<false, true>;
}  // namespace ne2b
