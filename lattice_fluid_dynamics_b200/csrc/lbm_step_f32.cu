// Step-kernel instantiations for StoreF32 populations (exact arithmetic) and
// their launcher table.
#include "lbm_step.cuh"

namespace lbm {
template struct exact::StepLaunch<exact::StoreF32>;
extern const StepOps step_ops_f32 = exact::make_step_ops<exact::StoreF32>();
}  // namespace lbm
