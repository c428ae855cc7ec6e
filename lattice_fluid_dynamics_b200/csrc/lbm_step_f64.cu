// Step-kernel instantiations for StoreF64 populations (exact arithmetic) and
// their launcher table.
#include "lbm_step.cuh"

namespace lbm {
template struct exact::StepLaunch<exact::StoreF64>;
extern const StepOps step_ops_f64 = exact::make_step_ops<exact::StoreF64>();
}  // namespace lbm
