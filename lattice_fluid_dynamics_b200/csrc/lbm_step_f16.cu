// Step-kernel instantiations for StoreF16 populations (exact arithmetic) and
// their launcher table.
#include "lbm_step.cuh"

namespace lbm {
template struct exact::StepLaunch<exact::StoreF16>;
extern const StepOps step_ops_f16 = exact::make_step_ops<exact::StoreF16>();
}  // namespace lbm
