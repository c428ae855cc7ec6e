// Step-kernel instantiations for StoreBF16 populations (exact arithmetic) and
// their launcher table.
#include "lbm_step.cuh"

namespace lbm {
template struct exact::StepLaunch<exact::StoreBF16>;
extern const StepOps step_ops_bf16 = exact::make_step_ops<exact::StoreBF16>();
}  // namespace lbm
