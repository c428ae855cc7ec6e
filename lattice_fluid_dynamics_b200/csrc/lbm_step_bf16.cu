// Step-kernel instantiations for StoreBF16 populations.
#include "lbm_step.cuh"

namespace lbm {
template struct exact::StepLaunch<exact::StoreBF16>;
}  // namespace lbm
