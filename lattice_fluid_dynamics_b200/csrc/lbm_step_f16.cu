// Step-kernel instantiations for StoreF16 populations.
#include "lbm_step.cuh"

namespace lbm {
template struct exact::StepLaunch<exact::StoreF16>;
}  // namespace lbm
