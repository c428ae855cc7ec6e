// Step-kernel instantiations for StoreF16 populations.
#include "lbm_step.cuh"

namespace lbm {
template struct StepLaunch<StoreF16>;
}  // namespace lbm
