// Step-kernel instantiations for StoreF32 populations.
#include "lbm_step.cuh"

namespace lbm {
template struct exact::StepLaunch<exact::StoreF32>;
}  // namespace lbm
