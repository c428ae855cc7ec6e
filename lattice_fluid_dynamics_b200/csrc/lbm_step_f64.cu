// Step-kernel instantiations for StoreF64 populations.
#include "lbm_step.cuh"

namespace lbm {
template struct exact::StepLaunch<exact::StoreF64>;
}  // namespace lbm
