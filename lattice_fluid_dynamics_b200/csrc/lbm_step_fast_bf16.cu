// Fast-arithmetic build of the step kernels for StoreBF16 populations: the
// same source as the exact kernels, compiled with FMA contraction and
// hardware-approximate division and square root (see build.py).  Selected
// per grid with LBMGrid.arithmetic = LBM_ARITH_FAST.
#define LBM_FAST_ARITH 1
#include "lbm_step.cuh"

namespace lbm {
template struct fast::StepLaunch<fast::StoreBF16>;
extern const StepOps step_ops_fast_bf16 = fast::make_step_ops<fast::StoreBF16>();
}  // namespace lbm
