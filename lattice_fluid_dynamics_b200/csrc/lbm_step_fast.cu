// Fast-arithmetic build of the step kernel (FP32, FP16 and BF16 storage):
// the same source as the exact kernels, compiled with FMA contraction and
// hardware-approximate division and square root (see build.py).  Selected
// per grid with LBMGrid.arithmetic = LBM_ARITH_FAST.
#define LBM_FAST_ARITH 1
#include "lbm_step.cuh"

namespace lbm {
namespace fast {

cudaError_t launch_step_fast(const GridImpl &g, const StepArgs &a, bool fused, int op, bool smag,
                             cudaStream_t s) {
    switch (g.storage) {
        case LBM_STORAGE_FP32: return StepLaunch<StoreF32>::step(g, a, fused, op, smag, s);
        case LBM_STORAGE_FP16: return StepLaunch<StoreF16>::step(g, a, fused, op, smag, s);
        case LBM_STORAGE_BF16: return StepLaunch<StoreBF16>::step(g, a, fused, op, smag, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t tma_prepare_fast(int storage) {
    switch (storage) {
        case LBM_STORAGE_FP32: return StepLaunch<StoreF32>::tma_prepare();
        case LBM_STORAGE_FP16: return StepLaunch<StoreF16>::tma_prepare();
        case LBM_STORAGE_BF16: return StepLaunch<StoreBF16>::tma_prepare();
        default: return cudaErrorNotSupported;
    }
}

}  // namespace fast
}  // namespace lbm
