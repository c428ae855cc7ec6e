// Launchers of the warm-start network's convolution kernels (lbm_nn.cu),
// shared with the network driver.  Not part of the public ABI.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace lbm {
namespace nn {

struct ConvFwdArgs;
struct ConvWgradArgs;

// K (27 taps x cin) rounded up to a multiple of 128
int k_pad_of(int cin);
cudaError_t conv_forward(const ConvFwdArgs &a, int nt, cudaStream_t s);
// dw rows written: cout_write (> 0) or a.cout.  With dbias set, the bias
// gradient (the sum of g over voxels) is written there too when the kernel
// can fold it into the weight gradient (*bias_done = true); otherwise the
// caller computes it.
// max_splits (> splits): the partial workspace holds that many, and a kernel
// that prefers more splits may use them.
cudaError_t conv_wgrad(const ConvWgradArgs &a, int nt, unsigned splits, float *dw, int accumulate,
                       cudaStream_t s, int cout_write = 0, float *dbias = nullptr,
                       bool *bias_done = nullptr, unsigned max_splits = 0);
cudaError_t weight_transpose(const __nv_bfloat16 *w, int cout, int cin, __nv_bfloat16 *wt,
                             int wt_rows, cudaStream_t s);
// reads and clears the device error word of the GEMM kernels (synchronous)
int take_error();

}  // namespace nn
}  // namespace lbm
