// Kernels of the warm-start network other than the convolution GEMMs, and
// the launchers of the convolutions (forward, input gradient, weight
// gradient) exported for the network and the tests.
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "lbm_internal.h"
#include "lbm_nn.h"
#include "lbm_nn_gemm.cuh"

namespace lbm {
namespace nn {

static __device__ int g_nn_error;  // set by a GEMM whose bounded wait gave up

int k_pad_of(int cin) { return ((27 * cin + 127) / 128) * 128; }

namespace {

std::mutex g_attr_lock;
bool g_attr_done[8] = {false};

template <int NT>
cudaError_t set_attr(int slot) {
    std::lock_guard<std::mutex> guard(g_attr_lock);
    if (g_attr_done[slot]) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_conv_fwd<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         gemm_smem_bytes<NT>());
    if constexpr (NT == 16 || NT == 32 || NT == 64 || NT == 128) {
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_conv_wgrad<NT>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     gemm_smem_bytes<NT>());
    }
    if (e == cudaSuccess) g_attr_done[slot] = true;
    return e;
}

int *err_ptr() {
    static int *p = nullptr;
    static std::mutex lock;
    std::lock_guard<std::mutex> guard(lock);
    if (!p) {
        void *q = nullptr;
        if (cudaGetSymbolAddress(&q, g_nn_error) != cudaSuccess) return nullptr;
        p = static_cast<int *>(q);
    }
    return p;
}

template <int NT>
cudaError_t fwd_nt(ConvFwdArgs a, int slot, cudaStream_t s) {
    cudaError_t e = set_attr<NT>(slot);
    if (e != cudaSuccess) return e;
    const unsigned blocks = (unsigned)((a.m + 127) / 128);
    k_conv_fwd<NT><<<blocks, 128, gemm_smem_bytes<NT>(), s>>>(a);
    return cudaGetLastError();
}

template <int NT>
cudaError_t wgrad_nt(ConvWgradArgs a, int slot, unsigned splits, cudaStream_t s) {
    static_assert(NT == 16 || NT == 32 || NT == 64 || NT == 128, "weight-gradient tile");
    cudaError_t e = set_attr<NT>(slot);
    if (e != cudaSuccess) return e;
    k_conv_wgrad<NT><<<dim3(a.k_pad / 128, splits), 128, gemm_smem_bytes<NT>(), s>>>(a);
    return cudaGetLastError();
}

// dW[n][k] = sum over splits of partial[split][k][n], n < cout, k < k_real
__global__ void k_wgrad_reduce(const float *__restrict__ partial, int splits, int k_pad, int nt,
                               int cout, int k_real, float *__restrict__ dw, int accumulate) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cout * k_real) return;
    const int n = i / k_real, k = i - n * k_real;
    float s = 0.f;
    for (int p = 0; p < splits; p++) s += partial[((long long)p * k_pad + k) * nt + n];
    dw[i] = accumulate ? dw[i] + s : s;
}

// Wt[ci][(26 - tap) * cout + co] = W[co][tap * cin + ci]  (flip and transpose)
__global__ void k_weight_transpose(const __nv_bfloat16 *__restrict__ w, int w_kpad, int cout,
                                   int cin, __nv_bfloat16 *__restrict__ wt, int wt_rows,
                                   int wt_kpad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= wt_rows * wt_kpad) return;
    const int ci = i / wt_kpad, k = i - ci * wt_kpad;
    __nv_bfloat16 v = __float2bfloat16_rn(0.f);
    if (ci < cin && k < 27 * cout) {
        const int tp = k / cout, co = k - tp * cout;
        v = w[(long long)co * w_kpad + (26 - tp) * cin + ci];
    }
    wt[i] = v;
}

}  // namespace

cudaError_t conv_forward(const ConvFwdArgs &a0, int nt, cudaStream_t s) {
    ConvFwdArgs a = a0;
    a.err = err_ptr();
    if (!a.err) return cudaErrorInvalidDevicePointer;
    switch (nt) {
        case 16: return fwd_nt<16>(a, 0, s);
        case 32: return fwd_nt<32>(a, 1, s);
        case 48: return fwd_nt<48>(a, 2, s);
        case 64: return fwd_nt<64>(a, 3, s);
        case 96: return fwd_nt<96>(a, 4, s);
        case 128: return fwd_nt<128>(a, 5, s);
        case 192: return fwd_nt<192>(a, 6, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t conv_wgrad(const ConvWgradArgs &a0, int nt, unsigned splits, float *dw,
                       int accumulate, cudaStream_t s, int cout_write) {
    ConvWgradArgs a = a0;
    a.err = err_ptr();
    if (!a.err) return cudaErrorInvalidDevicePointer;
    cudaError_t e;
    switch (nt) {
        case 16: e = wgrad_nt<16>(a, 0, splits, s); break;
        case 32: e = wgrad_nt<32>(a, 1, splits, s); break;
        case 64: e = wgrad_nt<64>(a, 3, splits, s); break;
        case 128: e = wgrad_nt<128>(a, 5, splits, s); break;
        default: return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
    const int rows = cout_write > 0 ? cout_write : a.cout;
    const int total = rows * a.k_real;
    k_wgrad_reduce<<<(total + 255) / 256, 256, 0, s>>>(a.partial, (int)splits, a.k_pad, nt,
                                                       rows, a.k_real, dw, accumulate);
    return cudaGetLastError();
}

cudaError_t weight_transpose(const __nv_bfloat16 *w, int cout, int cin, __nv_bfloat16 *wt,
                             int wt_rows, cudaStream_t s) {
    const int wt_kpad = k_pad_of(cout);
    const int total = wt_rows * wt_kpad;
    k_weight_transpose<<<(total + 255) / 256, 256, 0, s>>>(w, k_pad_of(cin), cout, cin, wt,
                                                           wt_rows, wt_kpad);
    return cudaGetLastError();
}

int take_error() {
    int *p = err_ptr();
    if (!p) return 1;
    int v = 0;
    if (cudaMemcpy(&v, p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
    if (v) {
        const int zero = 0;
        cudaMemcpy(p, &zero, sizeof(int), cudaMemcpyHostToDevice);
    }
    return v;
}

}  // namespace nn
}  // namespace lbm

using namespace lbm;
using namespace lbm::nn;

static int to_code(cudaError_t e) { return e == cudaSuccess ? LBM_OK : LBM_ERR_CUDA; }

extern "C" {

int LBM_NNKPad(int cin) { return cin > 0 ? k_pad_of(cin) : 0; }

int LBM_NNConvForward(const void *x, int xStride, int xOff, int cin, const void *w,
                      const float *bias, int coutPad, int act, void *y, float *y32, int yStride,
                      int yOff, int coutStore, int accumulate, int nb, int nz, int ny, int nx,
                      void *stream) {
    if (!x || !w || (!y && !y32) || cin <= 0 || cin % 8 || xStride % 8 || xOff % 8 ||
        coutStore % 8 || coutStore > coutPad || yStride % 8 || yOff % 8 || nb <= 0 || nz <= 0 ||
        ny <= 0 || nx <= 0)
        return LBM_ERR_INVALID_ARGUMENT;
    ConvFwdArgs a{};
    a.x = static_cast<const __nv_bfloat16 *>(x);
    a.x_stride = xStride;
    a.x_off = xOff;
    a.cin = cin;
    a.w = static_cast<const __nv_bfloat16 *>(w);
    a.k_real = 27 * cin;
    a.k_pad = k_pad_of(cin);
    a.bias = bias;
    a.act = act;
    a.y = static_cast<__nv_bfloat16 *>(y);
    a.y32 = y32;
    a.y_stride = yStride;
    a.y_off = yOff;
    a.cout_store = coutStore;
    a.accumulate = accumulate;
    a.d = Dims{nb, nz, ny, nx};
    a.m = (long long)nb * nz * ny * nx;
    return to_code(conv_forward(a, coutPad, static_cast<cudaStream_t>(stream)));
}

int LBM_NNWeightTranspose(const void *w, int cout, int cin, void *wt, int wtRows, void *stream) {
    if (!w || !wt || cout <= 0 || cin <= 0 || wtRows < cin) return LBM_ERR_INVALID_ARGUMENT;
    return to_code(weight_transpose(static_cast<const __nv_bfloat16 *>(w), cout, cin,
                                    static_cast<__nv_bfloat16 *>(wt), wtRows,
                                    static_cast<cudaStream_t>(stream)));
}

long long LBM_NNWgradWorkspaceBytes(int cin, int coutPad, int nb, int nz, int ny, int nx,
                                    int chunksPerSplit) {
    const long long m = (long long)nb * nz * ny * nx;
    const long long per = (long long)chunksPerSplit * KC;
    const long long splits = (m + per - 1) / per;
    return splits * k_pad_of(cin) * coutPad * (long long)sizeof(float);
}

int LBM_NNConvWeightGrad(const void *x, int xStride, int xOff, int cin, const void *g,
                         int gStride, int cout, int coutPad, float *dw, int accumulate,
                         float *workspace, long long workspaceBytes, int chunksPerSplit, int nb,
                         int nz, int ny, int nx, void *stream) {
    if (!x || !g || !dw || !workspace || cin <= 0 || cin % 8 || cout % 8 || cout > coutPad ||
        chunksPerSplit <= 0 || xStride % 8 || xOff % 8 || gStride % 8)
        return LBM_ERR_INVALID_ARGUMENT;
    if (workspaceBytes <
        LBM_NNWgradWorkspaceBytes(cin, coutPad, nb, nz, ny, nx, chunksPerSplit))
        return LBM_ERR_INVALID_ARGUMENT;
    ConvWgradArgs a{};
    a.x = static_cast<const __nv_bfloat16 *>(x);
    a.x_stride = xStride;
    a.x_off = xOff;
    a.cin = cin;
    a.g = static_cast<const __nv_bfloat16 *>(g);
    a.g_stride = gStride;
    a.cout = cout;
    a.k_real = 27 * cin;
    a.k_pad = k_pad_of(cin);
    a.partial = workspace;
    a.d = Dims{nb, nz, ny, nx};
    a.m = (long long)nb * nz * ny * nx;
    a.chunks_per_split = chunksPerSplit;
    const long long per = (long long)chunksPerSplit * KC;
    const unsigned splits = (unsigned)((a.m + per - 1) / per);
    return to_code(conv_wgrad(a, coutPad, splits, dw, accumulate,
                              static_cast<cudaStream_t>(stream)));
}

int LBM_NNTakeError(void) { return take_error() ? LBM_ERR_TIMEOUT : LBM_OK; }

}  // extern "C"
