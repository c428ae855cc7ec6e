// Kernels of the warm-start network other than the convolution GEMMs, and
// the launchers of the convolutions (forward, input gradient, weight
// gradient) exported for the network and the tests.
#include <stdio.h>
#include <string.h>

#include <map>
#include <mutex>
#include <utility>

#include "lbm_internal.h"
#include "lbm_nn.h"
#include "lbm_nn_gemm.cuh"
#include "lbm_nn_halo.cuh"
#include "lbm_nn_wgrad.cuh"
#include "lbm_nn_wgrad_halo.cuh"
#include "lbm_nn_zfold.cuh"
#include "lbm_nn_wgrad_zfold.cuh"

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

// Epilogue of a split forward convolution: the partial sums of each output
// (voxel, 8 columns) added over the splits in order, then fwd_store.
__global__ void k_conv_fwd_finish(const ConvFwdArgs a, int nt, int splits) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int groups = a.cout_store >> 3;
    if (i >= a.m * groups) return;
    const long long m = i / groups;
    const int col = (int)(i - m * groups) * 8;
    float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int p = 0; p < splits; p++) {
        const float4 *q =
            reinterpret_cast<const float4 *>(a.partial + ((long long)p * a.m + m) * nt + col);
        const float4 x = q[0], y = q[1];
        v[0] += x.x; v[1] += x.y; v[2] += x.z; v[3] += x.w;
        v[4] += y.x; v[5] += y.y; v[6] += y.z; v[7] += y.w;
    }
    fwd_store(a, m, col, v);
}

// FP32 workspace of split forward convolutions, one per stream (calls on
// one stream are ordered; calls on different streams do not share), grown
// on demand and kept.
float *split_workspace(cudaStream_t s, size_t bytes) {
    static std::mutex lock;
    static std::map<cudaStream_t, std::pair<void *, size_t>> bufs;
    std::lock_guard<std::mutex> guard(lock);
    auto &b = bufs[s];
    if (b.second < bytes) {
        if (b.first) {
            if (cudaStreamSynchronize(s) != cudaSuccess) return nullptr;
            cudaFree(b.first);
            b = {nullptr, 0};
        }
        void *p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
        b = {p, bytes};
    }
    return static_cast<float *>(b.first);
}

// Launch of the forward gather GEMM: the cp.async-pipelined kernel, or the
// original synchronous one (LBM_NNSetConvPath(1)).
template <int NT>
cudaError_t launch_fwd_gather(const ConvFwdArgs &a, dim3 grid, cudaStream_t s);

template <int NT>
cudaError_t fwd_nt(ConvFwdArgs a, int slot, cudaStream_t s) {
    cudaError_t e = set_attr<NT>(slot);
    if (e != cudaSuccess) return e;
    const unsigned blocks = (unsigned)((a.m + 127) / 128);
    const int nchunks = a.k_pad / KC;
    // Few row tiles and a long reduction: split the reduction over CTAs so
    // that about two CTAs per SM work, at least 4 slices each, and sum the
    // FP32 partials in a second kernel (not inside a stream capture).
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (blocks < 148 && nchunks >= 8 && cudaStreamIsCapturing(s, &cap) == cudaSuccess &&
        cap == cudaStreamCaptureStatusNone) {
        int splits = (int)((296 + blocks - 1) / blocks);
        if (splits > nchunks / 4) splits = nchunks / 4;
        const int cps = (nchunks + splits - 1) / splits;
        splits = (nchunks + cps - 1) / cps;
        float *ws = splits > 1 ? split_workspace(s, (size_t)splits * a.m * NT * sizeof(float))
                               : nullptr;
        if (ws) {
            a.partial = ws;
            a.chunks_per_split = cps;
            e = launch_fwd_gather<NT>(a, dim3(blocks, (unsigned)splits), s);
            if (e != cudaSuccess) return e;
            const long long outs = a.m * (a.cout_store / 8);
            k_conv_fwd_finish<<<(unsigned)((outs + 255) / 256), 256, 0, s>>>(a, NT, splits);
            return cudaGetLastError();
        }
    }
    a.partial = nullptr;
    return launch_fwd_gather<NT>(a, dim3(blocks), s);
}

// 0: the halo-tiled forward kernel where a convolution's shape allows it,
//    the cp.async-pipelined gather kernels elsewhere;
// 1: the original synchronous gather kernels for every shape;
// 2: the pipelined gather kernels for every shape;
// 3: as 0, with the z-folded forward wherever its shape allows it (not only
//    where there are enough tile columns to fill the GPU)
// (LBM_NNSetConvPath, for comparisons)
int g_conv_path = 0;

bool halo_shape_ok(const ConvFwdArgs &a, int nt) {
    return (g_conv_path == 0 || g_conv_path == 3) && a.cin % 16 == 0 && a.x_stride % 8 == 0 && a.x_off % 8 == 0 &&
           a.d.nx % 8 == 0 && a.d.ny % 16 == 0 &&
           (nt == 16 || nt == 32 || nt == 48 || nt == 64 || nt == 96) &&
           (long long)a.d.nb * a.d.nz * (a.d.ny / 16) * (a.d.nx / 8) < (1ll << 31);
}

// Output planes per CTA of the z-folded forward: ZF_SEG, fewer (down to 2)
// where that leaves fewer than ~2 CTAs per SM.
int zfold_seg(const ConvFwdArgs &a) {
    const long long cols = (long long)a.d.nb * (a.d.ny / 16) * (a.d.nx / 8);
    int seg = ZF_SEG;
    while (seg > 2 && cols * ((a.d.nz + seg - 1) / seg) < 296) seg /= 2;
    return seg;
}

// The z-folded forward where there are enough columns of tiles to keep
// every SM busy with at least 2 output planes per CTA and every input
// slice's weights fit in shared memory beside the halo stages (resident for
// the CTA's life).  Path 3 takes it wherever the kernel can run.
bool zfold_ok(const ConvFwdArgs &a, int nt) {
    const long long cols = (long long)a.d.nb * (a.d.ny / 16) * (a.d.nx / 8);
    const int seg = zfold_seg(a);
    const long long segs = (a.d.nz + seg - 1) / seg;
    const int ck = a.cin / 16;
    const int smem = nt == 16   ? zf_smem_bytes<16>(ck)
                     : nt == 32 ? zf_smem_bytes<32>(ck)
                                : zf_smem_bytes<48>(ck);
    return (nt == 16 || nt == 32 || nt == 48) && cols < (1ll << 31) && smem <= 110 * 1024 &&
           (g_conv_path == 3 || cols * segs >= 200);
}

template <int NT>
cudaError_t fwd_zfold_nt(const ConvFwdArgs &a, cudaStream_t s) {
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(k_conv_fwd_zfold<NT>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 110 * 1024);
        if (attr == cudaSuccess)
            attr = cudaFuncSetAttribute(k_conv_fwd_zfold<NT>,
                                        cudaFuncAttributePreferredSharedMemoryCarveout,
                                        cudaSharedmemCarveoutMaxShared);
    });
    if (attr != cudaSuccess) return attr;
    const unsigned cols = (unsigned)((long long)a.d.nb * (a.d.ny / 16) * (a.d.nx / 8));
    const int seg = zfold_seg(a);
    const unsigned segs = (unsigned)((a.d.nz + seg - 1) / seg);
    k_conv_fwd_zfold<NT><<<dim3(cols, segs), 128, zf_smem_bytes<NT>(a.cin / 16), s>>>(a, seg);
    return cudaGetLastError();
}

template <int NT>
cudaError_t fwd_halo_nt(ConvFwdArgs a, cudaStream_t s) {
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    static int per_sm = 0, sms = 0;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(k_conv_fwd_halo<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    halo_smem_bytes<NT>());
        if (attr == cudaSuccess)
            attr = cudaFuncSetAttribute(k_conv_fwd_halo<NT>,
                                        cudaFuncAttributePreferredSharedMemoryCarveout,
                                        cudaSharedmemCarveoutMaxShared);
        int dev = 0;
        if (attr == cudaSuccess) attr = cudaGetDevice(&dev);
        if (attr == cudaSuccess)
            attr = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        // CTAs per SM by shared memory (1 KB reserved per CTA); registers
        // and threads allow more
        int smem_sm = 0;
        if (attr == cudaSuccess)
            attr = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor,
                                          dev);
        per_sm = smem_sm / (halo_smem_bytes<NT>() + 1024);
        if (per_sm > 4) per_sm = 4;
        if (attr == cudaSuccess && per_sm < 1) attr = cudaErrorInvalidConfiguration;
    });
    if (attr != cudaSuccess) return attr;
    const long long tiles = (long long)a.d.nb * a.d.nz * (a.d.ny / 16) * (a.d.nx / 8);
    const long long cap = (long long)per_sm * sms;
    const unsigned blocks = (unsigned)(tiles < cap ? tiles : cap);
    k_conv_fwd_halo<NT><<<blocks, HALO_THREADS, halo_smem_bytes<NT>(), s>>>(a, (int)tiles);
    return cudaGetLastError();
}

template <int NT>
cudaError_t launch_fwd_gather(const ConvFwdArgs &a, dim3 grid, cudaStream_t s) {
    if (g_conv_path == 1 || a.m >= (1ll << 31)) {
        k_conv_fwd<NT><<<grid, 128, gemm_smem_bytes<NT>(), s>>>(a);
        return cudaGetLastError();
    }
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(k_conv_fwd_async<NT>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    fwdas_smem_bytes<NT>());
        if (attr == cudaSuccess)
            attr = cudaFuncSetAttribute(k_conv_fwd_async<NT>,
                                        cudaFuncAttributePreferredSharedMemoryCarveout,
                                        cudaSharedmemCarveoutMaxShared);
    });
    if (attr != cudaSuccess) return attr;
    k_conv_fwd_async<NT><<<grid, 128, fwdas_smem_bytes<NT>(), s>>>(a);
    return cudaGetLastError();
}

bool wgrad_halo_ok(const ConvWgradArgs &a, int nt) {
    return g_conv_path == 0 && (nt == 16 || nt == 32) && a.cin % 16 == 0 &&
           a.x_stride % 8 == 0 && a.x_off % 8 == 0 && a.g_stride % 8 == 0 && a.g_stride >= nt &&
           a.d.nx % 8 == 0 && a.d.ny % 16 == 0 && a.m < (1ll << 31);
}

// Runs k_conv_wgrad_zfold over columns of tiles x z ranges, at most
// `splits` CTAs per slice (the partial workspace holds that many); false
// (nothing launched) when there are more columns than that.
template <int NT>
bool wgrad_zfold_nt(const ConvWgradArgs &a, unsigned splits, unsigned *used, cudaStream_t s,
                    cudaError_t *e) {
    const long long cols = (long long)a.d.nb * (a.d.ny / 16) * (a.d.nx / 8);
    if (cols > (long long)splits || cols >= (1ll << 31)) return false;
    // about two CTAs per SM over all slices, within the workspace and nz
    const long long per_slice = cols * (a.cin / 16);
    long long zsegs = (296 + per_slice - 1) / per_slice;
    if (zsegs > (long long)splits / cols) zsegs = (long long)splits / cols;
    if (zsegs > a.d.nz) zsegs = a.d.nz;
    if (zsegs < 1) zsegs = 1;
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(k_conv_wgrad_zfold<NT>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    wz_smem_bytes<NT>());
        if (attr == cudaSuccess)
            attr = cudaFuncSetAttribute(k_conv_wgrad_zfold<NT>,
                                        cudaFuncAttributePreferredSharedMemoryCarveout,
                                        cudaSharedmemCarveoutMaxShared);
    });
    if (attr != cudaSuccess) {
        *e = attr;
        return true;
    }
    k_conv_wgrad_zfold<NT><<<dim3(a.cin / 16, (unsigned)(cols * zsegs)), WZ_THREADS,
                             wz_smem_bytes<NT>(), s>>>(a, (int)zsegs);
    *e = cudaGetLastError();
    *used = (unsigned)(cols * zsegs);
    return true;
}

// Runs k_conv_wgrad_halo with at most `splits` tile ranges (the partial
// workspace holds that many); returns the number used in *used.
template <int NT>
cudaError_t wgrad_halo_nt(const ConvWgradArgs &a, unsigned splits, unsigned *used,
                          cudaStream_t s) {
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    static int sms = 0;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(k_conv_wgrad_halo<NT>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    wgh_smem_bytes<NT>());
        if (attr == cudaSuccess)
            attr = cudaFuncSetAttribute(k_conv_wgrad_halo<NT>,
                                        cudaFuncAttributePreferredSharedMemoryCarveout,
                                        cudaSharedmemCarveoutMaxShared);
        int dev = 0;
        if (attr == cudaSuccess) attr = cudaGetDevice(&dev);
        if (attr == cudaSuccess)
            attr = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    });
    if (attr != cudaSuccess) return attr;
    const long long tiles = (long long)a.d.nb * a.d.nz * (a.d.ny / 16) * (a.d.nx / 8);
    const int slices = a.cin / 16;
    const int per_sm = NT <= 16 ? 2 : 1;  // shared memory: 108 / 117 KB per CTA
    long long sp = ((long long)per_sm * sms + slices - 1) / slices;
    if (sp > (long long)splits) sp = splits;
    if (sp > tiles) sp = tiles;
    if (sp < 1) sp = 1;
    const long long per = (tiles + sp - 1) / sp;
    sp = (tiles + per - 1) / per;
    k_conv_wgrad_halo<NT><<<dim3(slices, (unsigned)sp), WGH_THREADS, wgh_smem_bytes<NT>(), s>>>(
        a, (int)tiles, (int)per);
    *used = (unsigned)sp;
    return cudaGetLastError();
}

template <int NT>
cudaError_t wgrad_mn_nt(const ConvWgradArgs &a, unsigned splits, cudaStream_t s) {
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(k_conv_wgrad_mn<NT>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    wgmn_smem_bytes<NT>());
        if (attr == cudaSuccess)
            attr = cudaFuncSetAttribute(k_conv_wgrad_mn<NT>,
                                        cudaFuncAttributePreferredSharedMemoryCarveout,
                                        cudaSharedmemCarveoutMaxShared);
    });
    if (attr != cudaSuccess) return attr;
    k_conv_wgrad_mn<NT><<<dim3(a.k_pad / 128, splits), 128, wgmn_smem_bytes<NT>(), s>>>(a);
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


// dW[n][k] = sum over splits of partial[split][k][n], n < cout, k < k_real;
// with dbias set, row k_real of the partials (the rows of 1.0 in the
// reduction) summed the same way gives db[n].  A block of 256 threads owns
// 64 consecutive outputs o = k * cout + n (consecutive in the partials when
// cout == nt, so each warp's loads are one contiguous 128-byte line); thread
// group r (4 of them, two warps each) sums splits r, r + 4, ... and the four
// sums are added in order (deterministic).  (Measured: 4 x 64 outputs per
// block faster than 8 x 32 and 16 x 16.)
constexpr int WR_OUT = 64, WR_GROUPS = 4;
__global__ void k_wgrad_reduce(const float *__restrict__ partial, int splits, int k_pad, int nt,
                               int cout, int k_real, float *__restrict__ dw, int accumulate,
                               float *__restrict__ dbias) {
    __shared__ float part[WR_GROUPS][WR_OUT];
    const int ol = threadIdx.x % WR_OUT, r = threadIdx.x / WR_OUT;
    const long long o = (long long)blockIdx.x * WR_OUT + ol;
    const int rows = k_real + (dbias ? 1 : 0);
    const bool live = o < (long long)cout * rows;
    const int k = live ? (int)(o / cout) : 0, n = live ? (int)(o - (long long)k * cout) : 0;
    // eight independent loads in flight per thread, summed in split order
    float s = 0.f;
    if (live) {
        const float *src = partial + (long long)k * nt + n;
        const long long stride = (long long)k_pad * nt;
        int p = r;
        for (; p + 7 * WR_GROUPS < splits; p += 8 * WR_GROUPS) {
            float v[8];
#pragma unroll
            for (int u = 0; u < 8; u++) v[u] = src[(long long)(p + u * WR_GROUPS) * stride];
#pragma unroll
            for (int u = 0; u < 8; u++) s += v[u];
        }
        for (; p < splits; p += WR_GROUPS) s += src[(long long)p * stride];
    }
    part[r][ol] = s;
    __syncthreads();
    if (r == 0 && live) {
        float t = part[0][ol];
#pragma unroll
        for (int q = 1; q < WR_GROUPS; q++) t += part[q][ol];
        if (k == k_real) {
            dbias[n] = t;
        } else {
            float *d = dw + (long long)n * k_real + k;
            *d = accumulate ? *d + t : t;
        }
    }
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
    if (halo_shape_ok(a, nt)) {
        if (zfold_ok(a, nt))
            return nt == 16   ? fwd_zfold_nt<16>(a, s)
                   : nt == 32 ? fwd_zfold_nt<32>(a, s)
                              : fwd_zfold_nt<48>(a, s);
        switch (nt) {
            case 16: return fwd_halo_nt<16>(a, s);
            case 32: return fwd_halo_nt<32>(a, s);
            case 48: return fwd_halo_nt<48>(a, s);
            case 64: return fwd_halo_nt<64>(a, s);
            default: return fwd_halo_nt<96>(a, s);
        }
    }
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
                       int accumulate, cudaStream_t s, int cout_write, float *dbias,
                       bool *bias_done, unsigned max_splits) {
    if (max_splits < splits) max_splits = splits;
    ConvWgradArgs a = a0;
    a.err = err_ptr();
    if (!a.err) return cudaErrorInvalidDevicePointer;
    if (bias_done) *bias_done = false;
    const bool mn = g_conv_path != 1 && a.m < (1ll << 31);
    // the bias gradient rides on the first padding row group, if it exists
    a.ones_row = (mn && dbias && a.k_pad - a.k_real >= 8 && a.k_real % 8 == 0) ? a.k_real : -1;
    cudaError_t e;
    if (wgrad_halo_ok(a, nt)) {
        unsigned used = splits;
        const bool zf = nt == 16 ? wgrad_zfold_nt<16>(a, max_splits, &used, s, &e)
                                 : wgrad_zfold_nt<32>(a, max_splits, &used, s, &e);
        if (!zf)
            e = nt == 16 ? wgrad_halo_nt<16>(a, splits, &used, s)
                         : wgrad_halo_nt<32>(a, splits, &used, s);
        splits = used;
    } else if (mn) {
        switch (nt) {
            case 16: e = wgrad_mn_nt<16>(a, splits, s); break;
            case 32: e = wgrad_mn_nt<32>(a, splits, s); break;
            case 64: e = wgrad_mn_nt<64>(a, splits, s); break;
            case 128: e = wgrad_mn_nt<128>(a, splits, s); break;
            default: return cudaErrorInvalidValue;
        }
    } else {
        switch (nt) {
            case 16: e = wgrad_nt<16>(a, 0, splits, s); break;
            case 32: e = wgrad_nt<32>(a, 1, splits, s); break;
            case 64: e = wgrad_nt<64>(a, 3, splits, s); break;
            case 128: e = wgrad_nt<128>(a, 5, splits, s); break;
            default: return cudaErrorInvalidValue;
        }
    }
    if (e != cudaSuccess) return e;
    const int rows = cout_write > 0 ? cout_write : a.cout;
    float *db = a.ones_row >= 0 ? dbias : nullptr;  // ones_row == k_real
    const long long outs = (long long)rows * (a.k_real + (db ? 1 : 0));
    k_wgrad_reduce<<<(unsigned)((outs + WR_OUT - 1) / WR_OUT), WR_OUT * WR_GROUPS, 0, s>>>(
        a.partial, (int)splits, a.k_pad, nt, rows, a.k_real, dw, accumulate, db);
    if (db && bias_done) *bias_done = true;
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

int LBM_NNSetConvPath(int path) {
    if (path < 0 || path > 3) return LBM_ERR_INVALID_ARGUMENT;
    g_conv_path = path;
    return LBM_OK;
}

}  // extern "C"
