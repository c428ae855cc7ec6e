// Mass and momentum of a caller-owned population field, computed without
// allocating any memory.
//
// This is the allocation-free variant of the FP64 reduction behind
// LBM_ComputeMassMomentum (k_mass_momentum, which accumulates into scratch
// that LBM_Create allocates).  Some callers cannot call cudaMalloc: real-time
// loops that must not stall on an allocation (cudaMalloc may synchronise the
// device and its cost is unbounded), and host applications whose device
// memory is owned and budgeted by another allocator or framework, so that a
// library may not take any of it for itself.  They keep their populations in
// their own device buffer and need the mass and momentum of it.  Here the
// scratch is a file-scope __device__ array of a fixed size, so nothing is
// allocated at call time.  The call synchronises the caller's stream and
// copies the four sums to host memory before it returns.
//
// Scratch: one FP64 partial (mass, jx, jy, jz) per chunk of 65,536 cells,
// at most 4,096 chunks, plus the four totals: 4,096 * 4 * 8 + 32 bytes
// (128 KiB + 32 B), held by every GPU that loads this library until the
// process exits.  The largest field accepted is therefore 268,435,456
// cells.  Every chunk slot a call reads is written by the same call first,
// so nothing has to start at zero; but all calls share the one array, so
// calls that overlap on the GPU (different streams, or different host
// threads on one device) race and must be serialised by the caller.
#include <stdio.h>

#include <mutex>

#include "lbm_d3q19.cuh"
#include "lbm_internal.h"

namespace {

constexpr long long kChunkCells = 65536;
constexpr int kMaxChunks = 4096;
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_mass_momentum_scratch[kMaxChunks * 4 + 4];

// Block b reduces cells [b * kChunkCells, min(n, (b + 1) * kChunkCells)) of
// the SoA field f[i * n + cell] and writes its four sums to scratch[4b..].
// The summation order is fixed (thread-strided loop, shuffle tree, warp
// tree), so the result is deterministic.
__global__ void __launch_bounds__(kThreads) k_partials(const float *__restrict__ f, long long n,
                                                       double *scratch) {
    const long long start = (long long)blockIdx.x * kChunkCells;
    const long long end = start + kChunkCells < n ? start + kChunkCells : n;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long c = start + threadIdx.x; c < end; c += kThreads) {
#pragma unroll
        for (int i = 0; i < 19; i++) {
            const double v = (double)__ldg(f + (long long)i * n + c);
            acc[0] += v;
            acc[1] += (double)lbm::exact::cx(i) * v;
            acc[2] += (double)lbm::exact::cy(i) * v;
            acc[3] += (double)lbm::exact::cz(i) * v;
        }
    }
    __shared__ double part[kThreads / 32][4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0.0;
        for (int w = 0; w < kThreads / 32; w++) s += part[w][threadIdx.x];
        scratch[4 * (long long)blockIdx.x + threadIdx.x] = s;
    }
}

// One block sums the chunk partials in chunk order into the four totals.
__global__ void __launch_bounds__(32) k_totals(int nchunks, double *scratch) {
    if (threadIdx.x < 4) {
        double s = 0.0;
        for (int b = 0; b < nchunks; b++) s += scratch[4 * b + threadIdx.x];
        scratch[4 * kMaxChunks + threadIdx.x] = s;
    }
}

std::mutex g_lock;
double *g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device, looked up once
// per device (the array's name in host code is not a device address).
cudaError_t scratch_on_current_device(double **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> guard(g_lock);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_mass_momentum_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" int LBM_MassMomentumNoAlloc(const float *populations, long long numCells,
                                       double *out4, void *stream) {
    if (!populations || !out4 || numCells <= 0) return LBM_ERR_INVALID_ARGUMENT;
    if (numCells > (long long)kMaxChunks * kChunkCells) {
        fprintf(stderr,
                "LBM_MassMomentumNoAlloc: %lld cells exceed the maximum of %lld "
                "(fixed scratch of %d chunks of %lld cells)\n",
                numCells, (long long)kMaxChunks * kChunkCells, kMaxChunks, kChunkCells);
        return LBM_ERR_INVALID_ARGUMENT;
    }
    double *scratch = nullptr;
    if (scratch_on_current_device(&scratch) != cudaSuccess) return LBM_ERR_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int nchunks = (int)((numCells + kChunkCells - 1) / kChunkCells);
    // launched through cudaLaunchKernel so that the status checked is this
    // call's own, not an error left behind by earlier unrelated work
    void *pargs[] = {&populations, &numCells, &scratch};
    if (cudaLaunchKernel((const void *)k_partials, dim3(nchunks), dim3(kThreads), pargs, 0, s) !=
        cudaSuccess)
        return LBM_ERR_CUDA;
    void *targs[] = {&nchunks, &scratch};
    if (cudaLaunchKernel((const void *)k_totals, dim3(1), dim3(32), targs, 0, s) != cudaSuccess)
        return LBM_ERR_CUDA;
    if (cudaMemcpyAsync(out4, scratch + 4 * kMaxChunks, 4 * sizeof(double),
                        cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return LBM_ERR_CUDA;
    return cudaStreamSynchronize(s) == cudaSuccess ? LBM_OK : LBM_ERR_CUDA;
}
