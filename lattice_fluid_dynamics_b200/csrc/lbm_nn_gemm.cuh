// Implicit-GEMM 3x3x3 convolutions of the warm-start network on the sm_100a
// tensor cores (tcgen05.mma kind::f16, BF16 operands, FP32 accumulation in
// tensor memory).
//
// Activations are channels-last BF16: element (voxel v, channel c) of a
// tensor with channel stride S and channel offset O is at v * S + O + c, with
// v = ((b * NZ + z) * NY + y) * NX + x.  A tensor may therefore be a channel
// slice of a wider buffer (the decoder's concatenations).  Every channel
// count and offset is a multiple of 8, so 8 channels are one 16-byte load.
// Weights are BF16 [Cout_pad][K_pad] with k = tap * Cin + cin, tap =
// (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1), zero-padded.
//
// One CTA of 128 threads computes one 128-row tile of D = A * B^T:
//   forward / input-gradient: rows = output voxels, columns = output
//     channels, reduction over k (27 taps x input channels);
//   weight gradient: rows = k, columns = output channels, reduction over a
//     range of voxels (split over CTAs; partial tiles summed afterwards).
// Each 64-wide slice of the reduction is gathered by all threads into one of
// two shared-memory stages, then one thread issues four K = 16 MMAs and
// commits them to the stage's mbarrier; a stage is refilled only after its
// previous MMAs completed.  Every wait is bounded.  When a wait gives up the
// whole CTA stops: no stage is written and no MMA issued after it, the MMAs
// already committed are drained (a bounded wait on the last commit), the
// epilogue is skipped, *err gets bit 0 (bit 1 as well if the drain ran out),
// and the tensor memory is freed before the kernel returns.
#pragma once

#include <cuda_bf16.h>

#include "tc05.cuh"

namespace lbm {
namespace nn {

constexpr int KC = 64;                 // reduction slice per stage (bf16 elements)
constexpr int A_STAGE = 128 * KC * 2;  // bytes of one A stage (128 rows)
constexpr uint32_t WAIT_LIMIT = 1u << 24;

struct Dims {
    int nb, nz, ny, nx;  // batch and spatial extents
};

// byte offset of the 16-byte chunk (row r, 8-element group kc) in a stage
__device__ __forceinline__ int chunk_off(int r, int kc) { return (r >> 3) * 1024 + kc * 128 + (r & 7) * 16; }

__device__ __forceinline__ uint32_t tmem_cols(int nt) {
    return nt <= 32 ? 32u : nt <= 64 ? 64u : nt <= 128 ? 128u : 256u;
}

// Neighbour voxel of v (coordinates x, y, z, batch b) through tap, or -1.
__device__ __forceinline__ long long neighbour(const Dims &d, int b, int z, int y, int x, int tap) {
    const int zz = z + tap / 9 - 1, yy = y + (tap / 3) % 3 - 1, xx = x + tap % 3 - 1;
    if (zz < 0 || zz >= d.nz || yy < 0 || yy >= d.ny || xx < 0 || xx >= d.nx) return -1;
    return (((long long)b * d.nz + zz) * d.ny + yy) * d.nx + xx;
}

__device__ __forceinline__ void voxel_coords(const Dims &d, long long v, int &b, int &z, int &y,
                                             int &x) {
    x = (int)(v % d.nx);
    long long t = v / d.nx;
    y = (int)(t % d.ny);
    t /= d.ny;
    z = (int)(t % d.nz);
    b = (int)(t / d.nz);
}

struct ConvFwdArgs {
    const __nv_bfloat16 *x;  // input activations
    int x_stride, x_off, cin;
    const __nv_bfloat16 *w;  // [nt][k_pad]
    int k_real, k_pad;
    const float *bias;       // [nt] or null
    int act;                 // 0 linear, 1 leaky ReLU (slope 0.1)
    __nv_bfloat16 *y;        // output activations (bf16) or null
    float *y32;              // output (fp32) or null
    int y_stride, y_off, cout_store;
    int accumulate;          // fp32 output: add to the existing values
    Dims d;
    long long m;             // voxels
    int *err;
    // split reduction: CTA (x, y) sums reduction slices [y cps, (y + 1) cps)
    // into partial[y][m][nt] (FP32); k_conv_fwd_finish applies the epilogue
    float *partial;          // null: no split
    int chunks_per_split;
};

struct ConvWgradArgs {
    const __nv_bfloat16 *x;  // layer input
    int x_stride, x_off, cin;
    const __nv_bfloat16 *g;  // output gradient (pre-activation), [m][g_stride]
    int g_stride, cout;
    int k_real, k_pad;
    float *partial;          // [splits][k_pad][nt]
    Dims d;
    long long m;
    int chunks_per_split;    // reduction slices of KC voxels per CTA
    int *err;
    // >= 0: reduction rows [ones_row, ones_row + 8) read 1.0 instead of x, so
    // that partial row ones_row sums the gradient itself (the bias gradient);
    // a padding row (k_real <= ones_row < k_pad)
    int ones_row;
};

// ---------------------------------------------------------------------------
// The pipeline shared by both kernels.  LOAD(c, a_stage, b_stage) gathers
// reduction slice c; EPI(row, col0, v[8]) consumes 8 accumulator columns of
// one tile row.
template <int NT, class Load, class Epi>
__device__ __forceinline__ void gemm_tile(int nchunks, int *err, Load load, Epi epi) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *a_st[2] = {smem, smem + A_STAGE};
    uint8_t *b_st[2] = {smem + 2 * A_STAGE, smem + 2 * A_STAGE + NT * KC * 2};
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 2 * A_STAGE + 2 * NT * KC * 2);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2);
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t ncols = tmem_cols(NT);
    const uint32_t bar[2] = {tc::smem_addr(&bars[0]), tc::smem_addr(&bars[1])};

    if (warp == 0) {
        tc::tmem_alloc(tc::smem_addr(tslot), ncols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(bar[0], 1);
        tc::mbar_init(bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    constexpr uint32_t idesc = tc::idesc_bf16_f32(128, NT);
    bool ok = true;   // block-uniform: every wait so far completed
    int issued = 0;   // chunks whose MMAs were issued and committed

    for (int c = 0; c < nchunks; c++) {
        const int s = c & 1;
        if (c >= 2) {
            // stage s is refilled only once the MMAs of chunk c - 2 have read
            // it; the vote makes the decision block-uniform, so after a wait
            // that gave up no thread writes the stage and no MMA is issued
            const bool got = tc::mbar_wait(bar[s], ((c >> 1) - 1) & 1, WAIT_LIMIT);
            if (!__syncthreads_and(got)) {
                ok = false;
                break;
            }
        }
        load(c, a_st[s], b_st[s]);
        tc::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t a0 = tc::smem_addr(a_st[s]), b0 = tc::smem_addr(b_st[s]);
#pragma unroll
            for (int j = 0; j < KC / 16; j++) {
                const uint64_t ad = tc::kmajor_desc(a0 + j * 256, 128, 1024);
                const uint64_t bd = tc::kmajor_desc(b0 + j * 256, 128, 1024);
                tc::mma_bf16(tmem, ad, bd, idesc, (c | j) != 0);
            }
            tc::mma_commit(bar[s]);
        }
        issued = c + 1;
    }
    // Drain: the commit of the last issued chunk completes only when every
    // MMA issued before it has completed, so once it has arrived nothing
    // writes the accumulator or reads a stage any more.  The tensor core
    // always finishes its MMAs, so this wait depends on nothing outside the
    // CTA; it is still bounded (two limits).
    bool drained = true;
    if (issued > 0) {
        const int c = issued - 1;
        bool got = tc::mbar_wait(bar[c & 1], (c >> 1) & 1, WAIT_LIMIT);
        if (!__syncthreads_and(got)) {
            ok = false;
            got = tc::mbar_wait(bar[c & 1], (c >> 1) & 1, WAIT_LIMIT);
            drained = __syncthreads_and(got) != 0;
        }
    }
    tc::fence_after_sync();
    if (!ok && tid == 0) atomicOr(err, drained ? 1 : 3);
    if (ok) {
        // the accumulator is complete: read it back and hand it to the epilogue
        const int row = warp * 32 + (tid & 31);
#pragma unroll 1
        for (int col = 0; col < NT; col += 8) {
            float v[8];
            tc::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)col, v);
            tc::tmem_wait_ld();
            if (nchunks == 0) {
#pragma unroll
                for (int i = 0; i < 8; i++) v[i] = 0.f;
            }
            epi(row, col, v);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    // Freed in every case: a CTA that exits holding tensor memory would leave
    // later CTAs on its SM blocked in tcgen05.alloc.  If the drain itself ran
    // out (error bit 1 set beside bit 0) an MMA might still be writing those
    // columns; the launch's results are discarded through the error word.
    if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

__device__ __forceinline__ float leaky(float v) { return v > 0.f ? v : 0.1f * v; }

// Epilogue of the forward convolution for 8 accumulator columns of output
// voxel m: bias, activation, BF16 and / or FP32 store.
__device__ __forceinline__ void fwd_store(const ConvFwdArgs &a, long long m, int col,
                                          const float (&v)[8]) {
    if (m >= a.m || col >= a.cout_store) return;
    float o[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        float t = v[i] + (a.bias ? a.bias[col + i] : 0.f);
        o[i] = a.act == 1 ? leaky(t) : t;
    }
    if (a.y) {
        __align__(16) __nv_bfloat16 h[8];
#pragma unroll
        for (int i = 0; i < 8; i++) h[i] = __float2bfloat16_rn(o[i]);
        *reinterpret_cast<uint4 *>(a.y + m * a.y_stride + a.y_off + col) =
            *reinterpret_cast<const uint4 *>(h);
    }
    if (a.y32) {
        float *p = a.y32 + m * a.y_stride + a.y_off + col;
#pragma unroll
        for (int i = 0; i < 8; i++) p[i] = a.accumulate ? p[i] + o[i] : o[i];
    }
}

// Forward convolution (also the input gradient, run on the flipped,
// transposed weights with act = 0).
template <int NT>
__global__ void __launch_bounds__(128) k_conv_fwd(const ConvFwdArgs a) {
    const long long m0 = (long long)blockIdx.x * 128;
    const int tid = threadIdx.x;
    // rows owned by this thread in the A gather: r = tid / 8 + 16 i
    int rb[8], rz[8], ry[8], rx[8];
    bool rv[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const long long m = m0 + (tid >> 3) + 16 * i;
        rv[i] = m < a.m;
        voxel_coords(a.d, rv[i] ? m : 0, rb[i], rz[i], ry[i], rx[i]);
    }
    const int all_chunks = a.k_pad / KC;
    const int c0 = a.partial ? (int)blockIdx.y * a.chunks_per_split : 0;
    const int nchunks =
        a.partial ? max(0, min(all_chunks, c0 + a.chunks_per_split) - c0) : all_chunks;
    auto load = [&](int cl, uint8_t *as, uint8_t *bs) {
        const int c = c0 + cl;
        const int kc = tid & 7;
        const int k = c * KC + kc * 8;
        int tap = 0, cin = 0;
        const bool kv = k < a.k_real;
        if (kv) {
            tap = k / a.cin;
            cin = k - tap * a.cin;
        }
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int r = (tid >> 3) + 16 * i;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (kv && rv[i]) {
                const long long nb = neighbour(a.d, rb[i], rz[i], ry[i], rx[i], tap);
                if (nb >= 0)
                    val = *reinterpret_cast<const uint4 *>(a.x + nb * a.x_stride + a.x_off + cin);
            }
            *reinterpret_cast<uint4 *>(as + chunk_off(r, kc)) = val;
        }
        for (int idx = tid; idx < NT * 8; idx += 128) {
            const int n = idx >> 3, q = idx & 7;
            const uint4 val =
                *reinterpret_cast<const uint4 *>(a.w + (long long)n * a.k_pad + c * KC + q * 8);
            *reinterpret_cast<uint4 *>(bs + chunk_off(n, q)) = val;
        }
    };
    auto epi = [&](int row, int col, const float (&v)[8]) {
        if (!a.partial) {
            fwd_store(a, m0 + row, col, v);
        } else if (m0 + row < a.m) {
            float4 *p = reinterpret_cast<float4 *>(
                a.partial + ((long long)blockIdx.y * a.m + m0 + row) * NT + col);
            p[0] = make_float4(v[0], v[1], v[2], v[3]);
            p[1] = make_float4(v[4], v[5], v[6], v[7]);
        }
    };
    gemm_tile<NT>(nchunks, a.err, load, epi);
}

// Weight gradient partials: tile blockIdx.x covers k rows [128 bx, 128 bx +
// 128), blockIdx.y a range of chunks_per_split * 64 voxels.
template <int NT>
__global__ void __launch_bounds__(128) k_conv_wgrad(const ConvWgradArgs a) {
    const int k0 = blockIdx.x * 128;
    const long long vbase = (long long)blockIdx.y * a.chunks_per_split * KC;
    const int tid = threadIdx.x;
    auto load = [&](int c, uint8_t *as, uint8_t *bs) {
        const long long mb = vbase + (long long)c * KC;
        // A: rows k (groups of 8 sharing one tap), columns = 64 voxels
#pragma unroll 2
        for (int i = 0; i < 8; i++) {
            const int idx = tid + 128 * i;
            const int j = idx & 63, grp = idx >> 6;
            const int k = k0 + grp * 8;
            const long long m = mb + j;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (k < a.k_real && m < a.m) {
                const int tap = k / a.cin, cin = k - tap * a.cin;
                int b, z, y, x;
                voxel_coords(a.d, m, b, z, y, x);
                const long long nb = neighbour(a.d, b, z, y, x, tap);
                if (nb >= 0)
                    val = *reinterpret_cast<const uint4 *>(a.x + nb * a.x_stride + a.x_off + cin);
            }
            const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&val);
            uint8_t *base = as + grp * 1024 + (j >> 3) * 128 + (j & 7) * 2;
#pragma unroll
            for (int q = 0; q < 8; q++) *reinterpret_cast<__nv_bfloat16 *>(base + q * 16) = e[q];
        }
        // B: rows = output channels, columns = 64 voxels
        for (int idx = tid; idx < (NT / 8) * KC; idx += 128) {
            const int j = idx & 63, grp = idx >> 6;
            const long long m = mb + j;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (grp * 8 < a.cout && m < a.m)
                val = *reinterpret_cast<const uint4 *>(a.g + m * a.g_stride + grp * 8);
            const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&val);
            uint8_t *base = bs + grp * 1024 + (j >> 3) * 128 + (j & 7) * 2;
#pragma unroll
            for (int q = 0; q < 8; q++) *reinterpret_cast<__nv_bfloat16 *>(base + q * 16) = e[q];
        }
    };
    auto epi = [&](int row, int col, const float (&v)[8]) {
        float *p = a.partial + ((long long)blockIdx.y * a.k_pad + k0 + row) * NT + col;
#pragma unroll
        for (int i = 0; i < 8; i++) p[i] = v[i];
    };
    gemm_tile<NT>(a.chunks_per_split, a.err, load, epi);
}

template <int NT>
constexpr int gemm_smem_bytes() {
    return 2 * A_STAGE + 2 * NT * KC * 2 + 2 * 8 + 16;
}

}  // namespace nn
}  // namespace lbm
