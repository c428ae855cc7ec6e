// Weight gradient of the 3x3x3 convolution on the tensor cores, both
// operands MN-major so that every shared-memory write is a whole 16-byte
// copy (cp.async) of 8 channels of one voxel -- no transposition:
//
//     dW[co][k] = sum over voxels v of g[v][co] x[v + tap(k)][c(k)],
//     k = tap * cin + c
//
// CTA (blockIdx.x, blockIdx.y) owns the 128 reduction rows k0 = 128 bx ...
// (M: 16 groups of 8 rows, each group one tap and 8 consecutive channels)
// and the voxel range of split blockIdx.y, walked in chunks of 64 voxels
// (K).  Per chunk:
//   A: for each row group and each voxel, the 16 bytes of x at the voxel's
//      neighbour through the group's tap (zero outside the grid), stored as
//      MN-major core matrices [group][8-voxel block][voxel] x 16 bytes;
//   B: for each 8-channel group of the gradient and each voxel, 16 bytes of
//      g, stored the same way;
// one thread issues the four K = 16 MMAs (M = 128, N = NT) of the chunk and
// commits them to the stage's mbarrier.  Chunks are pipelined over S stages
// (copies of chunk c + S - 1 in flight while the tensor core works on chunk
// c).  The accumulator D[k][co] (TMEM, NT columns) is written as the FP32
// partial tile [split][k][NT] that k_wgrad_reduce sums in a fixed order.
//
// Every wait is bounded and block-uniform; when one gives up the CTA stops
// issuing copies and MMAs, drains what it committed (bounded), sets the
// error word and frees its tensor memory.
#pragma once

#include <cuda_bf16.h>

#include "lbm_nn_gemm.cuh"
#include "lbm_nn_halo.cuh"
#include "tc05.cuh"

namespace lbm {
namespace nn {

constexpr int WG_A_BYTES = 128 * KC * 2;  // 16 row groups x 8 voxel blocks x 128 B
template <int NT>
__host__ __device__ constexpr int wgmn_stages() {
#ifdef LBM_WGMN_STAGES
    return LBM_WGMN_STAGES;
#else
    return NT <= 32 ? 4 : 3;
#endif
}
template <int NT>
__host__ __device__ constexpr int wgmn_stage_bytes() {
    return WG_A_BYTES + NT * KC * 2;
}
template <int NT>
__host__ __device__ constexpr int wgmn_smem_bytes() {
    return wgmn_stages<NT>() * wgmn_stage_bytes<NT>() + 8 * (wgmn_stages<NT>() + 1) + 16;
}

// Instruction descriptor: BF16 x BF16 -> FP32, A and B MN-major.
__host__ __device__ constexpr uint32_t idesc_bf16_f32_mn(int M, int N) {
    return tc::idesc_bf16_f32(M, N) | (1u << 15) | (1u << 16);
}

// eight BF16 ones (0x3F80): the source of the bias row
__device__ __align__(16) unsigned short g_bf16_ones[8] = {0x3F80, 0x3F80, 0x3F80, 0x3F80,
                                                           0x3F80, 0x3F80, 0x3F80, 0x3F80};

template <int NT>
__global__ void __launch_bounds__(128) k_conv_wgrad_mn(const ConvWgradArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int S = wgmn_stages<NT>(), SB = wgmn_stage_bytes<NT>();
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + S * SB);  // S stage barriers, 1 final
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + S + 1);
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t ncols = tmem_cols(NT);
    const uint32_t bar_acc = tc::smem_addr(&bars[S]);
    auto bar_stage = [&](int s) { return tc::smem_addr(&bars[s]); };
    const int k0 = blockIdx.x * 128;
    const long long vbase = (long long)blockIdx.y * a.chunks_per_split * KC;
    const long long nchunk_all = (a.m + KC - 1) / KC;
    const int nq = (int)max(0ll, min((long long)a.chunks_per_split,
                                     nchunk_all - (long long)blockIdx.y * a.chunks_per_split));

    // This thread's copies: voxel j = tid & 63 of every chunk, A row groups
    // grp = (tid >> 6) + 2 i (i < 8), B channel groups n8 = (tid >> 6) + 2 i
    // (n8 < NT / 8).  Each A group's tap and channel offset, fixed for the CTA.
    const int j = tid & 63, g0 = tid >> 6;
    // per group: tap offsets, the neighbour's voxel offset (valid when the
    // neighbour is inside the grid: then it is voxel + toff) and channel
    int gdz[8], gdy[8], gdx[8], gch[8];
    long long toff[8];
    bool gval[8], gone[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int k = k0 + (g0 + 2 * i) * 8;
        gval[i] = k < a.k_real;
        gone[i] = k == a.ones_row;
        const int tap = gval[i] ? k / a.cin : 0;
        gch[i] = gval[i] ? k - tap * a.cin : 0;
        gdz[i] = tap / 9 - 1;
        gdy[i] = (tap / 3) % 3 - 1;
        gdx[i] = tap % 3 - 1;
        toff[i] = ((long long)gdz[i] * a.d.ny + gdy[i]) * a.d.nx + gdx[i];
    }
    // coordinates of voxel vbase + j, advanced by KC voxels per chunk (32-bit:
    // the launcher requires fewer than 2^31 voxels)
    int cx, cy, cz;
    {
        unsigned r = (unsigned)min(vbase + j, a.m > 0 ? a.m - 1 : 0);
        cx = (int)(r % (unsigned)a.d.nx);
        r /= (unsigned)a.d.nx;
        cy = (int)(r % (unsigned)a.d.ny);
        r /= (unsigned)a.d.ny;
        cz = (int)(r % (unsigned)a.d.nz);
    }
    int next_q = 0;  // chunk whose coordinates cx, cy, cz hold

    if (warp == 0) {
        tc::tmem_alloc(tc::smem_addr(tslot), ncols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        for (int s = 0; s <= S; s++) tc::mbar_init(tc::smem_addr(&bars[s]), 1);
        tc::mbar_init_fence();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    constexpr uint32_t idesc = idesc_bf16_f32_mn(128, NT);

    // all threads: copies of chunk q into stage q % S
    auto issue = [&](int q) {
        const uint32_t st = tc::smem_addr(smem + (q % S) * SB);
        const long long m = vbase + (long long)q * KC + j;
        const bool mv = m < a.m;
        // chunks are issued in order: step the coordinates by KC voxels per
        // chunk (x wraps into y, y into z, z into the sample)
        for (; next_q < q; next_q++) {
            cx += KC;
            while (cx >= a.d.nx) {
                cx -= a.d.nx;
                if (++cy == a.d.ny) {
                    cy = 0;
                    if (++cz == a.d.nz) cz = 0;
                }
            }
        }
        const int x = cx, y = cy, z = cz;
        // core-matrix offset of voxel j inside a row group: block j / 8, row j % 8
        const uint32_t voff = (uint32_t)((j >> 3) * 128 + (j & 7) * 16);
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const bool in = mv && gval[i] && (unsigned)(z + gdz[i]) < (unsigned)a.d.nz &&
                            (unsigned)(y + gdy[i]) < (unsigned)a.d.ny &&
                            (unsigned)(x + gdx[i]) < (unsigned)a.d.nx;
            const long long nb = in ? m + toff[i] : 0;
            if (gone[i])
                cp_async16(st + (uint32_t)((g0 + 2 * i) * 1024) + voff, g_bf16_ones,
                           mv ? 16u : 0u);
            else
                cp_async16(st + (uint32_t)((g0 + 2 * i) * 1024) + voff,
                           a.x + nb * a.x_stride + a.x_off + gch[i], in ? 16u : 0u);
        }
        const uint32_t bst = st + WG_A_BYTES;
#pragma unroll
        for (int i = 0; i < NT / 16; i++) {
            const int n8 = g0 + 2 * i;
            const bool in = mv && n8 * 8 < a.cout;
            cp_async16(bst + (uint32_t)(n8 * 1024) + voff,
                       a.g + (mv ? m : 0) * a.g_stride + (in ? n8 * 8 : 0), in ? 16u : 0u);
        }
    };

    bool ok = true;
    int last = -1;
    for (int q = 0; q < S - 1; q++) {
        if (q < nq) issue(q);
        cp_async_commit();
    }
    for (int q = 0; q < nq; q++) {
        const int s = q % S;
        cp_async_wait<S - 2>();
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (tid == 0) {
            const uint32_t ab = tc::smem_addr(smem + s * SB), bb = ab + WG_A_BYTES;
            const uint64_t ad = tc::kmajor_desc(ab, 128, 1024);
            const uint64_t bd = tc::kmajor_desc(bb, 128, 1024);
#pragma unroll
            for (int ks = 0; ks < KC / 16; ks++)  // 16 voxels = two 8-voxel blocks
                tc::mma_bf16(tmem, ad + (uint64_t)(ks * 16), bd + (uint64_t)(ks * 16), idesc,
                             (q | ks) != 0);
            tc::mma_commit(bar_stage(s));
            if (q == nq - 1) tc::mma_commit(bar_acc);
        }
        last = q;
        const int qn = q + S - 1;
        if (qn < nq) {
            if (q >= 1) {
                const bool got =
                    tc::mbar_wait(bar_stage((q - 1) % S), ((q - 1) / S) & 1, WAIT_LIMIT);
                if (!__syncthreads_and(got)) {
                    ok = false;
                    break;
                }
            }
            issue(qn);
        }
        cp_async_commit();
    }
    if (ok && nq > 0) {
        const bool got = tc::mbar_wait(bar_acc, 0, WAIT_LIMIT);
        ok = __syncthreads_and(got) != 0;
    }
    bool drained = true;
    if (!ok && last >= 0) {
        bool got = tc::mbar_wait(bar_stage(last % S), (last / S) & 1, WAIT_LIMIT);
        if (!__syncthreads_and(got)) {
            got = tc::mbar_wait(bar_stage(last % S), (last / S) & 1, WAIT_LIMIT);
            drained = __syncthreads_and(got) != 0;
        }
    }
    tc::fence_after_sync();
    // FP32 partial of this split: row k = k0 + tid, NT columns
    if (ok) {
        float *out = a.partial + ((long long)blockIdx.y * a.k_pad + k0 + tid) * NT;
#pragma unroll 1
        for (int col = 0; col < NT; col += 8) {
            float v[8];
            tc::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)col, v);
            tc::tmem_wait_ld();
            if (nq == 0) {
#pragma unroll
                for (int i = 0; i < 8; i++) v[i] = 0.f;
            }
            float4 *p = reinterpret_cast<float4 *>(out + col);
            p[0] = make_float4(v[0], v[1], v[2], v[3]);
            p[1] = make_float4(v[4], v[5], v[6], v[7]);
        }
    }
    cp_async_wait_all();
    if (!ok && tid == 0) atomicOr(a.err, drained ? 1 : 3);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}


// ---------------------------------------------------------------------------
// Forward convolution (and input gradient) for every shape: the implicit
// GEMM of the gather kernel (rows = 128 output voxels, K = 27 taps x cin in
// slices of 64, N = NT), its operands copied by cp.async straight into the
// K-major layout (row r's 16 bytes of one 8-channel group of one tap = one
// core-matrix row) and pipelined over S stages.  Thread t owns row t (its
// voxel's coordinates are computed once) and copies all 8 groups of the
// slice for it.  With a.partial set, CTA (x, y) sums only the slices of
// split y into FP32 partials (k_conv_fwd_finish adds them).
template <int NT>
__host__ __device__ constexpr int fwdas_stages() {
    return NT <= 64 ? 4 : 3;
}
template <int NT>
__host__ __device__ constexpr int fwdas_stage_bytes() {
    return A_STAGE + NT * KC * 2;
}
template <int NT>
__host__ __device__ constexpr int fwdas_smem_bytes() {
    return fwdas_stages<NT>() * fwdas_stage_bytes<NT>() + 8 * (fwdas_stages<NT>() + 1) + 16;
}

template <int NT>
__global__ void __launch_bounds__(128) k_conv_fwd_async(const ConvFwdArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int S = fwdas_stages<NT>(), SB = fwdas_stage_bytes<NT>();
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + S * SB);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + S + 1);
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t ncols = tmem_cols(NT);
    const uint32_t bar_acc = tc::smem_addr(&bars[S]);
    auto bar_stage = [&](int s) { return tc::smem_addr(&bars[s]); };
    const long long m0 = (long long)blockIdx.x * 128;
    const int all = a.k_pad / KC;
    const int c0 = a.partial ? (int)blockIdx.y * a.chunks_per_split : 0;
    const int nq = a.partial ? max(0, min(all, c0 + a.chunks_per_split) - c0) : all;

    // row tid's voxel (32-bit: the launcher requires fewer than 2^31 voxels)
    const long long mrow = m0 + tid;
    const bool rv = mrow < a.m;
    unsigned r = rv ? (unsigned)mrow : 0u;
    const int vx = (int)(r % (unsigned)a.d.nx);
    r /= (unsigned)a.d.nx;
    const int vy = (int)(r % (unsigned)a.d.ny);
    r /= (unsigned)a.d.ny;
    const int vz = (int)(r % (unsigned)a.d.nz);
    const uint32_t row_off = (uint32_t)((tid >> 3) * 1024 + (tid & 7) * 16);
    // which of the 27 neighbours of row tid's voxel are inside the grid
    unsigned nbmask = 0;
    if (rv) {
#pragma unroll
        for (int tap = 0; tap < 27; tap++) {
            const int zz = vz + tap / 9 - 1, yy = vy + (tap / 3) % 3 - 1, xx = vx + tap % 3 - 1;
            if ((unsigned)zz < (unsigned)a.d.nz && (unsigned)yy < (unsigned)a.d.ny &&
                (unsigned)xx < (unsigned)a.d.nx)
                nbmask |= 1u << tap;
        }
    }
    // k / cin as a multiply-high: exact for k * cin < 2^32 (k < 2^13 here)
    const unsigned cin_magic = 0xFFFFFFFFu / (unsigned)a.cin + 1u;

    if (warp == 0) {
        tc::tmem_alloc(tc::smem_addr(tslot), ncols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        for (int s = 0; s <= S; s++) tc::mbar_init(tc::smem_addr(&bars[s]), 1);
        tc::mbar_init_fence();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    constexpr uint32_t idesc = tc::idesc_bf16_f32(128, NT);

    auto issue = [&](int q) {
        const uint32_t st = tc::smem_addr(smem + (q % S) * SB);
        const int kb = (c0 + q) * KC;
#pragma unroll
        for (int g = 0; g < 8; g++) {
            const int k = kb + g * 8;
            const bool kv = k < a.k_real;
            const int tap = kv ? (int)__umulhi((unsigned)k, cin_magic) : 0;
            const int ch = kv ? k - tap * a.cin : 0;
            const bool in = kv && ((nbmask >> tap) & 1u);
            const long long toff =
                ((long long)(tap / 9 - 1) * a.d.ny + ((tap / 3) % 3 - 1)) * a.d.nx + (tap % 3 - 1);
            const long long nb = in ? mrow + toff : 0;
            cp_async16(st + row_off + (uint32_t)(g * 128),
                       a.x + nb * a.x_stride + a.x_off + ch, in ? 16u : 0u);
        }
        const uint32_t bst = st + A_STAGE;
#pragma unroll
        for (int i = 0; i < NT / 16; i++) {
            const int idx = tid + 128 * i, n = idx >> 3, g = idx & 7;
            cp_async16(bst + (uint32_t)((n >> 3) * 1024 + g * 128 + (n & 7) * 16),
                       a.w + (long long)n * a.k_pad + kb + g * 8, 16u);
        }
    };

    bool ok = true;
    int last = -1;
    for (int q = 0; q < S - 1; q++) {
        if (q < nq) issue(q);
        cp_async_commit();
    }
    for (int q = 0; q < nq; q++) {
        const int s = q % S;
        cp_async_wait<S - 2>();
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (tid == 0) {
            const uint32_t ab = tc::smem_addr(smem + s * SB), bb = ab + A_STAGE;
            const uint64_t ad = tc::kmajor_desc(ab, 128, 1024);
            const uint64_t bd = tc::kmajor_desc(bb, 128, 1024);
#pragma unroll
            for (int ks = 0; ks < KC / 16; ks++)
                tc::mma_bf16(tmem, ad + (uint64_t)(ks * 16), bd + (uint64_t)(ks * 16), idesc,
                             (q | ks) != 0);
            tc::mma_commit(bar_stage(s));
            if (q == nq - 1) tc::mma_commit(bar_acc);
        }
        last = q;
        const int qn = q + S - 1;
        if (qn < nq) {
            if (q >= 1) {
                const bool got =
                    tc::mbar_wait(bar_stage((q - 1) % S), ((q - 1) / S) & 1, WAIT_LIMIT);
                if (!__syncthreads_and(got)) {
                    ok = false;
                    break;
                }
            }
            issue(qn);
        }
        cp_async_commit();
    }
    if (ok && nq > 0) {
        const bool got = tc::mbar_wait(bar_acc, 0, WAIT_LIMIT);
        ok = __syncthreads_and(got) != 0;
    }
    bool drained = true;
    if (!ok && last >= 0) {
        bool got = tc::mbar_wait(bar_stage(last % S), (last / S) & 1, WAIT_LIMIT);
        if (!__syncthreads_and(got)) {
            got = tc::mbar_wait(bar_stage(last % S), (last / S) & 1, WAIT_LIMIT);
            drained = __syncthreads_and(got) != 0;
        }
    }
    tc::fence_after_sync();
    if (ok) {
#pragma unroll 1
        for (int col = 0; col < NT; col += 8) {
            float v[8];
            tc::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)col, v);
            tc::tmem_wait_ld();
            if (nq == 0) {
#pragma unroll
                for (int i = 0; i < 8; i++) v[i] = 0.f;
            }
            if (!a.partial) {
                fwd_store(a, mrow, col, v);
            } else if (rv) {
                float4 *p = reinterpret_cast<float4 *>(
                    a.partial + ((long long)blockIdx.y * a.m + mrow) * NT + col);
                p[0] = make_float4(v[0], v[1], v[2], v[3]);
                p[1] = make_float4(v[4], v[5], v[6], v[7]);
            }
        }
    }
    cp_async_wait_all();
    if (!ok && tid == 0) atomicOr(a.err, drained ? 1 : 3);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

}  // namespace nn
}  // namespace lbm
