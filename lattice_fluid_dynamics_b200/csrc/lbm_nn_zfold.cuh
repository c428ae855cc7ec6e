// Forward convolution with the three z taps folded into N, for the halo
// shapes (input channels a multiple of 16, NX a multiple of 8, NY of 16)
// with NT = 16, 32 or 48 output channels (N = 3 NT <= 256).
//
//     y[z] = Q_0[z - 1] + Q_1[z] + Q_2[z + 1],
//     Q_dz[z'][v][co] = sum over (dy, dx, c) of x[z'][v + (dx, dy)][c] W[co][(dz, dy, dx, c)]
//
// One CTA walks a column of 8 x 16 tiles through a range of `seg` output
// planes (input planes z0 - 1 .. z0 + seg, the ends read twice): for each
// input plane z' it copies the plane's 10 x 18 halo (per 16-channel slice,
// two 8-channel planes, as k_conv_fwd_halo) and issues, per (dy, dx) tap,
// one MMA of M = 128 voxels, N = 3 NT (the three dz blocks of output
// channels), K = 16 channels -- 9 MMAs per plane and slice instead of 27.
// The epilogue of plane z' completes output plane z' - 1 (its third
// contribution), carries z' and starts z' + 1, in registers (thread t:
// voxel t), then applies bias / activation / store.  The sum for each output
// is ((Q_0 + Q_1) + Q_2), a fixed order.  Every wait is bounded; a give-up
// stops the CTA's copies and MMAs, drains (bounded), sets the error word and
// frees its tensor memory.
#pragma once

#include <cuda_bf16.h>

#include "lbm_nn_gemm.cuh"
#include "lbm_nn_halo.cuh"
#include "tc05.cuh"

namespace lbm {
namespace nn {

constexpr int ZF_PVOX = HX * HY;            // 180 voxels of one halo plane
constexpr int ZF_PLANE = ZF_PVOX * 16;      // one 8-channel plane: 2,880 B
constexpr int ZF_HALO = 2 * ZF_PLANE;       // one 16-channel slice
constexpr int ZF_STAGES = 3;
constexpr int ZF_SEG = 8;                   // output planes per CTA, at most

// the weights of one 16-channel slice: [tap (dy, dx)][plane][n' = dz NT + co]
template <int NT>
__host__ __device__ constexpr int zf_slice_wbytes() {
    return 9 * 2 * 3 * NT * 16;
}
// halo stages, then every slice's weights (copied once, resident)
template <int NT>
__host__ __device__ constexpr int zf_smem_bytes(int ck) {
    return ZF_STAGES * ZF_HALO + ck * zf_slice_wbytes<NT>() + 8 * (ZF_STAGES + 1) + 16;
}

template <int NT>
__global__ void __launch_bounds__(128) k_conv_fwd_zfold(const ConvFwdArgs a, int seg) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int S = ZF_STAGES, SB = ZF_HALO, N3 = 3 * NT, WSL = zf_slice_wbytes<NT>();
    const int ck = a.cin >> 4;
    uint8_t *wsm = smem + S * SB;  // resident weights of all slices
    uint64_t *bars = reinterpret_cast<uint64_t *>(wsm + ck * WSL);  // S stage barriers, 1 plane
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + S + 1);
    const int tid = threadIdx.x, warp = tid >> 5;
    constexpr uint32_t ncols = N3 <= 64 ? 64u : N3 <= 128 ? 128u : 256u;
    const uint32_t bar_acc = tc::smem_addr(&bars[S]);
    auto bar_stage = [&](int s) { return tc::smem_addr(&bars[s]); };

    // the CTA's column of tiles and range of output planes
    const int txn = a.d.nx >> 3, tyn = a.d.ny >> 4;
    int col = blockIdx.x;
    const int tx = col % txn;
    col /= txn;
    const int ty = col % tyn;
    const int b = col / tyn;
    const int z0 = blockIdx.y * seg, z1 = min(a.d.nz, z0 + seg);
    const int planes = z1 - z0 + 2;  // input planes z0 - 1 .. z1
    const int nq = z0 < z1 ? planes * ck : 0;

    // this thread's halo elements (one plane): offsets and positions
    constexpr int HE = (2 * ZF_PVOX + 127) / 128;
    uint32_t h_soff[HE];
    int h_pos[HE];
#pragma unroll
    for (int i = 0; i < HE; i++) {
        const int e = tid + 128 * i;
        const int kc = e >= ZF_PVOX, v = e - kc * ZF_PVOX;
        h_soff[i] = (uint32_t)(kc * ZF_PLANE + v * 16);
        h_pos[i] = e < 2 * ZF_PVOX ? ((v % HX) | (v / HX) << 8 | kc << 16) : -1;
    }

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
    constexpr uint32_t idesc = tc::idesc_bf16_f32(128, N3);

    // all threads: halo plane of item q (plane q / ck, slice q % ck) into stage
    // q % S; with item 0, the weights of every slice
    auto issue = [&](int q) {
        const int p = q / ck, j = q - p * ck;
        const int zi = z0 - 1 + p;
        const uint32_t st = tc::smem_addr(smem + (q % S) * SB);
        const bool zin = (unsigned)zi < (unsigned)a.d.nz;
        const __nv_bfloat16 *xs = a.x + a.x_off + j * 16;
#pragma unroll
        for (int k = 0; k < HE; k++) {
            if (h_pos[k] < 0) break;
            const int hx = h_pos[k] & 255, hy = (h_pos[k] >> 8) & 255, kc = h_pos[k] >> 16;
            const int gx = tx * 8 + hx - 1, gy = ty * 16 + hy - 1;
            const bool in = zin && (unsigned)gx < (unsigned)a.d.nx && (unsigned)gy < (unsigned)a.d.ny;
            const long long vox =
                in ? (((long long)b * a.d.nz + zi) * a.d.ny + gy) * a.d.nx + gx : 0;
            cp_async16(st + h_soff[k], xs + vox * a.x_stride + kc * 8, in ? 16u : 0u);
        }
        if (q == 0) {
            // B rows n' = dz NT + co, K = (dy, dx) tap x 16 channels
            const uint32_t w_addr = tc::smem_addr(wsm);
            for (int e = tid; e < ck * 18 * N3; e += 128) {
                const int js = e / (18 * N3), r = e - js * 18 * N3;
                const int n = r % N3, tk = r / N3;  // tk = (dy 3 + dx) 2 + plane
                const int dz = n / NT, co = n - dz * NT, t9 = tk >> 1;
                const int tap = dz * 9 + t9;
                cp_async16(w_addr + (uint32_t)(js * WSL) + (tk * N3 + n) * 16,
                           a.w + (long long)co * a.k_pad + tap * a.cin + js * 16 + (tk & 1) * 8,
                           16u);
            }
        }
    };

    float accA[NT], accB[NT];  // output planes z' and z' + 1
#pragma unroll
    for (int i = 0; i < NT; i++) accA[i] = accB[i] = 0.f;
    const int vx = tid & 7, vy = tid >> 3;

    bool ok = true;
    int last = -1;
    for (int q = 0; q < S - 1; q++) {
        if (q < nq) issue(q);
        cp_async_commit();
    }
    for (int q = 0; q < nq; q++) {
        const int s = q % S, p = q / ck, j = q - p * ck;
        cp_async_wait<S - 2>();
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (tid == 0) {
            const uint32_t hb = tc::smem_addr(smem + s * SB);
            const uint32_t wb = tc::smem_addr(wsm) + (uint32_t)(j * WSL);
            const uint64_t a0 = tc::kmajor_desc(hb, ZF_PLANE, HX * 16);
            const uint64_t b0 = tc::kmajor_desc(wb, N3 * 16, 128);
#pragma unroll
            for (int t9 = 0; t9 < 9; t9++) {
                const int dy = t9 / 3, dx = t9 % 3;
                tc::mma_bf16(tmem, a0 + (uint64_t)(dy * HX + dx), b0 + (uint64_t)(t9 * 2 * N3),
                             idesc, (j | t9) != 0);
            }
            tc::mma_commit(bar_stage(s));
            if (j == ck - 1) tc::mma_commit(bar_acc);
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
        if (j == ck - 1) {
            // Q_0, Q_1, Q_2 of input plane z' = z0 - 1 + p for voxel tid
            const bool got = tc::mbar_wait(bar_acc, p & 1, WAIT_LIMIT);
            if (!__syncthreads_and(got)) {
                ok = false;
                break;
            }
            tc::fence_after_sync();
            const int zo = z0 - 2 + p;  // the output plane this input plane completes
            const bool emit = zo >= z0;
            const long long m =
                (((long long)b * a.d.nz + zo) * a.d.ny + ty * 16 + vy) * a.d.nx + tx * 8 + vx;
            const uint32_t lane = (uint32_t)(warp * 32) << 16;
#pragma unroll
            for (int c8 = 0; c8 < NT / 8; c8++) {
                float q0[8], q1[8], q2[8];
                tc::tmem_ld8(tmem + lane + (uint32_t)(c8 * 8), q0);
                tc::tmem_ld8(tmem + lane + (uint32_t)(NT + c8 * 8), q1);
                tc::tmem_ld8(tmem + lane + (uint32_t)(2 * NT + c8 * 8), q2);
                tc::tmem_wait_ld();
                float out[8];
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    out[i] = accA[c8 * 8 + i] + q2[i];
                    accA[c8 * 8 + i] = accB[c8 * 8 + i] + q1[i];
                    accB[c8 * 8 + i] = q0[i];
                }
                if (emit) fwd_store(a, m, c8 * 8, out);
            }
            tc::fence_before_sync();
        }
    }
    bool drained = true;
    if (last >= 0) {
        bool got = tc::mbar_wait(bar_stage(last % S), (last / S) & 1, WAIT_LIMIT);
        if (!__syncthreads_and(got)) {
            ok = false;
            got = tc::mbar_wait(bar_stage(last % S), (last / S) & 1, WAIT_LIMIT);
            drained = __syncthreads_and(got) != 0;
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
