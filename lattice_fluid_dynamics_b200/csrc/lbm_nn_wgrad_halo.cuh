// Weight gradient of a 16-channel input slice on the halo tiles of
// k_conv_fwd_halo (NX a multiple of 8, NY of 16, output channels NT <= 32).
// For one slice j (blockIdx.x) and a range of 8 x 16 x 1 tiles
// (blockIdx.y), with the 27 x 16 reduction rows (tap, c) of the slice in
// four row tiles of 128 (taps 8t .. 8t + 7; taps 27-31 of the last are
// padding):
//
//     D_t[(tap, c)][co] += sum over the tile's voxels v of
//                          x[v + tap][16 j + c] g[v][co]
//
// Per tile the halo (as in the forward) and the gradient tile are copied by
// cp.async; then for each row tile the A operand -- MN-major, [row group
// (tap, 8 channels)][8-voxel block][voxel] x 16 bytes, the tile's im2col
// transposed -- is built in shared memory from the halo (256 threads: thread
// t copies 8 of voxel t % 128's 16 row groups with 16-byte shared loads and
// stores at compile-time offsets) and one thread issues its 8 MMAs (M = 128, N = NT, K = 16
// voxels) against the gradient tile (MN-major [8-channel group][8-voxel
// block][voxel]).  A is double-buffered, so the build of row tile t + 1
// overlaps the MMAs of row tile t, and each voxel's data crosses L2 once per
// slice (the halo's 4.2x) instead of once per tap.  The accumulators D_0 ..
// D_3 (4 NT TMEM columns) are written at the end as the FP32 partial
// [split][k][NT], k = tap cin + 16 j + c.  Row group (tap 27, channels 0-7)
// of slice 0 reads 1.0 when a.ones_row >= 0: rows k_real .. k_real + 7 of
// the partial are then the bias gradient.
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

constexpr int WGH_A_BYTES = 16 * 16 * 128;  // 16 row groups x 16 voxel blocks x 128 B

template <int NT>
__host__ __device__ constexpr int wgh_stage_bytes() {
    return HALO_BYTES + (NT / 8) * 2048;
}
template <int NT>
__host__ __device__ constexpr int wgh_smem_bytes() {
    return 2 * wgh_stage_bytes<NT>() + 2 * WGH_A_BYTES + 8 * 5 + 16;
}

constexpr int WGH_THREADS = 256;

template <int NT>
__global__ void __launch_bounds__(WGH_THREADS) k_conv_wgrad_halo(const ConvWgradArgs a, int tiles,
                                                                 int tiles_per_split) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int SB = wgh_stage_bytes<NT>();
    uint8_t *abuf = smem + 2 * SB;
    uint64_t *bars = reinterpret_cast<uint64_t *>(abuf + 2 * WGH_A_BYTES);  // A0 A1 G0 G1 acc
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 5);
    const int tid = threadIdx.x, warp = tid >> 5;
    constexpr uint32_t ncols = 4 * NT <= 64 ? 64u : 128u;
    auto bar = [&](int i) { return tc::smem_addr(&bars[i]); };
    const int j = blockIdx.x;  // input-channel slice
    const int t0 = blockIdx.y * tiles_per_split;
    const int nq = max(0, min(tiles, t0 + tiles_per_split) - t0);
    const bool ones = a.ones_row >= 0 && j == 0;

    // per-thread halo copy offsets (as in the forward)
    constexpr int HE = (2 * HVOX + WGH_THREADS - 1) / WGH_THREADS;
    uint32_t h_soff[HE];
    int h_pos[HE], h_rel[HE];
#pragma unroll
    for (int i = 0; i < HE; i++) {
        const int e = tid + WGH_THREADS * i;
        const int kc = e >= HVOX, v = e - kc * HVOX;
        const int hx = v % HX, hy = (v / HX) % HY, hz = v / (HX * HY);
        h_soff[i] = (uint32_t)(kc * HPLANE + v * 16);
        h_pos[i] = e < 2 * HVOX ? (hx | hy << 8 | hz << 16 | kc << 24) : -1;
        h_rel[i] = ((hz - 1) * a.d.ny + (hy - 1)) * a.d.nx + (hx - 1);
    }
    // thread t handles voxel t % 128 = (x, y) of the tile (its 16-byte slot
    // in the MN-major layouts and its place in the halo, tap (0, 0, 0)
    // corner) for half t / 128 of the row groups and gradient channels
    const int vt = tid & 127, half = tid >> 7;
    const int vx = vt & 7, vy = vt >> 3;
    const uint32_t a_voff = (uint32_t)((vt >> 3) * 128 + (vt & 7) * 16);
    const uint32_t h_voff = (uint32_t)((vy * HX + vx) * 16);

    if (warp == 0) {
        tc::tmem_alloc(tc::smem_addr(tslot), ncols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        for (int i = 0; i < 5; i++) tc::mbar_init(bar(i), 1);
        tc::mbar_init_fence();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    constexpr uint32_t idesc = tc::idesc_bf16_f32(128, NT) | (1u << 15) | (1u << 16);

    // all threads: halo and gradient tile of item q into stage q % 2
    auto issue = [&](int q) {
        const HaloTile t = halo_tile(a.d, t0 + q);
        const uint32_t st = tc::smem_addr(smem + (q & 1) * SB);
        const long long base =
            (((long long)t.b * a.d.nz + t.z) * a.d.ny + t.ty * 16) * a.d.nx + t.tx * 8;
        const __nv_bfloat16 *xs = a.x + a.x_off + j * 16;
#pragma unroll
        for (int k = 0; k < HE; k++) {
            if (h_pos[k] < 0) break;
            const int hx = h_pos[k] & 255, hy = (h_pos[k] >> 8) & 255,
                      hz = (h_pos[k] >> 16) & 255, kc = h_pos[k] >> 24;
            const int gx = t.tx * 8 + hx - 1, gy = t.ty * 16 + hy - 1, gz = t.z + hz - 1;
            const bool in = (unsigned)gx < (unsigned)a.d.nx && (unsigned)gy < (unsigned)a.d.ny &&
                            (unsigned)gz < (unsigned)a.d.nz;
            const long long vox = in ? base + h_rel[k] : 0;
            cp_async16(st + h_soff[k], xs + vox * a.x_stride + kc * 8, in ? 16u : 0u);
        }
        const long long vox = base + (long long)vy * a.d.nx + vx;
#pragma unroll
        for (int i = 0; i < NT / 16; i++) {
            const int n8 = half + 2 * i;
            cp_async16(st + HALO_BYTES + (uint32_t)(n8 * 2048) + a_voff,
                       a.g + vox * a.g_stride + n8 * 8, n8 * 8 < a.cout ? 16u : 0u);
        }
    };

    // all threads: row tile rt of the A operand from halo stage s into buffer b
    auto build = [&](int rt, int s, int b) {
        const uint8_t *h = smem + s * SB + h_voff;
        uint8_t *dst = abuf + b * WGH_A_BYTES + a_voff;
#pragma unroll
        for (int gh = 0; gh < 8; gh++) {
            const int gi = half * 8 + gh;
            const int tap = 8 * rt + (gi >> 1), kc = gi & 1;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (tap < 27) {
                const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
                v = *reinterpret_cast<const uint4 *>(h + kc * HPLANE +
                                                     ((dz * HY + dy) * HX + dx) * 16);
            } else if (tap == 27 && kc == 0 && ones) {
                v = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);
            }
            *reinterpret_cast<uint4 *>(dst + gi * 2048) = v;
        }
    };

    bool ok = true;
    uint32_t last_bar = 0, last_par = 0;  // barrier and phase of the last commit
    bool committed = false;
    if (nq > 0) issue(0);
    cp_async_commit();
    for (int q = 0; q < nq && ok; q++) {
        const int s = q & 1;
        if (q + 1 < nq) {
            if (q >= 1) {
                // stage (q + 1) % 2: its gradient tile was read by item q - 1's MMAs
                const bool got = tc::mbar_wait(bar(2 + ((q - 1) & 1)), ((q - 1) >> 1) & 1,
                                               WAIT_LIMIT);
                if (!__syncthreads_and(got)) {
                    ok = false;
                    break;
                }
            }
            issue(q + 1);
        }
        cp_async_commit();
        cp_async_wait<1>();       // this thread's copies of item q have landed
        tc::fence_async_smem();   // the gradient tile, for the tensor core
        __syncthreads();
#pragma unroll
        for (int rt = 0; rt < 4; rt++) {
            const int u = 4 * q + rt, b = rt & 1;
            if (u >= 2) {
                // buffer b was read by the MMAs of row tile u - 2
                const bool got = tc::mbar_wait(bar(b), ((u - 2) >> 1) & 1, WAIT_LIMIT);
                if (!__syncthreads_and(got)) {
                    ok = false;
                    break;
                }
            }
            build(rt, s, b);
            tc::fence_async_smem();
            tc::fence_before_sync();
            __syncthreads();
            tc::fence_after_sync();
            if (tid == 0) {
                const uint64_t ad =
                    tc::kmajor_desc(tc::smem_addr(abuf + b * WGH_A_BYTES), 128, 2048);
                const uint64_t bd =
                    tc::kmajor_desc(tc::smem_addr(smem + s * SB + HALO_BYTES), 128, 2048);
#pragma unroll
                for (int ks = 0; ks < 8; ks++)  // 16 voxels = tile rows 2 ks, 2 ks + 1
                    tc::mma_bf16(tmem + (uint32_t)(rt * NT), ad + (uint64_t)(ks * 16),
                                 bd + (uint64_t)(ks * 16), idesc, (q | ks) != 0);
                tc::mma_commit(bar(b));
                if (rt == 3) tc::mma_commit(bar(2 + s));
                if (rt == 3 && q == nq - 1) tc::mma_commit(bar(4));
            }
            committed = true;
            last_bar = b;
            last_par = (u >> 1) & 1;
        }
    }
    if (ok && nq > 0) {
        const bool got = tc::mbar_wait(bar(4), 0, WAIT_LIMIT);
        ok = __syncthreads_and(got) != 0;
    }
    bool drained = true;
    if (!ok && committed) {
        bool got = tc::mbar_wait(bar(last_bar), last_par, WAIT_LIMIT);
        if (!__syncthreads_and(got)) {
            got = tc::mbar_wait(bar(last_bar), last_par, WAIT_LIMIT);
            drained = __syncthreads_and(got) != 0;
        }
    }
    tc::fence_after_sync();
    if (ok) {
        // row r = 32 (warp % 4) + lane of row tiles 2 half, 2 half + 1:
        // group r / 8, channel r % 8
        const int r = (warp & 3) * 32 + (tid & 31), gi = r >> 3;
        float *out = a.partial + (long long)blockIdx.y * a.k_pad * NT;
#pragma unroll 1
        for (int rt = 2 * half; rt < 2 * half + 2; rt++) {
            const int tap = 8 * rt + (gi >> 1), c = (gi & 1) * 8 + (r & 7);
            const bool keep = tap < 27 || (tap == 27 && (gi & 1) == 0 && ones);
            float *row = out + (long long)(tap * a.cin + j * 16 + c) * NT;
#pragma unroll
            for (int col = 0; col < NT; col += 8) {
                float v[8];
                tc::tmem_ld8(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(rt * NT + col),
                             v);
                tc::tmem_wait_ld();
                if (nq == 0) {
#pragma unroll
                    for (int i = 0; i < 8; i++) v[i] = 0.f;
                }
                if (keep) {
                    float4 *p = reinterpret_cast<float4 *>(row + col);
                    p[0] = make_float4(v[0], v[1], v[2], v[3]);
                    p[1] = make_float4(v[4], v[5], v[6], v[7]);
                }
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
