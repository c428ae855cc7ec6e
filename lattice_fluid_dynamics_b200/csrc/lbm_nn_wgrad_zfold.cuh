// Weight gradient with the three z taps folded into N, for 16-channel input
// slices on the halo shapes (NX a multiple of 8, NY of 16, NT <= 32):
//
//     dW[co][(dz, dy, dx, c)] = sum over input planes z' and tile voxels v of
//                               x[z'][v + (dx, dy)][c] g[z' - dz + 1][v][co]
//
// For each input plane z' of a CTA's column of 8 x 16 tiles: the plane's
// 10 x 18 halo (two 8-channel planes) and the three gradient planes z' + 1,
// z', z' - 1 (MN-major [dz][8-channel group][8-voxel block][voxel] x 16 B,
// so the three stack into N = 3 NT with one group stride) are copied by
// cp.async; the A operand -- rows (dy, dx, c), the plane's im2col transposed,
// MN-major -- is built in shared memory from the halo as two row tiles:
// taps (dy, dx) 0-7 (128 rows) and tap 8 with, in slice 0, a row group of
// 1.0 (the bias gradient) and zero padding.  16 MMAs (M = 128, N = 3 NT,
// K = 16 voxels) per plane accumulate D_0, D_1 in TMEM for the CTA's whole
// range of planes; the FP32 partial [split][k][NT] is written at the end,
// k = (dz 9 + tap) cin + 16 j + c.  Each (input plane, gradient plane) pair
// with |z' - z_g| <= 1 is covered by exactly one CTA (the one owning z');
// gradient planes outside the grid read zero.
//
// Every wait is bounded and block-uniform; a give-up stops the CTA's copies
// and MMAs, drains (bounded), sets the error word and frees its tensor
// memory.
#pragma once

#include <cuda_bf16.h>

#include "lbm_nn_gemm.cuh"
#include "lbm_nn_halo.cuh"
#include "lbm_nn_zfold.cuh"
#include "tc05.cuh"

namespace lbm {
namespace nn {

constexpr int WZ_A_BYTES = 16 * 16 * 128;  // one row tile: 16 groups x 16 voxel blocks x 128 B
constexpr int WZ_THREADS = 256;
constexpr int WZ_SEG = 8;                  // input planes per CTA

template <int NT>
__host__ __device__ constexpr int wz_stage_bytes() {
    return ZF_HALO + 3 * (NT / 8) * 2048;  // halo plane + three gradient planes
}
template <int NT>
__host__ __device__ constexpr int wz_smem_bytes() {
    return 2 * wz_stage_bytes<NT>() + 2 * WZ_A_BYTES + 8 * 4 + 16;
}

template <int NT>
__global__ void __launch_bounds__(WZ_THREADS) k_conv_wgrad_zfold(const ConvWgradArgs a, int zsegs) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int SB = wz_stage_bytes<NT>(), N3 = 3 * NT, G8 = NT / 8;
    uint8_t *abuf = smem + 2 * SB;  // row tile 0, row tile 1
    uint64_t *bars = reinterpret_cast<uint64_t *>(abuf + 2 * WZ_A_BYTES);  // stage 0, 1, final
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 3);
    const int tid = threadIdx.x, warp = tid >> 5;
    constexpr uint32_t ncols = 2 * N3 <= 128 ? 128u : 256u;
    auto bar = [&](int i) { return tc::smem_addr(&bars[i]); };
    const int j = blockIdx.x;  // input-channel slice
    // the CTA's column of tiles and its input planes [z0, z1)
    const int txn = a.d.nx >> 3, tyn = a.d.ny >> 4;
    int col = (int)blockIdx.y / zsegs;
    const int zs = (int)blockIdx.y - col * zsegs;
    const int tx = col % txn;
    col /= txn;
    const int ty = col % tyn;
    const int b = col / tyn;
    const int seg = (a.d.nz + zsegs - 1) / zsegs;
    const int z0 = zs * seg, z1 = min(a.d.nz, z0 + seg);
    const int np = max(0, z1 - z0);
    const bool ones = a.ones_row >= 0 && j == 0;

    const int vt = tid & 127, half = tid >> 7;
    const int vx = vt & 7, vy = vt >> 3;
    const uint32_t a_voff = (uint32_t)((vt >> 3) * 128 + (vt & 7) * 16);
    const uint32_t h_voff = (uint32_t)((vy * HX + vx) * 16);

    // row tile 1 holds only tap 8 (groups 0, 1) and the bias row group (2):
    // the rest is zero for the whole kernel
    for (int e = tid; e < WZ_A_BYTES / 16; e += WZ_THREADS) {
        const int gi = e / 128;  // 128 16-byte slots per group
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (gi == 2 && ones) v = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);
        *reinterpret_cast<uint4 *>(abuf + WZ_A_BYTES + e * 16) = v;
    }
    tc::fence_async_smem();
    if (warp == 0) {
        tc::tmem_alloc(tc::smem_addr(tslot), ncols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        for (int i = 0; i < 3; i++) tc::mbar_init(bar(i), 1);
        tc::mbar_init_fence();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    constexpr uint32_t idesc = tc::idesc_bf16_f32(128, N3) | (1u << 15) | (1u << 16);

    // all threads: halo plane z0 + p and gradient planes z0 + p + 1, z0 + p,
    // z0 + p - 1 into stage p % 2
    auto issue = [&](int p) {
        const int zi = z0 + p;
        const uint32_t st = tc::smem_addr(smem + (p & 1) * SB);
        const __nv_bfloat16 *xs = a.x + a.x_off + j * 16;
        for (int e = tid; e < 2 * ZF_PVOX; e += WZ_THREADS) {
            const int kc = e >= ZF_PVOX, v = e - kc * ZF_PVOX;
            const int hx = v % HX, hy = v / HX;
            const int gx = tx * 8 + hx - 1, gy = ty * 16 + hy - 1;
            const bool in = (unsigned)gx < (unsigned)a.d.nx && (unsigned)gy < (unsigned)a.d.ny;
            const long long vox =
                in ? (((long long)b * a.d.nz + zi) * a.d.ny + gy) * a.d.nx + gx : 0;
            cp_async16(st + (uint32_t)(kc * ZF_PLANE + v * 16), xs + vox * a.x_stride + kc * 8,
                       in ? 16u : 0u);
        }
#pragma unroll
        for (int i = 0; i < 3 * G8 / 2; i++) {
            const int piece = half + 2 * i, dz = piece / G8, n8 = piece - dz * G8;
            const int zg = zi - dz + 1;
            const bool in = (unsigned)zg < (unsigned)a.d.nz && n8 * 8 < a.cout;
            const long long vox =
                in ? (((long long)b * a.d.nz + zg) * a.d.ny + ty * 16 + vy) * a.d.nx + tx * 8 + vx
                   : 0;
            cp_async16(st + ZF_HALO + (uint32_t)(piece * 2048) + a_voff,
                       a.g + vox * a.g_stride + (in ? n8 * 8 : 0), in ? 16u : 0u);
        }
    };

    bool ok = true;
    int last = -1;  // last plane whose MMAs were committed
    if (np > 0) issue(0);
    cp_async_commit();
    for (int p = 0; p < np; p++) {
        const int s = p & 1;
        if (p >= 1) {
            // plane p - 1's MMAs read the A buffers and stage (p + 1) % 2
            const bool got = tc::mbar_wait(bar((p - 1) & 1), ((p - 1) >> 1) & 1, WAIT_LIMIT);
            if (!__syncthreads_and(got)) {
                ok = false;
                break;
            }
        }
        if (p + 1 < np) issue(p + 1);
        cp_async_commit();
        cp_async_wait<1>();      // this thread's copies of plane p have landed
        tc::fence_async_smem();  // the gradient planes, for the tensor core
        __syncthreads();
        {
            // row tile 0: taps (dy, dx) 0-7, groups half * 8 .. + 7; row tile
            // 1: tap 8, group `half`
            const uint8_t *h = smem + s * SB + h_voff;
            uint8_t *d0 = abuf + a_voff;
#pragma unroll
            for (int gh = 0; gh < 8; gh++) {
                const int gi = half * 8 + gh, t9 = gi >> 1, kc = gi & 1;
                const int dy = t9 / 3, dx = t9 % 3;
                *reinterpret_cast<uint4 *>(d0 + gi * 2048) = *reinterpret_cast<const uint4 *>(
                    h + kc * ZF_PLANE + (dy * HX + dx) * 16);
            }
            *reinterpret_cast<uint4 *>(abuf + WZ_A_BYTES + a_voff + half * 2048) =
                *reinterpret_cast<const uint4 *>(h + half * ZF_PLANE + (2 * HX + 2) * 16);
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (tid == 0) {
            const uint64_t bd =
                tc::kmajor_desc(tc::smem_addr(smem + s * SB + ZF_HALO), 128, 2048);
#pragma unroll
            for (int rt = 0; rt < 2; rt++) {
                const uint64_t ad =
                    tc::kmajor_desc(tc::smem_addr(abuf + rt * WZ_A_BYTES), 128, 2048);
#pragma unroll
                for (int ks = 0; ks < 8; ks++)  // 16 voxels = tile rows 2 ks, 2 ks + 1
                    tc::mma_bf16(tmem + (uint32_t)(rt * N3), ad + (uint64_t)(ks * 16),
                                 bd + (uint64_t)(ks * 16), idesc, (p | ks) != 0);
            }
            tc::mma_commit(bar(s));
            if (p == np - 1) tc::mma_commit(bar(2));
        }
        last = p;
    }
    if (ok && np > 0) {
        const bool got = tc::mbar_wait(bar(2), 0, WAIT_LIMIT);
        ok = __syncthreads_and(got) != 0;
    }
    bool drained = true;
    if (!ok && last >= 0) {
        bool got = tc::mbar_wait(bar(last & 1), (last >> 1) & 1, WAIT_LIMIT);
        if (!__syncthreads_and(got)) {
            got = tc::mbar_wait(bar(last & 1), (last >> 1) & 1, WAIT_LIMIT);
            drained = __syncthreads_and(got) != 0;
        }
    }
    tc::fence_after_sync();
    if (ok) {
        // warpgroup `half` writes row tile `half`: row r = 32 (warp % 4) + lane,
        // group r / 8, channel r % 8; columns dz NT + co
        const int r = (warp & 3) * 32 + (tid & 31), gi = r >> 3, e = r & 7;
        int t9 = -1, c = 0;
        if (half == 0) {
            t9 = gi >> 1;
            c = (gi & 1) * 8 + e;
        } else if (gi < 2) {
            t9 = 8;
            c = gi * 8 + e;
        }
        const bool bias_row = half == 1 && gi == 2 && ones;
        float *out = a.partial + (long long)blockIdx.y * a.k_pad * NT;
#pragma unroll 1
        for (int dz = 0; dz < 3; dz++) {
            long long k = -1;
            if (t9 >= 0) k = (long long)(dz * 9 + t9) * a.cin + j * 16 + c;
            else if (bias_row && dz == 1) k = a.ones_row + e;
#pragma unroll
            for (int c8 = 0; c8 < NT / 8; c8++) {
                float v[8];
                tc::tmem_ld8(tmem + ((uint32_t)((warp & 3) * 32) << 16) +
                                 (uint32_t)(half * N3 + dz * NT + c8 * 8),
                             v);
                tc::tmem_wait_ld();
                if (np == 0) {
#pragma unroll
                    for (int i = 0; i < 8; i++) v[i] = 0.f;
                }
                if (k >= 0) {
                    float4 *q = reinterpret_cast<float4 *>(out + k * NT + c8 * 8);
                    q[0] = make_float4(v[0], v[1], v[2], v[3]);
                    q[1] = make_float4(v[4], v[5], v[6], v[7]);
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
