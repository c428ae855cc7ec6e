// Forward convolution (and input gradient) without an im2col gather, for
// grids whose x extent is a multiple of 8 and y extent a multiple of 16 and
// input channel counts that are multiples of 16.
//
// Output tile: 8 (x) x 16 (y) voxels of one z plane of one sample = the 128
// rows of one tcgen05 MMA, row r = x + 8 y.  Its input neighbourhood, the
// halo tile of 10 x 18 x 3 voxels, is copied once per 16-channel slice into
// shared memory as two 8-channel planes, each voxel's 8 channels in 16
// bytes, x fastest:
//
//     offset(kc, hz, hy, hx) = kc * HPLANE + ((hz * HY + hy) * HX + hx) * 16
//
// In that layout the A operand of tap (dx, dy, dz) -- the 128 output rows'
// neighbours through that tap -- is itself a K-major no-swizzle operand:
// its 8-row core matrices are 8 consecutive x of one halo row (128
// contiguous bytes), the next 8-row group is the next halo row (SBO = HX x
// 16 bytes), and the second 8 channels of the K = 16 step are the next
// plane (LBO = HPLANE).  So the 27 taps are 27 MMAs whose A descriptors
// differ only in their start address; no tap slice is ever materialised.
// Out-of-grid halo voxels are zero-filled by the copy (cp.async with a
// source size of 0), which is the convolution's zero padding.
//
// The weights of the slice (27 taps x 16 channels x NT output channels) are
// copied beside the halo as [tap][plane][n] x 16 bytes (B operand: LBO = NT
// x 16, SBO = 128).  Work items (tile, slice) are pipelined over S stages of
// shared memory: every thread copies its share of item q + S - 1 while the
// tensor core works on item q, one thread issues the 27 MMAs of an item and
// commits them to the stage's mbarrier, and after the last slice of a tile
// every thread reads its accumulator row from tensor memory for the bias /
// activation / store epilogue (256 threads: warp w reads rows 32 (w % 4) ..
// + 31, columns of half w / 4).  CTAs are persistent over tiles (tile =
// blockIdx.x + i * gridDim.x).
//
// Every wait is bounded and block-uniform; when one gives up the CTA stops
// issuing copies and MMAs, drains the MMAs it committed (bounded), sets the
// error word and frees its tensor memory, as gemm_tile does.
#pragma once

#include <cuda_bf16.h>

#include "lbm_nn_gemm.cuh"
#include "tc05.cuh"

namespace lbm {
namespace nn {

constexpr int HX = 10, HY = 18, HZ = 3;   // halo tile of an 8 x 16 x 1 output tile
constexpr int HVOX = HX * HY * HZ;        // 540 voxels
constexpr int HPLANE = HVOX * 16;         // one 8-channel plane: 8,640 bytes
constexpr int HALO_BYTES = 2 * HPLANE;    // one 16-channel slice

template <int NT>
__host__ __device__ constexpr int halo_stages() {
#ifdef LBM_HALO_STAGES16
    return NT <= 16 ? LBM_HALO_STAGES16 : 2;
#else
    return NT <= 16 ? 3 : 2;
#endif
}
template <int NT>
__host__ __device__ constexpr int halo_stage_bytes() {
    return HALO_BYTES + 27 * 2 * NT * 16;
}
template <int NT>
__host__ __device__ constexpr int halo_smem_bytes() {
    // stages, S + 1 mbarriers, the TMEM address slot
    return halo_stages<NT>() * halo_stage_bytes<NT>() + 8 * (halo_stages<NT>() + 1) + 16;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_all;" ::: "memory");
}

// Tile index -> (tile x, tile y, z, sample).
struct HaloTile {
    int tx, ty, z, b;
};
__device__ __forceinline__ HaloTile halo_tile(const Dims &d, int tile) {
    const int txn = d.nx >> 3, tyn = d.ny >> 4;
    HaloTile t;
    t.tx = tile % txn;
    tile /= txn;
    t.ty = tile % tyn;
    tile /= tyn;
    t.z = tile % d.nz;
    t.b = tile / d.nz;
    return t;
}

constexpr int HALO_THREADS = 256;

template <int NT>
__global__ void __launch_bounds__(HALO_THREADS) k_conv_fwd_halo(const ConvFwdArgs a, int tiles) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int S = halo_stages<NT>(), SB = halo_stage_bytes<NT>();
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + S * SB);  // S stage barriers, 1 tile
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + S + 1);
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t ncols = tmem_cols(NT);
    const uint32_t bar_acc = tc::smem_addr(&bars[S]);
    auto bar_stage = [&](int s) { return tc::smem_addr(&bars[s]); };

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

    const int ck = a.cin >> 4;  // 16-channel slices per tile
    const int my_tiles = (int)blockIdx.x < tiles ? (tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const int nq = my_tiles * ck;

    // This thread's halo elements e = tid + 256 i: shared-memory offset,
    // position in the halo and voxel offset from the halo's (1, 1, 1) corner
    // -- the same for every tile.
    constexpr int HE = (2 * HVOX + HALO_THREADS - 1) / HALO_THREADS;
    uint32_t h_soff[HE];
    int h_pos[HE];   // hx | hy << 8 | hz << 16 | kc << 24, or -1 past the end
    int h_rel[HE];   // voxel offset
#pragma unroll
    for (int i = 0; i < HE; i++) {
        const int e = tid + HALO_THREADS * i;
        const int kc = e >= HVOX, v = e - kc * HVOX;
        const int hx = v % HX, hy = (v / HX) % HY, hz = v / (HX * HY);
        h_soff[i] = (uint32_t)(kc * HPLANE + v * 16);
        h_pos[i] = e < 2 * HVOX ? (hx | hy << 8 | hz << 16 | kc << 24) : -1;
        h_rel[i] = ((hz - 1) * a.d.ny + (hy - 1)) * a.d.nx + (hx - 1);
    }

    // all threads: copies of work item q (tile q / ck, slice q % ck) into
    // stage q % S; with a single slice the weights are copied once (item 0,
    // stage 0) and stay there
    auto issue = [&](int q) {
        const int i = q / ck, j = q - i * ck;
        const HaloTile t = halo_tile(a.d, (int)blockIdx.x + i * (int)gridDim.x);
        const uint32_t st_addr = tc::smem_addr(smem + (q % S) * SB);
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
            cp_async16(st_addr + h_soff[k], xs + vox * a.x_stride + kc * 8, in ? 16u : 0u);
        }
        if (ck > 1 || q == 0) {
            const uint32_t w_addr = st_addr + HALO_BYTES;
            for (int e = tid; e < 54 * NT; e += HALO_THREADS) {
                const int n = e % NT, tk = e / NT;  // tk = tap * 2 + plane
                cp_async16(w_addr + (tk * NT + n) * 16,
                           a.w + (long long)n * a.k_pad + (tk >> 1) * a.cin + j * 16 + (tk & 1) * 8,
                           16u);
            }
        }
    };

    bool ok = true;
    int last = -1;       // last work item whose MMAs were issued and committed
    int tiles_done = 0;  // completed phases of the tile barrier
    for (int q = 0; q < S - 1; q++) {
        if (q < nq) issue(q);
        cp_async_commit();
    }
    for (int q = 0; q < nq; q++) {
        const int s = q % S, j = q % ck;
        cp_async_wait<S - 2>();  // this thread's copies of item q have landed
        tc::fence_async_smem();  // ... and are visible to the tensor core
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (tid == 0) {
            // descriptors of tap 0; a tap moves only the start address, which
            // is the descriptor's low field in 16-byte units (no carry: shared
            // addresses stay below 256 KB)
            const uint32_t hb = tc::smem_addr(smem + s * SB);
            const uint32_t wb = tc::smem_addr(smem + (ck > 1 ? s : 0) * SB) + HALO_BYTES;
            const uint64_t a0 = tc::kmajor_desc(hb, HPLANE, HX * 16);
            const uint64_t b0 = tc::kmajor_desc(wb, NT * 16, 128);
#pragma unroll
            for (int tap = 0; tap < 27; tap++) {
                const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
                tc::mma_bf16(tmem, a0 + (uint64_t)((dz * HY + dy) * HX + dx),
                             b0 + (uint64_t)(tap * 2 * NT), idesc, (j | tap) != 0);
            }
            tc::mma_commit(bar_stage(s));
            if (j == ck - 1) tc::mma_commit(bar_acc);
        }
        last = q;
        // refill: item q + S - 1 goes into the stage of item q - 1 once its
        // MMAs have completed
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
            // the tile's accumulator is complete: epilogue, thread t = row t
            const bool got = tc::mbar_wait(bar_acc, tiles_done & 1, WAIT_LIMIT);
            if (!__syncthreads_and(got)) {
                ok = false;
                break;
            }
            tiles_done++;
            tc::fence_after_sync();
            const HaloTile t = halo_tile(a.d, (int)blockIdx.x + (q / ck) * (int)gridDim.x);
            const int row = (warp & 3) * 32 + (tid & 31);
            const long long m =
                (((long long)t.b * a.d.nz + t.z) * a.d.ny + t.ty * 16 + (row >> 3)) * a.d.nx +
                t.tx * 8 + (row & 7);
            const int c0 = (warp >> 2) * (NT / 2);
#pragma unroll 1
            for (int col = c0; col < c0 + NT / 2; col += 8) {
                float v[8];
                tc::tmem_ld8(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)col, v);
                tc::tmem_wait_ld();
                fwd_store(a, m, col, v);
            }
        }
    }
    // Drain: the commit of the last issued item arrives only after every MMA
    // issued before it has completed (bounded, two limits).
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
