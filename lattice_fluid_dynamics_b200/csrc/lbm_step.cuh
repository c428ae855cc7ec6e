// Step kernels of the D3Q19 solver, templated on the population storage
// format.  Included by one .cu file per storage format so the template
// instantiations compile in parallel.
//
// Layout in HBM: populations are SoA planes, pop[i * n + cell] with
// cell = x + NX * (y + NY * z); one plane per direction, two full copies
// (ping-pong).  A warp covers 32 consecutive x of one row, so every load
// of a plane is a 128-byte coalesced access (shifted by one element for
// the directions with e_x != 0) and every store is aligned.
//
// The fused kernel performs the reference's stream of step n
// (lbm_stream.comp:76-129, including Bouzidi interpolated bounce-back on
// the compacted boundary-link list) followed by the collision of step n+1
// (lbm_collide.comp:313-626), reading post-collision populations and
// writing post-collision populations: 2 x 19 population transfers and a
// one-byte cell flag per lattice update.
#pragma once

#include "lbm_d3q19.cuh"
#include "lbm_internal.h"
#include "tc05.cuh"

namespace lbm {
namespace LBM_ARITH_NS {

// Row offsets of the y/z neighbours of a cell after the reference's
// wrap (periodic) or clamp rule (lbm_stream.comp:63-74).
struct Rows {
    long long y[3], z[3];  // index 0: coordinate - 1, 1: itself, 2: + 1
};
__device__ __forceinline__ Rows neighbour_rows(const StepArgs &a, int y, int z) {
    const int ny = a.ny, nz = a.nz;
    int ym = y - 1, yp = y + 1, zm = z - 1, zp = z + 1;
    if (a.periodic == 1) {
        if (ym < 0) ym += ny;
        if (yp >= ny) yp -= ny;
        if (zm < 0) zm += nz;
        if (zp >= nz) zp -= nz;
    } else {
        ym = ym < 0 ? 0 : ym;
        yp = yp > ny - 1 ? ny - 1 : yp;
        zm = zm < 0 ? 0 : zm;
        zp = zp > nz - 1 ? nz - 1 : zp;
    }
    const long long nx = a.nx, plane = (long long)a.nx * a.ny;
    Rows r;
    r.y[0] = ym * nx;
    r.y[1] = y * nx;
    r.y[2] = yp * nx;
    r.z[0] = zm * plane;
    r.z[1] = z * plane;
    r.z[2] = zp * plane;
    return r;
}

// Plain pull of one cell anywhere in the grid (lbm_stream.comp:116-127):
// source x - e_x, y/z wrapped or clamped, own value when the source x is
// outside the grid.
template <class S>
__device__ __forceinline__ void gather_pull(const StepArgs &a, const typename S::T *__restrict__ src,
                                            int x, const Rows &rw, long long cell,
                                            typename S::R (&f)[19]) {
    const long long n = a.n;
#pragma unroll
    for (int i = 0; i < 19; i++) {
        const int sx = x - cx(i);
        const long long sidx =
            (sx < 0 || sx >= a.nx) ? cell : rw.y[1 - cy(i)] + rw.z[1 - cz(i)] + sx;
        f[i] = S::load(src + (long long)i * n + sidx, i);
    }
}

// Pull of CPT consecutive cells (cell0 even when CPT == 2) whose neighbours
// are all inside the grid: every direction reads at a warp-uniform offset
// from the cell, and the directions with e_x == 0 read both cells with one
// aligned pair load.
template <class S, int CPT, bool TAB>
__device__ __forceinline__ void gather_interior(const StepArgs &a, const long long *pull,
                                                const typename S::T *__restrict__ src,
                                                long long cell0, typename S::R (&f0)[19],
                                                typename S::R (&f1)[19]) {
    const typename S::T *p = src + cell0;
    const long long n = a.n, nx = a.nx, plane = (long long)a.nx * a.ny;
#pragma unroll
    for (int i = 0; i < 19; i++) {
        const long long off =
            TAB ? pull[i] : (long long)i * n - cx(i) - cy(i) * nx - cz(i) * plane;
        if (CPT == 2 && cx(i) == 0) {
            S::load2(p + off, i, f0[i], f1[i]);
        } else {
            f0[i] = S::load(p + off, i);
            if (CPT == 2) f1[i] = S::load(p + off + 1, i);
        }
    }
}

// Bouzidi interpolated bounce-back on the links of one boundary cell
// (lbm_stream.comp:88-115): overwrites the pulled value of every direction
// i whose opposite direction has a link with q >= 0.
template <class S>
__device__ __forceinline__ void bouzidi(const StepArgs &a, const typename S::T *__restrict__ src,
                                        int x, const Rows &rw, long long cell,
                                        typename S::R (&f)[19]) {
    using R = typename S::R;
    const long long n = a.n;
    const int b = a.slot[cell];
    const uint32_t mask = a.bmask[b];
    const int first = a.bfirst[b];
#pragma unroll
    for (int i = 0; i < 19; i++) {
        const int io = opp(i);
        if (mask & (1u << io)) {
            const float q = a.lq[first + __popc(mask & ((1u << io) - 1u))];
            const R fiopp = S::load(src + (long long)io * n + cell, io);
            const R qq = R(q);
            if (q >= 0.5f) {
                const R fi = S::load(src + (long long)i * n + cell, i);
                const R inv2q = ddiv<R>(R(1), R(2) * qq);
                f[i] = inv2q * fiopp + (R(1) - inv2q) * fi;
            } else {
                const int fx = x + cx(i);
                R ff;
                if (fx >= 0 && fx < a.nx)
                    ff = S::load(src + (long long)io * n + rw.y[1 + cy(i)] + rw.z[1 + cz(i)] + fx,
                                 io);
                else
                    ff = fiopp;
                const R twoq = R(2) * qq;
                f[i] = twoq * fiopp + (R(1) - twoq) * ff;
            }
        }
    }
}

// Full pull-stream gather of one cell (plain pull + Bouzidi links).
template <class S>
__device__ __forceinline__ void gather_stream(const StepArgs &a, const typename S::T *__restrict__ src,
                                              int x, int y, int z, long long cell, uint8_t flag,
                                              typename S::R (&f)[19]) {
    const Rows rw = neighbour_rows(a, y, z);
    gather_pull<S>(a, src, x, rw, cell, f);
    if (flag & FLAG_BOUNDARY) bouzidi<S>(a, src, x, rw, cell, f);
}

// Collision of one cell after the stream: solid rule, Zou-He, guard, then
// the operator.
template <class S, int OP, bool SMAG>
__device__ __forceinline__ int collide_cell(const StepArgs &a, typename S::R (&f)[19],
                                            typename S::R (&fn)[19], int x, uint8_t flag) {
    using R = typename S::R;
    R rho, ux, uy, uz;
    const int kind = prepare_cell<R>(f, flag & FLAG_SOLID_MASK, x, a.nx, R(a.inX), R(a.inY),
                                     R(a.inZ), rho, ux, uy, uz);
    if (kind == 1) {
#pragma unroll
        for (int i = 0; i < 19; i++) fn[i] = f[opp(i)];
    } else if (kind == 2) {
#pragma unroll
        for (int i = 0; i < 19; i++) fn[i] = wgt<R>(i);  // feq(1, 0): w_i * 1 * (((1+0)+0)-0)
    } else {
        const R omega = sizeof(R) == 8 ? R(a.omega_d) : R(a.omega);
        const R smag18 = sizeof(R) == 8 ? R(a.smag18_d) : R(a.smag18);
        collide<R, OP, SMAG>(f, fn, rho, ux, uy, uz, R(a.tau), omega, smag18);
    }
    return kind;
}

// One thread's share of a step: CPT cells starting at (x0, y, z).  CPT =
// cells per thread along x (1 or 2; 2 needs an even NX).  `lane` is the
// thread's lane in its warp (for the warp-aggregated guard count).
// TAB: take the interior pull offsets and the plane offsets from a
// StepOffsets kernel parameter (`o`, ignored otherwise) instead of deriving
// them from the grid sizes.
template <class S, int OP, bool SMAG, bool FUSED, int CPT, bool TAB = false>
__device__ __forceinline__ void step_cells(const StepArgs &a, const StepOffsets *o, int x0, int y,
                                           int z) {
    using T = typename S::T;
    using R = typename S::R;
    if (x0 >= a.nx || y >= a.ny) return;
    const long long n = a.n;
    const long long cell0 =
        (long long)x0 + (long long)a.nx * ((long long)y + (long long)a.ny * z);
    const T *__restrict__ src = static_cast<const T *>(a.src);
    T *__restrict__ dst = static_cast<T *>(a.dst);

    uint8_t flag0, flag1 = 0;
    if (CPT == 2) {
        const uchar2 fl = *reinterpret_cast<const uchar2 *>(a.flags + cell0);
        flag0 = fl.x;
        flag1 = fl.y;
    } else {
        flag0 = a.flags[cell0];
    }

    R cur[19], nxt[19];
    if (FUSED) {
        const bool interior = x0 > 0 && x0 + CPT < a.nx && y > 0 && y + 1 < a.ny && z > 0 &&
                              z + 1 < a.nz;
        if (interior) {
            gather_interior<S, CPT, TAB>(a, TAB ? o->pull : nullptr, src, cell0, cur, nxt);
        } else {
            const Rows rw = neighbour_rows(a, y, z);
            gather_pull<S>(a, src, x0, rw, cell0, cur);
            if (CPT == 2) gather_pull<S>(a, src, x0 + 1, rw, cell0 + 1, nxt);
        }
        if ((flag0 | flag1) & FLAG_BOUNDARY) {
            const Rows rw = neighbour_rows(a, y, z);
            if (flag0 & FLAG_BOUNDARY) bouzidi<S>(a, src, x0, rw, cell0, cur);
            if (CPT == 2 && (flag1 & FLAG_BOUNDARY))
                bouzidi<S>(a, src, x0 + 1, rw, cell0 + 1, nxt);
        }
    } else {
#pragma unroll
        for (int i = 0; i < 19; i++) {
            cur[i] = S::load(src + (long long)i * n + cell0, i);
            if (CPT == 2) nxt[i] = S::load(src + (long long)i * n + cell0 + 1, i);
        }
    }

    // One code instance of the collision for both cells; the second cell's
    // populations rotate into `cur`, the first cell's results wait in `keep`.
    R keep[19];
    int resets = 0;
#pragma unroll 1
    for (int c = 0; c < CPT; c++) {
        R fn[19];
        const int kind = collide_cell<S, OP, SMAG>(a, cur, fn, x0 + c, c ? flag1 : flag0);
        resets += kind == 2;
        if (c == CPT - 1) {
#pragma unroll
            for (int i = 0; i < 19; i++) {
                const long long plane_i = TAB ? o->dir[i] : (long long)i * n;
                if (CPT == 2)
                    S::store2(dst + plane_i + cell0, keep[i], fn[i], i);
                else
                    S::store(dst + plane_i + cell0, fn[i], i);
            }
        } else {
#pragma unroll
            for (int i = 0; i < 19; i++) {
                keep[i] = fn[i];
                cur[i] = nxt[i];
            }
        }
    }
    const unsigned active = __activemask();
    const unsigned any = __ballot_sync(active, resets > 0);
    if (any) {
        int v = resets;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(active, v, o);
        const unsigned lane = (threadIdx.x + blockDim.x * threadIdx.y) & 31u;
        if (lane == (unsigned)(__ffs(active) - 1) && v) atomicAdd(a.guard, (unsigned long long)v);
    }
}

// The step over one grid: a 2D block tile of (bx * CPT) x by cells per z.
// Whether k_step takes its offsets from the StepOffsets table.  Measured on
// B200 at 256x128x128: +2.5 % for exact FP32 MRT + Smagorinsky (issue-bound,
// and the table frees the registers that held the derived offsets), -1 to
// -2 % for FP32 BGK / regularized / MRT, -8 to -9 % for FP16 BGK and
// regularized; so only FP32 MRT + Smagorinsky uses it.
template <class S, int OP, bool SMAG>
__host__ __device__ constexpr bool step_offset_table() {
    return sizeof(typename S::T) == 4 && OP == OP_MRT && SMAG;
}

template <class S, int OP, bool SMAG, bool FUSED, int CPT, int MINB>
__global__ void __launch_bounds__(256, MINB)
    k_step(const StepArgs a, const __grid_constant__ StepOffsets o) {
    constexpr bool TAB = step_offset_table<S, OP, SMAG>();
    step_cells<S, OP, SMAG, FUSED, CPT, TAB>(a, &o, (blockIdx.x * blockDim.x + threadIdx.x) * CPT,
                                             blockIdx.y * blockDim.y + threadIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------
// The fused step with the pull neighbourhood staged in shared memory by TMA.
//
// A 32 x 8 thread block owns a 32 x TMA_BOX_Y tile of rows and walks up to
// TMA_ZSEG z-planes.  For a plane z its 19 boxes are loaded by one thread:
// direction i's box starts at (x0 - XPAD, y0 - e_y, z - e_z, i), so the
// thread for cell (x0 + tx, y0 + ty) finds its pulled value f_i at row ty,
// column tx + XPAD - e_x of that box.  Two stages alternate; each has an
// mbarrier that completes when its 19 boxes have landed.  This trades the
// 19 dependent read-only loads per cell for bulk copies that keep more bytes
// in flight per SM, which is what limits the two-byte storage formats.
//
// Cells whose pull leaves the tile's interior rule (x, y or z on the grid
// edge) pull directly from global memory with the wrap / clamp / own-value
// rules of gather_pull; only interior cells read the staged boxes, so the
// zero fill of boxes that overhang the grid is never read.  Bouzidi links,
// collision, store and guard are those of step_cells: results are identical
// to k_step's.  A wait that gives up (it never should) sets bit 0 of the
// error word and the block finishes the remaining planes on the direct path
// after a bounded wait for its copies in flight.
constexpr uint32_t TMA_WAIT_LIMIT = 1u << 22;

template <class S, int OP, bool SMAG>
__device__ __forceinline__ int tma_cell(const StepArgs &a, const typename S::T *__restrict__ box,
                                        bool staged, int x, int y, int z, int col) {
    using T = typename S::T;
    using R = typename S::R;
    constexpr int BX = tma_box_x(sizeof(T));
    constexpr int BOX = BX * TMA_BOX_Y;
    const long long n = a.n;
    const long long cell = (long long)x + (long long)a.nx * ((long long)y + (long long)a.ny * z);
    const T *__restrict__ src = static_cast<const T *>(a.src);
    T *__restrict__ dst = static_cast<T *>(a.dst);
    const uint8_t flag = a.flags[cell];
    R f[19], fn[19];
    if (staged) {
#pragma unroll
        for (int i = 0; i < 19; i++) f[i] = S::lds(box + i * BOX + col - cx(i), i);
    } else {
        gather_pull<S>(a, src, x, neighbour_rows(a, y, z), cell, f);
    }
    if (flag & FLAG_BOUNDARY) bouzidi<S>(a, src, x, neighbour_rows(a, y, z), cell, f);
    const int kind = collide_cell<S, OP, SMAG>(a, f, fn, x, flag);
#pragma unroll
    for (int i = 0; i < 19; i++) S::store(dst + (long long)i * n + cell, fn[i], i);
    return kind == 2;
}

template <class S, int OP, bool SMAG, int MINB>
__global__ void __launch_bounds__(256, MINB)
    k_step_tma(const StepArgs a, const __grid_constant__ CUtensorMap map) {
    using T = typename S::T;
    constexpr int XPAD = tma_xpad(sizeof(T));
    constexpr int BX = tma_box_x(sizeof(T));
    constexpr uint32_t BOX_BYTES = (uint32_t)(BX * TMA_BOX_Y * sizeof(T));
    constexpr uint32_t STAGE = (uint32_t)tma_stage_bytes(sizeof(T));
    extern __shared__ unsigned char tma_raw[];
    const uint32_t raw = tc::smem_addr(tma_raw);
    const uint32_t base = (raw + 127u) & ~127u;  // barriers at base, stages from base + 128
    const T *stage_ptr = reinterpret_cast<const T *>(tma_raw + (base - raw) + 128);
    const uint32_t bar[2] = {base, base + 8};

    const int tx = threadIdx.x, ty = threadIdx.y;
    const bool leader = tx == 0 && ty == 0;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * TMA_BOX_Y;
    const int x = x0 + tx, y = y0 + ty;
    const int zb = blockIdx.z * TMA_ZSEG;
    const int ze = min(zb + TMA_ZSEG, a.nz);
    const int zs = max(zb, 1), zt = min(ze, a.nz - 1);  // staged planes [zs, zt)
    const int K = zt > zs ? zt - zs : 0;
    const bool inside = x < a.nx && y < a.ny;
    const bool interior = x > 0 && x + 1 < a.nx && y > 0 && y + 1 < a.ny;
    const int col = ty * BX + tx + XPAD;
    int resets = 0;

    auto issue = [&](int k) {
        const int z = zs + k;
        const uint32_t b = bar[k & 1];
        const uint32_t dst = base + 128 + (uint32_t)(k & 1) * STAGE;
        tc::mbar_arrive_expect_tx(b, STAGE);
#pragma unroll
        for (int i = 0; i < 19; i++)
            tc::tma_load_4d(dst + (uint32_t)i * BOX_BYTES, &map, x0 - XPAD, y0 - cy(i), z - cz(i),
                            i, b);
    };

    if (leader && K > 0) {
        tc::mbar_init(bar[0], 1);
        tc::mbar_init(bar[1], 1);
        tc::mbar_init_fence();
        issue(0);
        if (K > 1) issue(1);
    }
    __syncthreads();

    // One pass over the segment's planes; the planes on the z edges of the
    // grid (outside [zs, zt)) take the direct path.
    bool tma_ok = true;  // block-uniform
    int failed_at = K;   // first plane whose wait gave up
#pragma unroll 1
    for (int z = zb; z < ze; z++) {
        const int k = z - zs;
        const bool stage_plane = k >= 0 && k < K;
        bool staged = false;
        if (stage_plane && tma_ok) {
            const bool got = tc::mbar_wait(bar[k & 1], (uint32_t)(k >> 1) & 1u, TMA_WAIT_LIMIT);
            tma_ok = __syncthreads_and(got) != 0;
            staged = tma_ok;
            if (!tma_ok) {
                failed_at = k;
                if (leader && a.err) atomicOr(a.err, 1);
            }
        }
        if (inside)
            resets += tma_cell<S, OP, SMAG>(a, stage_ptr + (k & 1) * (STAGE / sizeof(T)),
                                            staged && interior, x, y, z, col);
        if (staged && k + 2 < K) {
            __syncthreads();  // every thread is done with stage k & 1
            if (leader) issue(k + 2);
        }
    }
    if (!tma_ok && leader) {
        // let the copies still in flight (planes failed_at and the next one)
        // land before the block exits
        for (int k = failed_at; k < K && k < failed_at + 2; k++)
            tc::mbar_wait(bar[k & 1], (uint32_t)(k >> 1) & 1u, TMA_WAIT_LIMIT);
    }

    const unsigned any = __ballot_sync(0xffffffffu, resets > 0);
    if (any) {
        int v = resets;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (tx == 0 && v) atomicAdd(a.guard, (unsigned long long)v);
    }
}

// ---------------------------------------------------------------------------
// Batched step: one launch advances up to BATCH_LAUNCH_MAX grids by one
// fused step.  Work unit: a column of up to BATCH_ZB consecutive z-planes of
// one 256-cell tile, one 256-thread block per unit; the block finds its grid
// by binary search over the unit offsets and reads that grid's StepArgs
// straight from the kernel parameter (constant bank, uniform across the
// block), then walks its z-planes.  The per-cell code is k_step's, so every
// grid's result is bit-identical to a solo step.  Each grid has its own tile
// shape (BatchEntry::lbx).
template <class S, int SET>
__global__ void __launch_bounds__(256, 4) k_step_batch(const __grid_constant__ BatchLaunchParams p) {
    const unsigned b = blockIdx.x;
    int lo = 0, hi = p.count - 1;  // largest grid index with starts <= b
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (p.starts[mid] <= b) lo = mid; else hi = mid - 1;
    }
    const BatchEntry &e = p.e[lo];
    const unsigned local = b - p.starts[lo];
    const unsigned tx = local % (unsigned)e.tiles_x;
    const unsigned rest = local / (unsigned)e.tiles_x;
    const int ty = (int)(rest % (unsigned)e.tiles_y);
    const int z0 = (int)(rest / (unsigned)e.tiles_y) * BATCH_ZB;
    const int z1 = min(z0 + BATCH_ZB, e.a.nz);
    const int bx = 1 << e.lbx;
    const int x = (int)tx * bx + (threadIdx.x & (bx - 1));
    const int y = ty * (256 >> e.lbx) + (threadIdx.x >> e.lbx);
    constexpr unsigned M = batch_set_mask(SET);
    auto cells = [&](int z) {
        switch (e.combo) {
            case 0: if constexpr ((M & 1u) != 0) step_cells<S, OP_BGK, false, true, 1>(e.a, nullptr, x, y, z); break;
            case 1: if constexpr ((M & 2u) != 0) step_cells<S, OP_BGK, true, true, 1>(e.a, nullptr, x, y, z); break;
            case 2: if constexpr ((M & 4u) != 0) step_cells<S, OP_REG, false, true, 1>(e.a, nullptr, x, y, z); break;
            case 3: if constexpr ((M & 8u) != 0) step_cells<S, OP_REG, true, true, 1>(e.a, nullptr, x, y, z); break;
            case 4: if constexpr ((M & 16u) != 0) step_cells<S, OP_MRT, false, true, 1>(e.a, nullptr, x, y, z); break;
            default: if constexpr ((M & 32u) != 0) step_cells<S, OP_MRT, true, true, 1>(e.a, nullptr, x, y, z); break;
        }
    };
    if constexpr (BATCH_ZB == 1) {
        (void)z1;
        cells(z0);
    } else {
#pragma unroll 1
        for (int z = z0; z < z1; z++) cells(z);
    }
}

// Stream only: materialise the post-stream populations f = Stream(g).
template <class S>
__global__ void __launch_bounds__(256) k_stream_only(const StepArgs a) {
    using T = typename S::T;
    using R = typename S::R;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const long long n = a.n;
    const long long cell = (long long)x + (long long)a.nx * ((long long)y + (long long)a.ny * z);
    R f[19];
    gather_stream<S>(a, static_cast<const T *>(a.src), x, y, z, cell, a.flags[cell], f);
    T *dst = static_cast<T *>(a.dst);
#pragma unroll
    for (int i = 0; i < 19; i++) S::store(dst + (long long)i * n + cell, f[i], i);
}

// Velocity/density of a step (lbm_collide.comp:322-443): the moments of the
// step's input after the solid rule, Zou-He and the guard.
template <class S>
__global__ void __launch_bounds__(256) k_velocity(const StepArgs a, int kind_in, float4 *vel,
                                                   double4 *vel64) {
    using T = typename S::T;
    using R = typename S::R;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const long long n = a.n;
    const long long cell = (long long)x + (long long)a.nx * ((long long)y + (long long)a.ny * z);
    const uint8_t flag = a.flags[cell];
    const T *src = static_cast<const T *>(a.src);
    R f[19];
    if (kind_in == IN_POST_COLLISION) {
        gather_stream<S>(a, src, x, y, z, cell, flag, f);
    } else {
#pragma unroll
        for (int i = 0; i < 19; i++) f[i] = S::load(src + (long long)i * n + cell, i);
    }
    R rho, ux, uy, uz;
    prepare_cell<R>(f, flag & FLAG_SOLID_MASK, x, a.nx, R(a.inX), R(a.inY), R(a.inZ), rho, ux,
                    uy, uz);
    vel[cell] = make_float4(float(ux), float(uy), float(uz), float(rho));
    if (vel64) vel64[cell] = make_double4(double(ux), double(uy), double(uz), double(rho));
}

// Uniform equilibrium initialisation (lbm.c:670-721) of both buffers.
template <class S>
__global__ void k_init_uniform(typename S::T *a, typename S::T *b, long long n, float ux,
                               float uy, float uz) {
    using R = typename S::R;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= n) return;
#pragma unroll
    for (int i = 0; i < 19; i++) {
        const R e = feq<R>(i, R(1), R(ux), R(uy), R(uz));
        S::store(a + (long long)i * n + cell, e, i);
        S::store(b + (long long)i * n + cell, e, i);
    }
}

template <class S>
__global__ void k_init_field(typename S::T *a, typename S::T *b, long long n,
                             const float *__restrict__ rho, const float *__restrict__ u) {
    using R = typename S::R;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= n) return;
    const R r = R(rho[cell]);
    const R ux = R(u[3 * cell]), uy = R(u[3 * cell + 1]), uz = R(u[3 * cell + 2]);
#pragma unroll
    for (int i = 0; i < 19; i++) {
        const R e = feq<R>(i, r, ux, uy, uz);
        S::store(a + (long long)i * n + cell, e, i);
        S::store(b + (long long)i * n + cell, e, i);
    }
}

// SoA storage -> AoS float/double in the reference order f[i + 19*cell]
template <class S, typename O>
__global__ void k_export_aos(const typename S::T *__restrict__ src, O *__restrict__ dst,
                             long long n) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= n) return;
#pragma unroll
    for (int i = 0; i < 19; i++) dst[19 * cell + i] = O(S::load(src + (long long)i * n + cell, i));
}

template <class S>
__global__ void k_import_aos(const float *__restrict__ src, typename S::T *__restrict__ dst,
                             long long n) {
    using R = typename S::R;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= n) return;
#pragma unroll
    for (int i = 0; i < 19; i++) S::store(dst + (long long)i * n + cell, R(src[19 * cell + i]), i);
}

// FP64 mass and momentum of explicit post-stream populations.
template <class S>
__global__ void __launch_bounds__(256) k_mass_momentum(const typename S::T *__restrict__ f,
                                                        long long n, double *out4) {
    double acc[4] = {0, 0, 0, 0};
    for (long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x; cell < n;
         cell += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int i = 0; i < 19; i++) {
            const double v = double(S::load(f + (long long)i * n + cell, i));
            acc[0] += v;
            acc[1] += double(cx(i)) * v;
            acc[2] += double(cy(i)) * v;
            acc[3] += double(cz(i)) * v;
        }
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(out4 + k, v);
    }
}

}  // namespace LBM_ARITH_NS
}  // namespace lbm

// the two-cells-per-thread paired step (uses the per-cell pieces above)
#include "lbm_step_pair.cuh"

namespace lbm {
namespace LBM_ARITH_NS {

// ---------------------------------------------------------------------
// Host-side launchers for one storage format
// ---------------------------------------------------------------------
template <class S>
struct StepLaunch {
    static dim3 grid3(const GridImpl &g, int cpt = 1) {
        const int wx = (g.nx + cpt - 1) / cpt;
        return dim3((wx + g.bx - 1) / g.bx, (g.ny + g.by - 1) / g.by, g.nz);
    }

    // whether a fused step of this grid runs k_step_tma
    static bool use_tma(const GridImpl &g, const StepArgs &a) {
        return sizeof(typename S::T) <= 4 && g.tma && g.bx == 32 && g.by == TMA_BOX_Y &&
               (a.src == g.pop[0] || a.src == g.pop[1]);
    }

    template <int OP, bool SMAG>
    static void go(const GridImpl &g, const StepArgs &a, bool fused, cudaStream_t s) {
        const dim3 blk(g.bx, g.by, 1);
        if constexpr (sizeof(typename S::T) <= 4) {
            if (fused && use_tma(g, a)) {
                const dim3 grd((g.nx + 31) / 32, (g.ny + TMA_BOX_Y - 1) / TMA_BOX_Y,
                               (g.nz + TMA_ZSEG - 1) / TMA_ZSEG);
                k_step_tma<S, OP, SMAG, 4><<<grd, dim3(32, TMA_BOX_Y, 1),
                                             tma_smem_bytes(sizeof(typename S::T)), s>>>(
                    a, g.tmap[a.src == g.pop[0] ? 0 : 1]);
                return;
            }
        }
        if constexpr (sizeof(typename S::T) <= 4) {
            if (use_pair(g)) {
                const PairTable t = pair_table(a);
                const int pbx = g.pbx, pby = PAIR_THREADS / g.pbx;
                const dim3 grd((g.nx / 2 + pbx - 1) / pbx, (g.ny + pby - 1) / pby, g.nz);
                const dim3 blk2(pbx, pby, 1);
                if (fused)
                    k_step_pair<S, OP, SMAG, true><<<grd, blk2, 0, s>>>(a, t);
                else
                    k_step_pair<S, OP, SMAG, false><<<grd, blk2, 0, s>>>(a, t);
                return;
            }
        }
        StepOffsets o;
        const long long plane = (long long)a.nx * a.ny;
        for (int i = 0; i < 19; i++) {
            o.dir[i] = (long long)i * a.n;
            o.pull[i] = o.dir[i] - cx(i) - cy(i) * (long long)a.nx - cz(i) * plane;
        }
        if (fused) {
            if (g.minb == 4)
                k_step<S, OP, SMAG, true, 1, 4><<<grid3(g, 1), blk, 0, s>>>(a, o);
            else
                k_step<S, OP, SMAG, true, 1, 1><<<grid3(g, 1), blk, 0, s>>>(a, o);
        } else {
            k_step<S, OP, SMAG, false, 1, 1><<<grid3(g, 1), blk, 0, s>>>(a, o);
        }
    }

    // whether a step of this grid runs the two-cells-per-thread paired kernel:
    // FP32 / FP16 / BF16 storage, an even NX and cell indices below 2^31
    static bool use_pair(const GridImpl &g) {
        return sizeof(typename S::T) <= 4 && g.cpt == 2 && g.nx % 2 == 0 &&
               g.n < (1ll << 31) && (g.pbx == 32 || g.pbx == 64 || g.pbx == 128);
    }

    static PairTable pair_table(const StepArgs &a) {
        using T = typename S::T;
        PairTable t;
        const T *src = static_cast<const T *>(a.src);
        T *dst = static_cast<T *>(a.dst);
        const long long plane = (long long)a.nx * a.ny;
        for (int i = 0; i < 19; i++) {
            t.own[i] = src + (long long)i * a.n;
            t.pull[i] = src + (long long)i * a.n - cx(i) - cy(i) * (long long)a.nx - cz(i) * plane;
            t.dst[i] = dst + (long long)i * a.n;
        }
        t.nz = make_float2(-0.0f, -0.0f);
        return t;
    }

    static cudaError_t step(const GridImpl &g, const StepArgs &a, bool fused, int op, bool smag,
                            cudaStream_t s) {
        switch (op * 2 + (smag ? 1 : 0)) {
            case 0: go<OP_BGK, false>(g, a, fused, s); break;
            case 1: go<OP_BGK, true>(g, a, fused, s); break;
            case 2: go<OP_REG, false>(g, a, fused, s); break;
            case 3: go<OP_REG, true>(g, a, fused, s); break;
            case 4: go<OP_MRT, false>(g, a, fused, s); break;
            default: go<OP_MRT, true>(g, a, fused, s); break;
        }
        return cudaGetLastError();
    }

    // Allow k_step_tma's dynamic shared memory for every operator.
    static cudaError_t tma_prepare() {
        if constexpr (sizeof(typename S::T) <= 4) {
            const int bytes = tma_smem_bytes(sizeof(typename S::T));
            cudaError_t e = cudaSuccess;
            auto set = [&](const void *fn) {
                if (e == cudaSuccess)
                    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             bytes);
            };
            set((const void *)k_step_tma<S, OP_BGK, false, 4>);
            set((const void *)k_step_tma<S, OP_BGK, true, 4>);
            set((const void *)k_step_tma<S, OP_REG, false, 4>);
            set((const void *)k_step_tma<S, OP_REG, true, 4>);
            set((const void *)k_step_tma<S, OP_MRT, false, 4>);
            set((const void *)k_step_tma<S, OP_MRT, true, 4>);
            return e;
        } else {
            return cudaErrorNotSupported;
        }
    }

    static cudaError_t stream_only(const GridImpl &g, const StepArgs &a, cudaStream_t s) {
        k_stream_only<S><<<grid3(g), dim3(g.bx, g.by, 1), 0, s>>>(a);
        return cudaGetLastError();
    }

    static cudaError_t velocity(const GridImpl &g, const StepArgs &a, int kind, float4 *vel,
                                double4 *vel64, cudaStream_t s) {
        k_velocity<S><<<grid3(g), dim3(g.bx, g.by, 1), 0, s>>>(a, kind, vel, vel64);
        return cudaGetLastError();
    }

    static cudaError_t init_uniform(const GridImpl &g, void *a, void *b, float ux, float uy,
                                    float uz, cudaStream_t s) {
        const unsigned blocks = (unsigned)((g.n + 255) / 256);
        k_init_uniform<S><<<blocks, 256, 0, s>>>(static_cast<typename S::T *>(a),
                                                 static_cast<typename S::T *>(b), g.n, ux, uy, uz);
        return cudaGetLastError();
    }

    static cudaError_t init_field(const GridImpl &g, void *a, void *b, const float *rho,
                                  const float *u, cudaStream_t s) {
        const unsigned blocks = (unsigned)((g.n + 255) / 256);
        k_init_field<S><<<blocks, 256, 0, s>>>(static_cast<typename S::T *>(a),
                                               static_cast<typename S::T *>(b), g.n, rho, u);
        return cudaGetLastError();
    }

    static cudaError_t export_aos(const GridImpl &g, const void *src, void *dst, bool as_double,
                                  cudaStream_t s) {
        const unsigned blocks = (unsigned)((g.n + 255) / 256);
        if (as_double)
            k_export_aos<S, double><<<blocks, 256, 0, s>>>(
                static_cast<const typename S::T *>(src), static_cast<double *>(dst), g.n);
        else
            k_export_aos<S, float><<<blocks, 256, 0, s>>>(
                static_cast<const typename S::T *>(src), static_cast<float *>(dst), g.n);
        return cudaGetLastError();
    }

    static cudaError_t import_aos(const GridImpl &g, const float *src, void *dst, cudaStream_t s) {
        const unsigned blocks = (unsigned)((g.n + 255) / 256);
        k_import_aos<S><<<blocks, 256, 0, s>>>(src, static_cast<typename S::T *>(dst), g.n);
        return cudaGetLastError();
    }

    static cudaError_t mass_momentum(const GridImpl &g, const void *f, double *out4,
                                     cudaStream_t s) {
        k_mass_momentum<S><<<148 * 8, 256, 0, s>>>(static_cast<const typename S::T *>(f), g.n,
                                                   out4);
        return cudaGetLastError();
    }

    static cudaError_t batch_pair(const BatchPairParams &p, int set, cudaStream_t s) {
        if constexpr (sizeof(typename S::T) <= 4) {
            if (p.count <= 0 || p.count > BATCH_LAUNCH_MAX || p.starts[p.count] == 0 || !p.grids)
                return cudaErrorInvalidValue;
            const unsigned tiles = p.starts[p.count];
            const dim3 blk(PAIR_THREADS);
            switch (set) {
                case BATCH_SET_BGK: k_step_batch_pair<S, BATCH_SET_BGK><<<tiles, blk, 0, s>>>(p); break;
                case BATCH_SET_BGK_SMAG: k_step_batch_pair<S, BATCH_SET_BGK_SMAG><<<tiles, blk, 0, s>>>(p); break;
                case BATCH_SET_REG: k_step_batch_pair<S, BATCH_SET_REG><<<tiles, blk, 0, s>>>(p); break;
                case BATCH_SET_REG_SMAG: k_step_batch_pair<S, BATCH_SET_REG_SMAG><<<tiles, blk, 0, s>>>(p); break;
                case BATCH_SET_MRT: k_step_batch_pair<S, BATCH_SET_MRT><<<tiles, blk, 0, s>>>(p); break;
                case BATCH_SET_MRT_SMAG: k_step_batch_pair<S, BATCH_SET_MRT_SMAG><<<tiles, blk, 0, s>>>(p); break;
                // a launch group holds one operator (lbm_batch.cu, make_groups)
                default: return cudaErrorInvalidValue;
            }
            return cudaGetLastError();
        } else {
            (void)p;
            (void)set;
            (void)s;
            return cudaErrorNotSupported;
        }
    }

    static cudaError_t batch(const BatchLaunchParams &p, int set, cudaStream_t s) {
        const unsigned tiles = p.starts[p.count];
        if (p.count <= 0 || p.count > BATCH_LAUNCH_MAX || tiles == 0) return cudaErrorInvalidValue;
        switch (set) {
            case BATCH_SET_BGK: k_step_batch<S, BATCH_SET_BGK><<<tiles, 256, 0, s>>>(p); break;
            case BATCH_SET_BGK_SMAG: k_step_batch<S, BATCH_SET_BGK_SMAG><<<tiles, 256, 0, s>>>(p); break;
            case BATCH_SET_REG: k_step_batch<S, BATCH_SET_REG><<<tiles, 256, 0, s>>>(p); break;
            case BATCH_SET_REG_SMAG: k_step_batch<S, BATCH_SET_REG_SMAG><<<tiles, 256, 0, s>>>(p); break;
            case BATCH_SET_MRT: k_step_batch<S, BATCH_SET_MRT><<<tiles, 256, 0, s>>>(p); break;
            case BATCH_SET_MRT_SMAG: k_step_batch<S, BATCH_SET_MRT_SMAG><<<tiles, 256, 0, s>>>(p); break;
            // a launch group holds one operator (lbm_batch.cu, make_groups)
            default: return cudaErrorInvalidValue;
        }
        return cudaGetLastError();
    }
};

// The launcher table of one storage format (exported by its translation unit).
template <class S>
StepOps make_step_ops() {
    using L = StepLaunch<S>;
    StepOps o;
    o.step = &L::step;
    o.batch = &L::batch;
    o.batch_pair = &L::batch_pair;
    o.tma_prepare = &L::tma_prepare;
    o.stream_only = &L::stream_only;
    o.velocity = &L::velocity;
    o.init_uniform = &L::init_uniform;
    o.init_field = &L::init_field;
    o.export_aos = &L::export_aos;
    o.import_aos = &L::import_aos;
    o.mass_momentum = &L::mass_momentum;
    return o;
}

}  // namespace LBM_ARITH_NS
}  // namespace lbm
