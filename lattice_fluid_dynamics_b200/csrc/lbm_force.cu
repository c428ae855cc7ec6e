// Momentum-exchange drag with pressure/friction split, evaluated on the
// compacted boundary-link list.
//
// Reference: simulation/shaders/lbm_force.comp:94-151 (Mei-Luo-Shyy
// F += e_i (f*_i + f_opp(i)), pressure part from feq_i + feq_opp(i), each
// cell's sums rounded to int(round(F * 1e4)) and atomically added) and
// simulation/src/lbm.c:835-918.  The reference dispatches over the whole
// grid although only cells owning a link contribute.  Here one warp
// handles one boundary cell: lane i evaluates direction i (its pulled
// population for the cell's velocity, and its link's momentum exchange),
// so a cell's ~20 dependent loads run side by side instead of one link
// after another.  The cell's sums are then formed by every lane in the
// reference's index order (i = 1..18) from shuffled per-link terms, and
// rounded per cell (round half to even), so the integer totals match the
// oracle exactly.  An FP64 sum of the unrounded per-cell forces is
// produced alongside.  Each block writes its partial sums; the last block
// to finish adds all partials in a fixed order and writes the totals, so
// the FP64 sums do not depend on scheduling either.
#include "lbm_step.cuh"

namespace lbm {

using namespace exact;

namespace {

constexpr int FORCE_CELLS_PER_BLOCK = 8;  // one warp each
constexpr int FORCE_THREADS = 32 * FORCE_CELLS_PER_BLOCK;

struct ForceArgs {
    StepArgs st;              // g (src), links, flags, periodic of g's stream
    const int32_t *bcell;     // boundary cells
    const void *fexp;         // explicit post-stream f, or null
    const float4 *vel;        // valid velocity field, or null
    const double4 *vel64;     // its FP64 copy (FP64 grids), or null
    StepArgs vin;             // input of the last step when vel is null
    int vin_kind;
    long long *i64;           // totals: 7 integer sums
    double *f64;              // totals: 6 FP64 sums
    long long *part;          // per block: 7 integer sums, 6 FP64 sums (bits) in 16 slots
    unsigned *ticket;         // blocks finished (0 between launches)
};

template <typename R> __device__ __forceinline__ long long round_ll(R v);
template <> __device__ __forceinline__ long long round_ll<float>(float v) {
    return (long long)__float2int_rn(v);
}
template <> __device__ __forceinline__ long long round_ll<double>(double v) {
    return (long long)__double2int_rn(v);
}

// r[k] without indexing a local array by a runtime k (k in 0..2)
__device__ __forceinline__ long long row_sel(const long long (&r)[3], int k) {
    return k == 0 ? r[0] : (k == 1 ? r[1] : r[2]);
}

// Direction i of the plain pull at the cell (the per-direction body of
// gather_pull: source x - e_x, y/z wrapped or clamped, own value when the
// source x is outside the grid).
template <class S>
__device__ __forceinline__ typename S::R pull_dir(const StepArgs &a,
                                                  const typename S::T *__restrict__ src, int x,
                                                  const Rows &rw, long long cell, int i) {
    const int sx = x - cx(i);
    const long long sidx = (sx < 0 || sx >= a.nx)
                               ? cell
                               : row_sel(rw.y, 1 - cy(i)) + row_sel(rw.z, 1 - cz(i)) + sx;
    return S::load(src + (long long)i * a.n + sidx, i);
}

// Direction i of Bouzidi's bounce-back at a boundary cell (the per-direction
// body of bouzidi): replaces the pulled f_i when the opposite direction has
// a link.
template <class S>
__device__ __forceinline__ typename S::R bouzidi_dir(const StepArgs &a,
                                                     const typename S::T *__restrict__ src, int x,
                                                     const Rows &rw, long long cell, int i,
                                                     uint32_t mask, int first, typename S::R f) {
    using R = typename S::R;
    const long long n = a.n;
    const int io = opp(i);
    if (!(mask & (1u << io))) return f;
    const float q = a.lq[first + __popc(mask & ((1u << io) - 1u))];
    const R fiopp = S::load(src + (long long)io * n + cell, io);
    const R qq = R(q);
    if (q >= 0.5f) {
        const R fi = S::load(src + (long long)i * n + cell, i);
        const R inv2q = ddiv<R>(R(1), R(2) * qq);
        return inv2q * fiopp + (R(1) - inv2q) * fi;
    }
    const int fx = x + cx(i);
    R ff;
    if (fx >= 0 && fx < a.nx)
        ff = S::load(src + (long long)io * n + row_sel(rw.y, 1 + cy(i)) + row_sel(rw.z, 1 + cz(i)) +
                         fx,
                     io);
    else
        ff = fiopp;
    const R twoq = R(2) * qq;
    return twoq * fiopp + (R(1) - twoq) * ff;
}

template <class S>
__global__ void __launch_bounds__(FORCE_THREADS, 6) k_force(const ForceArgs a, int nb) {
    using T = typename S::T;
    using R = typename S::R;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int b = blockIdx.x * FORCE_CELLS_PER_BLOCK + w;  // warp-uniform
    R lx = R(0), ly = R(0), lz = R(0), px = R(0), py = R(0), pz = R(0);
    int has = 0;
    if (b < nb) {
        const StepArgs &st = a.st;
        const long long n = st.n;
        const long long cell = a.bcell[b];
        const uint8_t flag = st.flags[cell];
        if ((flag & FLAG_SOLID_MASK) == 0) {
            const int nx = st.nx, ny = st.ny;
            const int c32 = (int)cell;  // cells < 2^31 (LBM_CreateEx)
            const int x = c32 % nx;
            const int r = c32 / nx;
            const int y = r % ny;
            const int z = r / ny;
            const int bi = st.slot[cell];
            const uint32_t mask = st.bmask[bi];
            const int first = st.bfirst[bi];
            // velocity and density of the last collide
            R rho, ux, uy, uz;
            if (a.vel64) {
                const double4 v = a.vel64[cell];
                ux = R(v.x);
                uy = R(v.y);
                uz = R(v.z);
                rho = R(v.w);
            } else if (a.vel) {
                const float4 v = a.vel[cell];
                ux = R(v.x);
                uy = R(v.y);
                uz = R(v.z);
                rho = R(v.w);
            } else {
                // lane i < 19: the post-stream population i the last step read
                const T *src = static_cast<const T *>(a.vin.src);
                R fl = R(0);
                if (lane < 19) {
                    if (a.vin_kind == IN_POST_COLLISION) {
                        const Rows rw = neighbour_rows(a.vin, y, z);
                        fl = pull_dir<S>(a.vin, src, x, rw, cell, lane);
                        if (flag & FLAG_BOUNDARY)
                            fl = bouzidi_dir<S>(a.vin, src, x, rw, cell, lane, mask, first, fl);
                    } else {
                        fl = S::load(src + (long long)lane * n + cell, lane);
                    }
                }
                R fin[19];
#pragma unroll
                for (int j = 0; j < 19; j++) fin[j] = __shfl_sync(FULL, fl, j);
                prepare_cell<R>(fin, 0, x, nx, R(a.vin.inX), R(a.vin.inY), R(a.vin.inZ), rho, ux,
                                uy, uz);
            }
            // lane i in 1..18: the momentum exchange of link i
            R tx = R(0), ty = R(0), tz = R(0), qx = R(0), qy = R(0), qz = R(0);
            const int i = lane;
            if (i >= 1 && i < 19 && (mask & (1u << i))) {
                const T *g = static_cast<const T *>(st.src);
                const T *fe = static_cast<const T *>(a.fexp);
                const int io = opp(i);
                const R fi_star = S::load(g + (long long)i * n + cell, i);
                R f_iopp;
                if (fe) {
                    f_iopp = S::load(fe + (long long)io * n + cell, io);
                } else {
                    // post-stream f of direction io at this cell: Bouzidi
                    // with the q of link i (lbm_stream.comp:90-115)
                    const float q = st.lq[first + __popc(mask & ((1u << i) - 1u))];
                    const R qq = R(q);
                    if (q >= 0.5f) {
                        const R fio = S::load(g + (long long)io * n + cell, io);
                        const R inv2q = ddiv<R>(R(1), R(2) * qq);
                        f_iopp = inv2q * fi_star + (R(1) - inv2q) * fio;
                    } else {
                        const int fx = x + cx(io);
                        R ff;
                        if (fx >= 0 && fx < nx) {
                            const Rows rg = neighbour_rows(st, y, z);
                            ff = S::load(g + (long long)i * n + row_sel(rg.y, 1 + cy(io)) +
                                             row_sel(rg.z, 1 + cz(io)) + fx,
                                         i);
                        } else {
                            ff = fi_star;
                        }
                        const R twoq = R(2) * qq;
                        f_iopp = twoq * fi_star + (R(1) - twoq) * ff;
                    }
                }
                const R ftotal = fi_star + f_iopp;
                tx = ftotal * R(cx(i));
                ty = ftotal * R(cy(i));
                tz = ftotal * R(cz(i));
                const R fpressure = feq<R>(i, rho, ux, uy, uz) + feq<R>(io, rho, ux, uy, uz);
                qx = fpressure * R(cx(i));
                qy = fpressure * R(cy(i));
                qz = fpressure * R(cz(i));
            }
            // The cell's sums in the reference's order of directions.  A
            // direction without a link contributes +0 here where the
            // reference skips it: the same, since a sum that starts at +0
            // never becomes -0 under round-to-nearest and x + (+0) = x.
#pragma unroll
            for (int j = 1; j < 19; j++) {
                lx += __shfl_sync(FULL, tx, j);
                ly += __shfl_sync(FULL, ty, j);
                lz += __shfl_sync(FULL, tz, j);
                px += __shfl_sync(FULL, qx, j);
                py += __shfl_sync(FULL, qy, j);
                pz += __shfl_sync(FULL, qz, j);
            }
            has = (mask & 0x7fffeu) != 0;
        }
    }

    // per-cell rounding, block partials, and the last block's fixed-order total
    __shared__ long long s_i[FORCE_CELLS_PER_BLOCK][7];
    __shared__ double s_d[FORCE_CELLS_PER_BLOCK][6];
    __shared__ int s_last;
    if (lane == 0) {
        s_i[w][0] = has ? round_ll<R>(lx * R(10000)) : 0;
        s_i[w][1] = has ? round_ll<R>(ly * R(10000)) : 0;
        s_i[w][2] = has ? round_ll<R>(lz * R(10000)) : 0;
        s_i[w][3] = has;
        s_i[w][4] = has ? round_ll<R>(px * R(10000)) : 0;
        s_i[w][5] = has ? round_ll<R>(py * R(10000)) : 0;
        s_i[w][6] = has ? round_ll<R>(pz * R(10000)) : 0;
        s_d[w][0] = has ? double(lx) : 0.0;
        s_d[w][1] = has ? double(ly) : 0.0;
        s_d[w][2] = has ? double(lz) : 0.0;
        s_d[w][3] = has ? double(px) : 0.0;
        s_d[w][4] = has ? double(py) : 0.0;
        s_d[w][5] = has ? double(pz) : 0.0;
    }
    __syncthreads();
    long long *part = a.part + (long long)blockIdx.x * 16;
    if (threadIdx.x < 7) {
        long long v = 0;
        for (int k = 0; k < FORCE_CELLS_PER_BLOCK; k++) v += s_i[k][threadIdx.x];
        part[threadIdx.x] = v;
    } else if (threadIdx.x >= 8 && threadIdx.x < 14) {
        double v = 0.0;
        for (int k = 0; k < FORCE_CELLS_PER_BLOCK; k++) v += s_d[k][threadIdx.x - 8];
        part[threadIdx.x] = __double_as_longlong(v);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // one pass over the partials: thread t adds the rows of blocks t, t +
    // FORCE_THREADS, ...; then a fixed shuffle tree per warp and the warps
    // in order
    long long vi[7] = {0, 0, 0, 0, 0, 0, 0};
    double vd[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll 4
    for (int blk = threadIdx.x; blk < (int)gridDim.x; blk += FORCE_THREADS) {
        const long long *row = a.part + (long long)blk * 16;
        long long v[14];
#pragma unroll
        for (int k = 0; k < 14; k++) v[k] = __ldcg(row + k);
#pragma unroll
        for (int k = 0; k < 7; k++) vi[k] += v[k];
#pragma unroll
        for (int k = 0; k < 6; k++) vd[k] += __longlong_as_double(v[8 + k]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 7; k++) vi[k] += __shfl_down_sync(FULL, vi[k], o);
#pragma unroll
        for (int k = 0; k < 6; k++) vd[k] += __shfl_down_sync(FULL, vd[k], o);
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 7; k++) s_i[w][k] = vi[k];
#pragma unroll
        for (int k = 0; k < 6; k++) s_d[w][k] = vd[k];
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        long long v = 0;
        for (int k = 0; k < FORCE_CELLS_PER_BLOCK; k++) v += s_i[k][threadIdx.x];
        a.i64[threadIdx.x] = v;
    } else if (threadIdx.x >= 8 && threadIdx.x < 14) {
        double v = 0.0;
        for (int k = 0; k < FORCE_CELLS_PER_BLOCK; k++) v += s_d[k][threadIdx.x - 8];
        a.f64[threadIdx.x - 8] = v;
    } else if (threadIdx.x == 32) {
        *a.ticket = 0u;
    }
}

template <class S>
cudaError_t force_launch(const ForceArgs &a, int nb, cudaStream_t s) {
    const int blocks = (nb + FORCE_CELLS_PER_BLOCK - 1) / FORCE_CELLS_PER_BLOCK;
    k_force<S><<<blocks, FORCE_THREADS, 0, s>>>(a, nb);
    return cudaGetLastError();
}

}  // namespace

int force_blocks(int nb) {
    return (nb + FORCE_CELLS_PER_BLOCK - 1) / FORCE_CELLS_PER_BLOCK;
}

cudaError_t launch_force(const GridImpl &g, const void *gsrc, const void *f_explicit,
                         int periodic, const float4 *vel_or_null, const double4 *vel64_or_null,
                         const void *vin_src,
                         int vin_kind, int vin_periodic, const float vin_inlet[3],
                         long long *i64, double *f64, long long *part, unsigned *ticket,
                         cudaStream_t s) {
    if (g.links.nb == 0) {  // no link: every sum is zero
        cudaError_t e = cudaMemsetAsync(i64, 0, sizeof(long long) * 7, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(f64, 0, sizeof(double) * 6, s);
        return e;
    }
    ForceArgs a{};
    a.st.src = gsrc;
    a.bcell = g.links.bcell;
    a.st.flags = g.flags;
    a.st.slot = g.slot;
    a.st.bmask = g.links.bmask;
    a.st.bfirst = g.links.bfirst;
    a.st.lq = g.links.lq;
    a.st.nx = g.nx;
    a.st.ny = g.ny;
    a.st.nz = g.nz;
    a.st.n = g.n;
    a.st.periodic = periodic;
    a.fexp = f_explicit;
    a.vel = vel_or_null;
    a.vel64 = vel_or_null ? vel64_or_null : nullptr;
    a.vin = a.st;
    a.vin.src = vin_src;
    a.vin.periodic = vin_periodic;
    a.vin.inX = vin_inlet[0];
    a.vin.inY = vin_inlet[1];
    a.vin.inZ = vin_inlet[2];
    a.vin_kind = vin_kind;
    a.i64 = i64;
    a.f64 = f64;
    a.part = part;
    a.ticket = ticket;
    const int nb = g.links.nb;
    switch (g.storage) {
        case LBM_STORAGE_FP32: return force_launch<StoreF32>(a, nb, s);
        case LBM_STORAGE_FP64: return force_launch<StoreF64>(a, nb, s);
        case LBM_STORAGE_FP16: return force_launch<StoreF16>(a, nb, s);
        case LBM_STORAGE_BF16: return force_launch<StoreBF16>(a, nb, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace lbm
