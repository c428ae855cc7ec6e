// The warm-start network (LBM_WarmNet*): a 4-level 3D conv encoder-decoder
// mapping (voxel mask, inflow speed, Re) at quarter resolution to
// (rho, u), trained and run with this library's own kernels -- tensor-core
// convolutions (lbm_nn.cu) and the element-wise kernels below.  BF16
// activations and weights, FP32 accumulation, FP32 master weights with Adam.
//
// Architecture (level 1 = the quarter-resolution input, NX x NY x NZ):
//   level 1: conv 8->16, 16->16 = s1        decoder 1: [s1, up(d2)] 48->16->16 = d1
//   level 2: pool, 16->32, 32->32 = s2      decoder 2: [s2, up(d3)] 96->32->32 = d2
//   level 3: pool, 32->64, 64->64 = s3      decoder 3: [s3, up(s4)] 192->64->64 = d3
//   level 4: pool, 64->128, 128->128, 128->128 = s4
//   output:  conv 16->4, linear
// 3x3x3 convolutions with zero padding, leaky ReLU (slope 0.1), 2x2x2
// average pooling, nearest-neighbour upsampling; ~1.9 M parameters.
// Input channels: solid fraction, U / 0.1, log(Re / 100) / log(20), five
// zeros.  Outputs: (rho - 1) / U^2, u / U.  Loss: mean squared error.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <new>
#include <vector>

#include "lbm_internal.h"
#include "lbm_nn.h"
#include "lbm_nn_gemm.cuh"

namespace lbm {
namespace nn {

struct LayerSpec {
    int cin, cout, act;
};
constexpr int NLAYERS = 16;
constexpr LayerSpec kLayers[NLAYERS] = {
    {8, 16, 1},   {16, 16, 1},  {16, 32, 1},  {32, 32, 1},  {32, 64, 1},  {64, 64, 1},
    {64, 128, 1}, {128, 128, 1}, {128, 128, 1}, {192, 64, 1}, {64, 64, 1},  {96, 32, 1},
    {32, 32, 1},  {48, 16, 1},  {16, 16, 1},  {16, 4, 0}};
// level of each layer (0 = input resolution)
constexpr int kLevel[NLAYERS] = {0, 0, 1, 1, 2, 2, 3, 3, 3, 2, 2, 1, 1, 0, 0, 0};

inline int nt_of(int cout) { return cout < 16 ? 16 : cout; }
inline int pad16(int c) { return (c + 15) / 16 * 16; }
inline int round8(int c) { return (c + 7) / 8 * 8; }

// ---------------------------------------------------------------------------
// element-wise kernels

__global__ void k_features(const float *__restrict__ f, long long m, __nv_bfloat16 *__restrict__ x) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= m) return;
    __align__(16) __nv_bfloat16 h[8];
    h[0] = __float2bfloat16_rn(f[3 * v]);
    h[1] = __float2bfloat16_rn(f[3 * v + 1] / 0.1f);
    h[2] = __float2bfloat16_rn(logf(f[3 * v + 2] / 100.0f) / logf(20.0f));
#pragma unroll
    for (int i = 3; i < 8; i++) h[i] = __float2bfloat16_rn(0.f);
    *reinterpret_cast<uint4 *>(x + 8 * v) = *reinterpret_cast<const uint4 *>(h);
}

struct Lvl {
    int nz, ny, nx;
};

__device__ __forceinline__ long long vox(int b, int z, int y, int x, const Lvl &l) {
    return (((long long)b * l.nz + z) * l.ny + y) * l.nx + x;
}

// out[coarse][c] = bf16(mean of the 8 children of in (slice))
__global__ void k_pool(const __nv_bfloat16 *__restrict__ in, int is, int io, int c, Lvl fine,
                       __nv_bfloat16 *__restrict__ out, Lvl coarse, long long mc) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= mc * c) return;
    const int ch = (int)(i % c);
    long long v = i / c;
    const int x = (int)(v % coarse.nx);
    v /= coarse.nx;
    const int y = (int)(v % coarse.ny);
    v /= coarse.ny;
    const int z = (int)(v % coarse.nz);
    const int b = (int)(v / coarse.nz);
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const long long f = vox(b, 2 * z + (k >> 2), 2 * y + ((k >> 1) & 1), 2 * x + (k & 1), fine);
        acc += __bfloat162float(in[f * is + io + ch]);
    }
    out[i] = __float2bfloat16_rn(acc * 0.125f);
}

// fine slice (stride os, offset oo) += dout[coarse] / 8
__global__ void k_pool_bwd(const float *__restrict__ dout, int c, Lvl coarse, float *__restrict__ d,
                           int ds, int dof, Lvl fine, long long mf) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= mf * c) return;
    const int ch = (int)(i % c);
    long long v = i / c;
    const int x = (int)(v % fine.nx);
    long long t = v / fine.nx;
    const int y = (int)(t % fine.ny);
    t /= fine.ny;
    const int z = (int)(t % fine.nz);
    const int b = (int)(t / fine.nz);
    d[v * ds + dof + ch] += dout[vox(b, z / 2, y / 2, x / 2, coarse) * c + ch] * 0.125f;
}

// out slice [fine] = in[coarse]
__global__ void k_upsample(const __nv_bfloat16 *__restrict__ in, int c, Lvl coarse,
                           __nv_bfloat16 *__restrict__ out, int os, int oo, Lvl fine,
                           long long mf) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= mf * (c / 8)) return;
    const int q = (int)(i % (c / 8));
    long long v = i / (c / 8);
    const int x = (int)(v % fine.nx);
    long long t = v / fine.nx;
    const int y = (int)(t % fine.ny);
    t /= fine.ny;
    const int z = (int)(t % fine.nz);
    const int b = (int)(t / fine.nz);
    *reinterpret_cast<uint4 *>(out + v * os + oo + 8 * q) =
        *reinterpret_cast<const uint4 *>(in + vox(b, z / 2, y / 2, x / 2, coarse) * c + 8 * q);
}

// dd[coarse][c] = sum over the 8 children of the slice of dout
__global__ void k_upsample_bwd(const float *__restrict__ dout, int os, int oo, int c, Lvl fine,
                               float *__restrict__ dd, Lvl coarse, long long mc) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= mc * c) return;
    const int ch = (int)(i % c);
    long long v = i / c;
    const int x = (int)(v % coarse.nx);
    v /= coarse.nx;
    const int y = (int)(v % coarse.ny);
    v /= coarse.ny;
    const int z = (int)(v % coarse.nz);
    const int b = (int)(v / coarse.nz);
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const long long f = vox(b, 2 * z + (k >> 2), 2 * y + ((k >> 1) & 1), 2 * x + (k & 1), fine);
        acc += dout[f * os + oo + ch];
    }
    dd[i] = acc;
}

// g[m][nt] = bf16(dout * act'(out)) for ch < c, 0 above
__global__ void k_act_bwd(const float *__restrict__ dout, int ds, int dof,
                          const __nv_bfloat16 *__restrict__ out, int os, int oo, int c, int act,
                          __nv_bfloat16 *__restrict__ g, int nt, long long m) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m * nt) return;
    const int ch = (int)(i % nt);
    const long long v = i / nt;
    float r = 0.f;
    if (ch < c) {
        r = dout[v * ds + dof + ch];
        if (act && !(__bfloat162float(out[v * os + oo + ch]) > 0.f)) r *= 0.1f;
    }
    g[i] = __float2bfloat16_rn(r);
}

// k_act_bwd for 8 channels per thread: two float4 loads of the output
// gradient, one 16-byte load of the activations and one 16-byte store
// (strides and offsets multiples of 8, c a multiple of 8, fewer than 2^31
// groups -- checked by the caller).
__global__ void k_act_bwd8(const float *__restrict__ dout, int ds, int dof,
                           const __nv_bfloat16 *__restrict__ out, int os, int oo, int c, int act,
                           __nv_bfloat16 *__restrict__ g, int nt, unsigned groups) {
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= groups) return;
    const unsigned gq = (unsigned)nt >> 3, v = t / gq;
    const int ch0 = (int)(t - v * gq) * 8;
    __align__(16) __nv_bfloat16 h[8];
    if (ch0 < c) {
        const float4 *dp = reinterpret_cast<const float4 *>(dout + (long long)v * ds + dof + ch0);
        const float4 a = dp[0], b = dp[1];
        float r[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        if (act) {
            const uint4 q = *reinterpret_cast<const uint4 *>(out + (long long)v * os + oo + ch0);
            const __nv_bfloat16 *o = reinterpret_cast<const __nv_bfloat16 *>(&q);
#pragma unroll
            for (int i = 0; i < 8; i++)
                if (!(__bfloat162float(o[i]) > 0.f)) r[i] *= 0.1f;
        }
#pragma unroll
        for (int i = 0; i < 8; i++) h[i] = __float2bfloat16_rn(r[i]);
    } else {
#pragma unroll
        for (int i = 0; i < 8; i++) h[i] = __float2bfloat16_rn(0.f);
    }
    *reinterpret_cast<uint4 *>(g + (long long)v * nt + ch0) = *reinterpret_cast<const uint4 *>(h);
}

// loss and its gradient on the 4 output channels (prediction stride 16)
// Loss gradient of every output channel (16 per voxel, 4 real) and the
// squared error summed into *loss: a grid-stride loop, one FP64 atomic per
// block.
__global__ void k_loss(const __nv_bfloat16 *__restrict__ pred, const float *__restrict__ target,
                       long long m, float scale, __nv_bfloat16 *__restrict__ g,
                       double *__restrict__ loss) {
    double local = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m * 16;
         i += (long long)gridDim.x * blockDim.x) {
        const int ch = (int)(i & 15);
        const long long v = i >> 4;
        float r = 0.f;
        if (ch < 4) {
            const float d = __bfloat162float(pred[i]) - target[4 * v + ch];
            local += (double)d * d;
            r = scale * d;
        }
        g[i] = __float2bfloat16_rn(r);
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
    __shared__ double part[8];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += part[w];
        if (t != 0.0) atomicAdd(loss, t);
    }
}

// Bias gradient, pass 1: block b sums rows [b * BG_ROWS, (b + 1) * BG_ROWS)
// of g (nt channels per row, 8 per thread and 16-byte load) per channel in
// FP32 and writes partial[b][nt].
constexpr int BG_ROWS = 512;
__global__ void k_bias_grad_part(const __nv_bfloat16 *__restrict__ g, int nt, long long m,
                                 float *__restrict__ partial) {
    const int groups = nt >> 3;             // 16-byte groups per row
    const int rows_per_pass = 256 / groups;  // nt <= 256
    const int grp = threadIdx.x % groups, r0 = threadIdx.x / groups;
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const long long base = (long long)blockIdx.x * BG_ROWS;
    if (r0 < rows_per_pass) {
        for (int r = r0; r < BG_ROWS; r += rows_per_pass) {
            const long long v = base + r;
            if (v >= m) break;
            const uint4 q = *reinterpret_cast<const uint4 *>(g + v * nt + grp * 8);
            const __nv_bfloat16 *h = reinterpret_cast<const __nv_bfloat16 *>(&q);
#pragma unroll
            for (int i = 0; i < 8; i++) acc[i] += __bfloat162float(h[i]);
        }
    }
    __shared__ float red[256][9];
#pragma unroll
    for (int i = 0; i < 8; i++) red[threadIdx.x][i] = acc[i];
    __syncthreads();
    // thread c < nt sums channel c over the passes in a fixed order
    if ((int)threadIdx.x < nt) {
        const int c = threadIdx.x, cg = c >> 3, ci = c & 7;
        float t = 0.f;
        for (int r = 0; r < rows_per_pass; r++) t += red[r * groups + cg][ci];
        partial[(long long)blockIdx.x * nt + c] = t;
    }
}

// Bias gradient, pass 2: db[c] = sum over blocks of partial[b][c] in FP64;
// one warp per channel, lane l summing blocks l, l + 32, ... and the lanes
// combined by a fixed shuffle tree (deterministic).
__global__ void k_bias_grad_sum(const float *__restrict__ partial, int blocks, int nt, int cout,
                                float *__restrict__ db) {
    const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (c >= cout) return;
    double t = 0.0;
    for (int b = lane; b < blocks; b += 32) t += partial[(long long)b * nt + c];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) db[c] = (float)t;
}

// sum of squares of the gradient (for global-norm clipping)
__global__ void k_sqnorm(const float *__restrict__ g, long long n, double *__restrict__ out) {
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        acc += (double)g[i] * g[i];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

// Adam; with clip > 0 the gradient is scaled by min(1, clip / ||g||)
__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ mo,
                       float *__restrict__ ve, long long n, float lr_t, float b1, float b2,
                       float eps, float clip, const double *__restrict__ sq) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float gi = g[i];
    if (clip > 0.f) {
        const double norm = sqrt(*sq);
        if (norm > clip) gi *= (float)(clip / norm);
    }
    const float mi = b1 * mo[i] + (1.f - b1) * gi;
    const float vi = b2 * ve[i] + (1.f - b2) * gi * gi;
    mo[i] = mi;
    ve[i] = vi;
    p[i] -= lr_t * mi / (sqrtf(vi) + eps);
}

// All layers' packing in one launch: per layer the BF16 weights [nt][k_pad]
// and FP32 bias [nt] of k_pack, and (layers > 0) the flipped, transposed
// BF16 weights of the input gradient, wt[ci][(26 - tap) nt + co] =
// bf16(W[co][tap cin + ci]) (zero for ci >= cin or co >= cout) -- the values
// k_pack + k_weight_transpose produce, computed from the FP32 masters.
struct PackLayer {
    const float *w, *b;
    __nv_bfloat16 *wb, *wt;
    float *bias;
    int cout, cin, nt, kpad, wt_rows, wt_kpad;
    long long start;  // first element of this layer in the launch
};
struct PackTable {
    PackLayer l[16];
    long long total;
};

__global__ void k_pack_all(const __grid_constant__ PackTable t) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.total) return;
    int l = 0;
    while (l < 15 && i >= t.l[l + 1].start) l++;
    const PackLayer &L = t.l[l];
    long long e = i - L.start;
    const int kreal = 27 * L.cin;
    const long long nwb = (long long)L.nt * L.kpad;
    if (e < nwb) {
        const int n = (int)(e / L.kpad), k = (int)(e - (long long)n * L.kpad);
        L.wb[e] = __float2bfloat16_rn((n < L.cout && k < kreal) ? L.w[(long long)n * kreal + k]
                                                                 : 0.f);
        return;
    }
    e -= nwb;
    if (e < L.nt) {
        L.bias[e] = e < L.cout ? L.b[e] : 0.f;
        return;
    }
    e -= L.nt;
    // transposed weights
    const int ci = (int)(e / L.wt_kpad), k = (int)(e - (long long)ci * L.wt_kpad);
    float v = 0.f;
    if (ci < L.cin && k < 27 * L.nt) {
        const int tp = k / L.nt, co = k - tp * L.nt;
        if (co < L.cout) v = L.w[(long long)co * kreal + (26 - tp) * L.cin + ci];
    }
    L.wt[e] = __float2bfloat16_rn(v);
}

struct OutScale {
    float scale[4], shift[4];
};

// pred [m][16] bf16 -> [m][4] fp32 in physical units: shift + scale * p
__global__ void k_pred_out(const __nv_bfloat16 *__restrict__ pred, long long m, OutScale os,
                           float *__restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m * 4) return;
    const int k = (int)(i & 3);
    out[i] = os.shift[k] + os.scale[k] * __bfloat162float(pred[(i >> 2) * 16 + k]);
}

inline unsigned nblk(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// Per x-plane sums of a full-resolution field: flux rho * u_x over all
// cells, fluid-cell count, and the density sum over fluid cells.  One block
// per plane, fixed summation order.
__global__ void k_plane_sums(const float *__restrict__ rho, const float *__restrict__ u,
                             const int32_t *__restrict__ solid, int NX, int NY, int NZ,
                             double *__restrict__ out) {
    const int x = blockIdx.x;
    double flux = 0.0, cnt = 0.0, rs = 0.0;
    for (long long q = threadIdx.x; q < (long long)NY * NZ; q += blockDim.x) {
        const long long c = q * NX + x;
        flux += (double)rho[c] * u[3 * c];
        if (solid[c] == 0) {
            cnt += 1.0;
            rs += rho[c];
        }
    }
    __shared__ double sh[3][256];
    sh[0][threadIdx.x] = flux;
    sh[1][threadIdx.x] = cnt;
    sh[2][threadIdx.x] = rs;
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st)
            for (int k = 0; k < 3; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x < 3) out[3 * x + threadIdx.x] = sh[threadIdx.x][0];
}

// Continuity: shift u_x of the fluid cells of every x-plane so that the
// plane carries the inlet mass flux U * NY * NZ, and shift the density so
// that the outlet plane's fluid mean is the outlet's rho = 1.
__global__ void k_flux_correct(float *__restrict__ rho, float *__restrict__ u,
                               const int32_t *__restrict__ solid, int NX, int NY, int NZ, float U,
                               const double *__restrict__ sums) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)NX * NY * NZ || solid[c] != 0) return;
    const int x = (int)(c % NX);
    const double cnt = sums[3 * x + 1];
    if (cnt <= 0.0) return;
    const double target = (double)U * NY * NZ;
    u[3 * c] += (float)((target - sums[3 * x]) / cnt);
    const double cout_ = sums[3 * (NX - 1) + 1];
    if (cout_ > 0.0) rho[c] += (float)(1.0 - sums[3 * (NX - 1) + 2] / cout_);
}

// features of a grid at 1/f resolution: solid fraction of each f^3 block
// (cells with solid == 1), U and Re
__global__ void k_grid_features(const int32_t *__restrict__ solid, int NX, int NY, int NZ, int f,
                                float U, float Re, float *__restrict__ feat) {
    const int nx = NX / f, ny = NY / f, nz = NZ / f;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= (long long)nx * ny * nz) return;
    const int x = (int)(v % nx), y = (int)((v / nx) % ny), z = (int)(v / ((long long)nx * ny));
    int cnt = 0;
    for (int dz = 0; dz < f; dz++)
        for (int dy = 0; dy < f; dy++)
            for (int dx = 0; dx < f; dx++)
                cnt += solid[((long long)(z * f + dz) * NY + y * f + dy) * NX + x * f + dx] == 1;
    feat[3 * v] = (float)cnt / (float)(f * f * f);
    feat[3 * v + 1] = U;
    feat[3 * v + 2] = Re;
}

// training targets of a grid at 1/f resolution: block means of
// ((rho - 1) / U^2, u / U) with solid cells taken as rho = 1, u = 0
__global__ void k_grid_targets(const float4 *__restrict__ vel, const int32_t *__restrict__ solid,
                               int NX, int NY, int NZ, int f, float U, float *__restrict__ tgt) {
    const int nx = NX / f, ny = NY / f, nz = NZ / f;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= (long long)nx * ny * nz) return;
    const int x = (int)(v % nx), y = (int)((v / nx) % ny), z = (int)(v / ((long long)nx * ny));
    float s[4] = {0.f, 0.f, 0.f, 0.f};
    for (int dz = 0; dz < f; dz++)
        for (int dy = 0; dy < f; dy++)
            for (int dx = 0; dx < f; dx++) {
                const long long c = ((long long)(z * f + dz) * NY + y * f + dy) * NX + x * f + dx;
                if (solid[c] != 0) continue;
                const float4 q = vel[c];
                s[0] += (q.w - 1.f) / (U * U);
                s[1] += q.x / U;
                s[2] += q.y / U;
                s[3] += q.z / U;
            }
    const float inv = 1.f / (float)(f * f * f);
#pragma unroll
    for (int k = 0; k < 4; k++) tgt[4 * v + k] = s[k] * inv;
}

// full-resolution (rho, u) from the prediction at 1/f resolution: trilinear
// interpolation at cell centres ((x + 0.5) / f - 0.5, clamped), decoded as
// rho = 1 + U^2 p0 (or 1 when use_density is 0), u = U (p1, p2, p3); solid
// cells rho = 1, u = 0
__global__ void k_decode_upsample(const float *__restrict__ pred, int nx, int ny, int nz, int f,
                                  float U, const int32_t *__restrict__ solid, int NX, int NY,
                                  int NZ, float *__restrict__ rho, float *__restrict__ u,
                                  int use_density) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)NX * NY * NZ) return;
    const int X = (int)(c % NX), Y = (int)((c / NX) % NY), Z = (int)(c / ((long long)NX * NY));
    if (solid[c] != 0) {
        rho[c] = 1.f;
        u[3 * c] = u[3 * c + 1] = u[3 * c + 2] = 0.f;
        return;
    }
    const float inv = 1.f / (float)f;
    float px = fminf(fmaxf((X + 0.5f) * inv - 0.5f, 0.f), (float)(nx - 1));
    float py = fminf(fmaxf((Y + 0.5f) * inv - 0.5f, 0.f), (float)(ny - 1));
    float pz = fminf(fmaxf((Z + 0.5f) * inv - 0.5f, 0.f), (float)(nz - 1));
    const int x0 = (int)px, y0 = (int)py, z0 = (int)pz;
    const int x1 = min(x0 + 1, nx - 1), y1 = min(y0 + 1, ny - 1), z1 = min(z0 + 1, nz - 1);
    const float fx = px - x0, fy = py - y0, fz = pz - z0;
    float o[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        auto P = [&](int zz, int yy, int xx) {
            return pred[4 * (((long long)zz * ny + yy) * nx + xx) + k];
        };
        const float c00 = P(z0, y0, x0) * (1 - fx) + P(z0, y0, x1) * fx;
        const float c01 = P(z0, y1, x0) * (1 - fx) + P(z0, y1, x1) * fx;
        const float c10 = P(z1, y0, x0) * (1 - fx) + P(z1, y0, x1) * fx;
        const float c11 = P(z1, y1, x0) * (1 - fx) + P(z1, y1, x1) * fx;
        o[k] = (c00 * (1 - fy) + c01 * fy) * (1 - fz) + (c10 * (1 - fy) + c11 * fy) * fz;
    }
    rho[c] = use_density ? 1.f + U * U * o[0] : 1.f;
    u[3 * c] = U * o[1];
    u[3 * c + 1] = U * o[2];
    u[3 * c + 2] = U * o[3];
}

}  // namespace nn
}  // namespace lbm

using namespace lbm;
using namespace lbm::nn;

struct LBMWarmNet {
    int nx = 0, ny = 0, nz = 0, maxb = 0;
    Lvl lvl[4];
    long long vox1 = 0;  // voxels of one sample at level 1
    cudaStream_t stream = nullptr;
    std::vector<void *> allocs;
    long long P = 0;
    long long woff[NLAYERS], boff[NLAYERS];
    float *params = nullptr, *grad = nullptr, *am = nullptr, *av = nullptr;
    long long adam_t = 0;
    __nv_bfloat16 *wb[NLAYERS] = {}, *wt[NLAYERS] = {};
    float *bias[NLAYERS] = {};
    bool packed = false;
    // activations (bf16)
    __nv_bfloat16 *in0, *a1, *cat1, *in2, *a2, *cat2, *in3, *a3, *cat3, *in4, *a4, *b4, *s4, *c3,
        *d3, *c2, *d2, *c1, *d1, *pred;
    // activation gradients (fp32)
    float *dd1, *dc1, *dcat1, *dd2, *dc2, *dcat2, *dd3, *dc3, *dcat3, *ds4, *db4, *da4, *din4,
        *da3, *din3, *da2, *din2, *da1;
    __nv_bfloat16 *g = nullptr;  // pre-activation gradient of the current layer
    float *ws = nullptr;
    long long ws_bytes = 0;
    float *feat = nullptr, *target = nullptr, *pred32 = nullptr;
    double *loss = nullptr;
    float *bias_part = nullptr;  // per-block partial bias gradients
    int error = 0;
    OutScale out_scale = {{1.f, 1.f, 1.f, 1.f}, {0.f, 0.f, 0.f, 0.f}};
    float clip = 0.f;
    double *sq = nullptr;

    template <class T>
    T *alloc(long long n) {
        void *p = nullptr;
        if (cudaMalloc(&p, (size_t)(n > 0 ? n : 1) * sizeof(T)) != cudaSuccess) {
            error = 1;
            return nullptr;
        }
        cudaMemsetAsync(p, 0, (size_t)(n > 0 ? n : 1) * sizeof(T), stream);
        allocs.push_back(p);
        return static_cast<T *>(p);
    }
    long long m(int level, int nb) const {
        return (long long)nb * lvl[level].nz * lvl[level].ny * lvl[level].nx;
    }
};

namespace {

struct Wsplit {
    unsigned splits;
    int chunks;
};

Wsplit wgrad_split(long long m, int kpad) {
    const long long tiles = kpad / 128;
    const long long max_chunks = (m + KC - 1) / KC;
    long long splits = (1184 + tiles - 1) / tiles;  // about eight CTAs per SM
    if (splits > max_chunks) splits = max_chunks;
    if (splits < 1) splits = 1;
    const int chunks = (int)((max_chunks + splits - 1) / splits);
    return {(unsigned)((max_chunks + chunks - 1) / chunks), chunks};
}

// deterministic uniform in [-1, 1) from (seed, index)
float hash_uniform(uint32_t seed, uint64_t i) {
    uint64_t x = (uint64_t)seed * 0x9E3779B97F4A7C15ull + i + 0x632BE59BD9B4E019ull;
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return (float)((double)(x >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0);
}

bool ok(LBMWarmNet *n, cudaError_t e) {
    if (e != cudaSuccess) n->error = 1;
    return e == cudaSuccess;
}

// layer io: input buffer/stride/offset, output buffer/stride/offset
struct Io {
    const __nv_bfloat16 *x;
    int xs, xo;
    __nv_bfloat16 *y;
    int ys, yo;
};

Io layer_io(const LBMWarmNet &n, int l) {
    switch (l) {
        case 0: return {n.in0, 8, 0, n.a1, 16, 0};
        case 1: return {n.a1, 16, 0, n.cat1, 48, 0};
        case 2: return {n.in2, 16, 0, n.a2, 32, 0};
        case 3: return {n.a2, 32, 0, n.cat2, 96, 0};
        case 4: return {n.in3, 32, 0, n.a3, 64, 0};
        case 5: return {n.a3, 64, 0, n.cat3, 192, 0};
        case 6: return {n.in4, 64, 0, n.a4, 128, 0};
        case 7: return {n.a4, 128, 0, n.b4, 128, 0};
        case 8: return {n.b4, 128, 0, n.s4, 128, 0};
        case 9: return {n.cat3, 192, 0, n.c3, 64, 0};
        case 10: return {n.c3, 64, 0, n.d3, 64, 0};
        case 11: return {n.cat2, 96, 0, n.c2, 32, 0};
        case 12: return {n.c2, 32, 0, n.d2, 32, 0};
        case 13: return {n.cat1, 48, 0, n.c1, 16, 0};
        case 14: return {n.c1, 16, 0, n.d1, 16, 0};
        default: return {n.d1, 16, 0, n.pred, 16, 0};
    }
}

// gradient of a layer's output (fp32 buffer, stride, offset) and of its
// input (the input-gradient convolution's destination)
struct Gio {
    float *dout;
    int ds, dof;
    float *din;
    int dis, dio;
};

Gio layer_gio(const LBMWarmNet &n, int l) {
    switch (l) {
        case 0: return {n.da1, 16, 0, nullptr, 0, 0};
        case 1: return {n.dcat1, 48, 0, n.da1, 16, 0};
        case 2: return {n.da2, 32, 0, n.din2, 16, 0};
        case 3: return {n.dcat2, 96, 0, n.da2, 32, 0};
        case 4: return {n.da3, 64, 0, n.din3, 32, 0};
        case 5: return {n.dcat3, 192, 0, n.da3, 64, 0};
        case 6: return {n.da4, 128, 0, n.din4, 64, 0};
        case 7: return {n.db4, 128, 0, n.da4, 128, 0};
        case 8: return {n.ds4, 128, 0, n.db4, 128, 0};
        case 9: return {n.dc3, 64, 0, n.dcat3, 192, 0};
        case 10: return {n.dd3, 64, 0, n.dc3, 64, 0};
        case 11: return {n.dc2, 32, 0, n.dcat2, 96, 0};
        case 12: return {n.dd2, 32, 0, n.dc2, 32, 0};
        case 13: return {n.dc1, 16, 0, n.dcat1, 48, 0};
        case 14: return {n.dd1, 16, 0, n.dc1, 16, 0};
        default: return {nullptr, 0, 0, n.dd1, 16, 0};
    }
}

bool pack(LBMWarmNet *n) {
    static_assert(NLAYERS == 16, "PackTable holds 16 layers");
    PackTable t{};
    long long at = 0;
    for (int l = 0; l < NLAYERS; l++) {
        PackLayer &L = t.l[l];
        L.w = n->params + n->woff[l];
        L.b = n->params + n->boff[l];
        L.wb = n->wb[l];
        L.wt = l > 0 ? n->wt[l] : nullptr;
        L.bias = n->bias[l];
        L.cout = kLayers[l].cout;
        L.cin = kLayers[l].cin;
        L.nt = nt_of(L.cout);
        L.kpad = k_pad_of(L.cin);
        L.wt_rows = l > 0 ? pad16(L.cin) : 0;
        L.wt_kpad = k_pad_of(L.nt);
        L.start = at;
        at += (long long)L.nt * L.kpad + L.nt + (long long)L.wt_rows * L.wt_kpad;
    }
    t.total = at;
    k_pack_all<<<nblk(at), 256, 0, n->stream>>>(t);
    if (!ok(n, cudaGetLastError())) return false;
    n->packed = true;
    return true;
}

Dims dims_of(const LBMWarmNet &n, int level, int nb) {
    return Dims{nb, n.lvl[level].nz, n.lvl[level].ny, n.lvl[level].nx};
}

bool forward(LBMWarmNet *n, const float *feat_dev, int nb) {
    if (!n->packed && !pack(n)) return false;
    cudaStream_t s = n->stream;
    const long long m1 = n->m(0, nb);
    k_features<<<nblk(m1), 256, 0, s>>>(feat_dev, m1, n->in0);
    auto conv = [&](int l) {
        const Io io = layer_io(*n, l);
        ConvFwdArgs a{};
        a.x = io.x;
        a.x_stride = io.xs;
        a.x_off = io.xo;
        a.cin = kLayers[l].cin;
        a.w = n->wb[l];
        a.k_real = 27 * kLayers[l].cin;
        a.k_pad = k_pad_of(kLayers[l].cin);
        a.bias = n->bias[l];
        a.act = kLayers[l].act;
        a.y = io.y;
        a.y_stride = io.ys;
        a.y_off = io.yo;
        a.cout_store = l == NLAYERS - 1 ? 16 : kLayers[l].cout;
        a.d = dims_of(*n, kLevel[l], nb);
        a.m = n->m(kLevel[l], nb);
        return ok(n, conv_forward(a, nt_of(kLayers[l].cout), s));
    };
    auto pool = [&](const __nv_bfloat16 *in, int is, int c, int lf, __nv_bfloat16 *out) {
        const long long mc = n->m(lf + 1, nb);
        k_pool<<<nblk(mc * c), 256, 0, s>>>(in, is, 0, c, n->lvl[lf], out, n->lvl[lf + 1], mc);
        return ok(n, cudaGetLastError());
    };
    auto up = [&](const __nv_bfloat16 *in, int c, int lc, __nv_bfloat16 *out, int os, int oo) {
        const long long mf = n->m(lc - 1, nb);
        k_upsample<<<nblk(mf * (c / 8)), 256, 0, s>>>(in, c, n->lvl[lc], out, os, oo,
                                                      n->lvl[lc - 1], mf);
        return ok(n, cudaGetLastError());
    };
    return conv(0) && conv(1) && pool(n->cat1, 48, 16, 0, n->in2) && conv(2) && conv(3) &&
           pool(n->cat2, 96, 32, 1, n->in3) && conv(4) && conv(5) &&
           pool(n->cat3, 192, 64, 2, n->in4) && conv(6) && conv(7) && conv(8) &&
           up(n->s4, 128, 3, n->cat3, 192, 64) && conv(9) && conv(10) &&
           up(n->d3, 64, 2, n->cat2, 96, 32) && conv(11) && conv(12) &&
           up(n->d2, 32, 1, n->cat1, 48, 16) && conv(13) && conv(14) && conv(15);
}

// loss, then the gradient of every parameter into n->grad
bool backward(LBMWarmNet *n, const float *target_dev, int nb) {
    cudaStream_t s = n->stream;
    const long long m1 = n->m(0, nb);
    if (!ok(n, cudaMemsetAsync(n->loss, 0, sizeof(double), s))) return false;
    k_loss<<<148 * 8, 256, 0, s>>>(n->pred, target_dev, m1, 2.0f / (float)(m1 * 4), n->g,
                                   n->loss);
    if (!ok(n, cudaGetLastError())) return false;
    for (int l = NLAYERS - 1; l >= 0; l--) {
        const int lv = kLevel[l], nt = nt_of(kLayers[l].cout), cin = kLayers[l].cin;
        const long long m = n->m(lv, nb);
        const Io io = layer_io(*n, l);
        const Gio gi = layer_gio(*n, l);
        if (l < NLAYERS - 1) {
            const int c = kLayers[l].cout;
            if (gi.ds % 4 == 0 && gi.dof % 4 == 0 && io.ys % 8 == 0 && io.yo % 8 == 0 &&
                c % 8 == 0 && nt % 8 == 0 && m * (nt / 8) < (1ll << 31))
                k_act_bwd8<<<nblk(m * (nt / 8)), 256, 0, s>>>(gi.dout, gi.ds, gi.dof, io.y, io.ys,
                                                              io.yo, c, kLayers[l].act, n->g, nt,
                                                              (unsigned)(m * (nt / 8)));
            else
                k_act_bwd<<<nblk(m * nt), 256, 0, s>>>(gi.dout, gi.ds, gi.dof, io.y, io.ys, io.yo,
                                                       c, kLayers[l].act, n->g, nt, m);
            if (!ok(n, cudaGetLastError())) return false;
        }
        // weight and bias gradients
        ConvWgradArgs w{};
        w.x = io.x;
        w.x_stride = io.xs;
        w.x_off = io.xo;
        w.cin = cin;
        w.g = n->g;
        w.g_stride = nt;
        w.cout = round8(kLayers[l].cout);
        w.k_real = 27 * cin;
        w.k_pad = k_pad_of(cin);
        w.partial = n->ws;
        w.d = dims_of(*n, lv, nb);
        w.m = m;
        const Wsplit sp = wgrad_split(m, w.k_pad);
        w.chunks_per_split = sp.chunks;
        bool bias_done = false;
        const unsigned room = (unsigned)(n->ws_bytes / ((long long)w.k_pad * nt * 4));
        if (!ok(n, conv_wgrad(w, nt, sp.splits, n->grad + n->woff[l], 0, s, kLayers[l].cout,
                              n->grad + n->boff[l], &bias_done, room)))
            return false;
        if (!bias_done) {
            const unsigned bb = nblk(m, BG_ROWS);
            k_bias_grad_part<<<bb, 256, 0, s>>>(n->g, nt, m, n->bias_part);
            k_bias_grad_sum<<<(kLayers[l].cout + 7) / 8, 256, 0, s>>>(
                n->bias_part, (int)bb, nt, kLayers[l].cout, n->grad + n->boff[l]);
        }
        if (!ok(n, cudaGetLastError())) return false;
        // input gradient
        if (l > 0) {
            ConvFwdArgs a{};
            a.x = n->g;
            a.x_stride = nt;
            a.x_off = 0;
            a.cin = nt;
            a.w = n->wt[l];
            a.k_real = 27 * nt;
            a.k_pad = k_pad_of(nt);
            a.act = 0;
            a.y32 = gi.din;
            a.y_stride = gi.dis;
            a.y_off = gi.dio;
            a.cout_store = cin;
            a.d = w.d;
            a.m = m;
            if (!ok(n, conv_forward(a, pad16(cin), s))) return false;
        }
        // routing through the upsampling and pooling joints
        auto up_bwd = [&](const float *dcat, int cs, int co, int c, int lf, float *dd) {
            const long long mc = n->m(lf + 1, nb);
            k_upsample_bwd<<<nblk(mc * c), 256, 0, s>>>(dcat, cs, co, c, n->lvl[lf], dd,
                                                         n->lvl[lf + 1], mc);
            return ok(n, cudaGetLastError());
        };
        auto pool_bwd = [&](const float *din, int c, int lc, float *dcat, int cs) {
            const long long mf = n->m(lc - 1, nb);
            k_pool_bwd<<<nblk(mf * c), 256, 0, s>>>(din, c, n->lvl[lc], dcat, cs, 0,
                                                    n->lvl[lc - 1], mf);
            return ok(n, cudaGetLastError());
        };
        bool good = true;
        if (l == 13) good = up_bwd(n->dcat1, 48, 16, 32, 0, n->dd2);
        if (l == 11) good = up_bwd(n->dcat2, 96, 32, 64, 1, n->dd3);
        if (l == 9) good = up_bwd(n->dcat3, 192, 64, 128, 2, n->ds4);
        if (l == 6) good = pool_bwd(n->din4, 64, 3, n->dcat3, 192);
        if (l == 4) good = pool_bwd(n->din3, 32, 2, n->dcat2, 96);
        if (l == 2) good = pool_bwd(n->din2, 16, 1, n->dcat1, 48);
        if (!good) return false;
    }
    return true;
}

int finish(LBMWarmNet *n) {
    if (!ok(n, cudaStreamSynchronize(n->stream))) return LBM_ERR_CUDA;
    if (take_error()) return LBM_ERR_TIMEOUT;
    return n->error ? LBM_ERR_CUDA : LBM_OK;
}

bool valid_batch(const LBMWarmNet *n, int nb) { return n && nb > 0 && nb <= n->maxb; }

}  // namespace

extern "C" {

long long LBM_WarmNetParamCount(void) {
    long long p = 0;
    for (int l = 0; l < NLAYERS; l++) p += (long long)kLayers[l].cout * (27 * kLayers[l].cin + 1);
    return p;
}

LBMWarmNet *LBM_WarmNetCreate(int nx, int ny, int nz, int maxBatch, unsigned seed) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || nx % 8 || ny % 8 || nz % 8 || maxBatch <= 0 ||
        (long long)nx * ny * nz < 1024)
        return nullptr;
    LBMWarmNet *n = new (std::nothrow) LBMWarmNet();
    if (!n) return nullptr;
    n->nx = nx;
    n->ny = ny;
    n->nz = nz;
    n->maxb = maxBatch;
    for (int i = 0; i < 4; i++) n->lvl[i] = Lvl{nz >> i, ny >> i, nx >> i};
    n->vox1 = (long long)nx * ny * nz;
    if (cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete n;
        return nullptr;
    }
    const int B = maxBatch;
    long long off = 0;
    for (int l = 0; l < NLAYERS; l++) {
        n->woff[l] = off;
        off += (long long)kLayers[l].cout * 27 * kLayers[l].cin;
        n->boff[l] = off;
        off += kLayers[l].cout;
    }
    n->P = off;
    n->params = n->alloc<float>(n->P);
    n->grad = n->alloc<float>(n->P);
    n->am = n->alloc<float>(n->P);
    n->av = n->alloc<float>(n->P);
    for (int l = 0; l < NLAYERS; l++) {
        const int nt = nt_of(kLayers[l].cout);
        n->wb[l] = n->alloc<__nv_bfloat16>((long long)nt * k_pad_of(kLayers[l].cin));
        n->bias[l] = n->alloc<float>(nt);
        if (l > 0)
            n->wt[l] = n->alloc<__nv_bfloat16>((long long)pad16(kLayers[l].cin) * k_pad_of(nt));
    }
    const long long m1 = n->m(0, B), m2 = n->m(1, B), m3 = n->m(2, B), m4 = n->m(3, B);
    typedef __nv_bfloat16 H;
    n->in0 = n->alloc<H>(m1 * 8);
    n->a1 = n->alloc<H>(m1 * 16);
    n->cat1 = n->alloc<H>(m1 * 48);
    n->in2 = n->alloc<H>(m2 * 16);
    n->a2 = n->alloc<H>(m2 * 32);
    n->cat2 = n->alloc<H>(m2 * 96);
    n->in3 = n->alloc<H>(m3 * 32);
    n->a3 = n->alloc<H>(m3 * 64);
    n->cat3 = n->alloc<H>(m3 * 192);
    n->in4 = n->alloc<H>(m4 * 64);
    n->a4 = n->alloc<H>(m4 * 128);
    n->b4 = n->alloc<H>(m4 * 128);
    n->s4 = n->alloc<H>(m4 * 128);
    n->c3 = n->alloc<H>(m3 * 64);
    n->d3 = n->alloc<H>(m3 * 64);
    n->c2 = n->alloc<H>(m2 * 32);
    n->d2 = n->alloc<H>(m2 * 32);
    n->c1 = n->alloc<H>(m1 * 16);
    n->d1 = n->alloc<H>(m1 * 16);
    n->pred = n->alloc<H>(m1 * 16);
    n->dd1 = n->alloc<float>(m1 * 16);
    n->dc1 = n->alloc<float>(m1 * 16);
    n->dcat1 = n->alloc<float>(m1 * 48);
    n->dd2 = n->alloc<float>(m2 * 32);
    n->dc2 = n->alloc<float>(m2 * 32);
    n->dcat2 = n->alloc<float>(m2 * 96);
    n->dd3 = n->alloc<float>(m3 * 64);
    n->dc3 = n->alloc<float>(m3 * 64);
    n->dcat3 = n->alloc<float>(m3 * 192);
    n->ds4 = n->alloc<float>(m4 * 128);
    n->db4 = n->alloc<float>(m4 * 128);
    n->da4 = n->alloc<float>(m4 * 128);
    n->din4 = n->alloc<float>(m4 * 64);
    n->da3 = n->alloc<float>(m3 * 64);
    n->din3 = n->alloc<float>(m3 * 32);
    n->da2 = n->alloc<float>(m2 * 32);
    n->din2 = n->alloc<float>(m2 * 16);
    n->da1 = n->alloc<float>(m1 * 16);
    long long gmax = 0, wsmax = 0;
    for (int l = 0; l < NLAYERS; l++) {
        const long long m = n->m(kLevel[l], B);
        const int nt = nt_of(kLayers[l].cout), kp = k_pad_of(kLayers[l].cin);
        gmax = m * nt > gmax ? m * nt : gmax;
        const Wsplit sp = wgrad_split(m, kp);
        // layers of <= 32 output channels: room for 256 partials (at most one
        // per 64 voxels) as well -- the z-folded weight gradient gives each
        // column of tiles (128 at the finest level, batch 8, 64x32x32) and
        // range of z its own
        long long room = sp.splits;
        if (nt <= 32) {
            const long long cap = (m + KC - 1) / KC < 256 ? (m + KC - 1) / KC : 256;
            room = room > cap ? room : cap;
        }
        const long long ws = room * kp * nt;
        wsmax = ws > wsmax ? ws : wsmax;
    }
    n->g = n->alloc<H>(gmax);
    n->ws = n->alloc<float>(wsmax);
    n->ws_bytes = wsmax * 4;
    n->feat = n->alloc<float>(m1 * 3);
    n->target = n->alloc<float>(m1 * 4);
    n->pred32 = n->alloc<float>(m1 * 4);
    n->loss = n->alloc<double>(1);
    n->sq = n->alloc<double>(1);
    {
        long long bp = 0;  // largest (blocks x nt) of the bias-gradient partials
        for (int l = 0; l < NLAYERS; l++) {
            const long long b = (n->m(kLevel[l], B) + BG_ROWS - 1) / BG_ROWS;
            bp = b * nt_of(kLayers[l].cout) > bp ? b * nt_of(kLayers[l].cout) : bp;
        }
        n->bias_part = n->alloc<float>(bp);
    }
    if (n->error) {
        LBM_WarmNetFree(n);
        return nullptr;
    }
    // He-style uniform initialisation from the seed; the output layer small
    std::vector<float> h((size_t)n->P, 0.f);
    for (int l = 0; l < NLAYERS; l++) {
        const long long nw = (long long)kLayers[l].cout * 27 * kLayers[l].cin;
        const float a = sqrtf(6.0f / (27.0f * kLayers[l].cin)) * (l == NLAYERS - 1 ? 0.1f : 1.0f);
        for (long long i = 0; i < nw; i++) h[n->woff[l] + i] = a * hash_uniform(seed, n->woff[l] + i);
    }
    if (cudaMemcpyAsync(n->params, h.data(), sizeof(float) * n->P, cudaMemcpyHostToDevice,
                        n->stream) != cudaSuccess ||
        cudaStreamSynchronize(n->stream) != cudaSuccess) {
        LBM_WarmNetFree(n);
        return nullptr;
    }
    return n;
}

void LBM_WarmNetFree(LBMWarmNet *n) {
    if (!n) return;
    if (n->stream) cudaStreamSynchronize(n->stream);
    for (void *p : n->allocs) cudaFree(p);
    if (n->stream) cudaStreamDestroy(n->stream);
    delete n;
}

int LBM_WarmNetGetParams(LBMWarmNet *n, float *host) {
    if (!n || !host) return LBM_ERR_INVALID_ARGUMENT;
    if (!ok(n, cudaMemcpyAsync(host, n->params, sizeof(float) * n->P, cudaMemcpyDeviceToHost,
                               n->stream)))
        return LBM_ERR_CUDA;
    return finish(n);
}

int LBM_WarmNetSetParams(LBMWarmNet *n, const float *host) {
    if (!n || !host) return LBM_ERR_INVALID_ARGUMENT;
    if (!ok(n, cudaMemcpyAsync(n->params, host, sizeof(float) * n->P, cudaMemcpyHostToDevice,
                               n->stream)))
        return LBM_ERR_CUDA;
    n->packed = false;
    return finish(n);
}

int LBM_WarmNetForwardDevice(LBMWarmNet *n, const float *features, int batch, float *pred) {
    if (!valid_batch(n, batch) || !features || !pred) return LBM_ERR_INVALID_ARGUMENT;
    if (!forward(n, features, batch)) return LBM_ERR_CUDA;
    const long long m1 = n->m(0, batch);
    k_pred_out<<<nblk(m1 * 4), 256, 0, n->stream>>>(n->pred, m1, n->out_scale, pred);
    return ok(n, cudaGetLastError()) ? finish(n) : LBM_ERR_CUDA;
}

int LBM_WarmNetForward(LBMWarmNet *n, const float *features, int batch, float *pred) {
    if (!valid_batch(n, batch) || !features || !pred) return LBM_ERR_INVALID_ARGUMENT;
    const long long m1 = n->m(0, batch);
    if (!ok(n, cudaMemcpyAsync(n->feat, features, sizeof(float) * m1 * 3, cudaMemcpyHostToDevice,
                               n->stream)))
        return LBM_ERR_CUDA;
    int rc = LBM_WarmNetForwardDevice(n, n->feat, batch, n->pred32);
    if (rc != LBM_OK) return rc;
    if (!ok(n, cudaMemcpyAsync(pred, n->pred32, sizeof(float) * m1 * 4, cudaMemcpyDeviceToHost,
                               n->stream)))
        return LBM_ERR_CUDA;
    return finish(n);
}

int LBM_WarmNetLossGradDevice(LBMWarmNet *n, const float *features, const float *target,
                              int batch, double *loss, float *gradHost) {
    if (!valid_batch(n, batch) || !features || !target) return LBM_ERR_INVALID_ARGUMENT;
    if (!forward(n, features, batch) || !backward(n, target, batch)) return LBM_ERR_CUDA;
    if (loss && !ok(n, cudaMemcpyAsync(loss, n->loss, sizeof(double), cudaMemcpyDeviceToHost,
                                       n->stream)))
        return LBM_ERR_CUDA;
    if (gradHost && !ok(n, cudaMemcpyAsync(gradHost, n->grad, sizeof(float) * n->P,
                                           cudaMemcpyDeviceToHost, n->stream)))
        return LBM_ERR_CUDA;
    const int rc = finish(n);
    if (rc == LBM_OK && loss) *loss /= (double)(n->m(0, batch) * 4);
    return rc;
}

int LBM_WarmNetLossGrad(LBMWarmNet *n, const float *features, const float *target, int batch,
                        double *loss, float *gradHost) {
    if (!valid_batch(n, batch) || !features || !target) return LBM_ERR_INVALID_ARGUMENT;
    const long long m1 = n->m(0, batch);
    if (!ok(n, cudaMemcpyAsync(n->feat, features, sizeof(float) * m1 * 3, cudaMemcpyHostToDevice,
                               n->stream)) ||
        !ok(n, cudaMemcpyAsync(n->target, target, sizeof(float) * m1 * 4, cudaMemcpyHostToDevice,
                               n->stream)))
        return LBM_ERR_CUDA;
    return LBM_WarmNetLossGradDevice(n, n->feat, n->target, batch, loss, gradHost);
}

int LBM_WarmNetTrainStepDevice(LBMWarmNet *n, const float *features, const float *target,
                               int batch, float lr, double *loss) {
    if (!valid_batch(n, batch) || !features || !target || !(lr > 0.f))
        return LBM_ERR_INVALID_ARGUMENT;
    if (!forward(n, features, batch) || !backward(n, target, batch)) return LBM_ERR_CUDA;
    n->adam_t++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float lr_t = lr * sqrtf(1.f - powf(b2, (float)n->adam_t)) /
                       (1.f - powf(b1, (float)n->adam_t));
    if (n->clip > 0.f) {
        if (!ok(n, cudaMemsetAsync(n->sq, 0, sizeof(double), n->stream))) return LBM_ERR_CUDA;
        k_sqnorm<<<148 * 4, 256, 0, n->stream>>>(n->grad, n->P, n->sq);
    }
    k_adam<<<nblk(n->P), 256, 0, n->stream>>>(n->params, n->grad, n->am, n->av, n->P, lr_t, b1, b2,
                                              1e-8f, n->clip, n->sq);
    if (!ok(n, cudaGetLastError())) return LBM_ERR_CUDA;
    n->packed = false;
    if (!pack(n)) return LBM_ERR_CUDA;
    if (loss && !ok(n, cudaMemcpyAsync(loss, n->loss, sizeof(double), cudaMemcpyDeviceToHost,
                                       n->stream)))
        return LBM_ERR_CUDA;
    const int rc = finish(n);
    if (rc == LBM_OK && loss) *loss /= (double)(n->m(0, batch) * 4);
    return rc;
}

int LBM_WarmNetTrainStep(LBMWarmNet *n, const float *features, const float *target, int batch,
                         float lr, double *loss) {
    if (!valid_batch(n, batch) || !features || !target) return LBM_ERR_INVALID_ARGUMENT;
    const long long m1 = n->m(0, batch);
    if (!ok(n, cudaMemcpyAsync(n->feat, features, sizeof(float) * m1 * 3, cudaMemcpyHostToDevice,
                               n->stream)) ||
        !ok(n, cudaMemcpyAsync(n->target, target, sizeof(float) * m1 * 4, cudaMemcpyHostToDevice,
                               n->stream)))
        return LBM_ERR_CUDA;
    return LBM_WarmNetTrainStepDevice(n, n->feat, n->target, batch, lr, loss);
}

void *LBM_WarmNetGetStream(LBMWarmNet *n) { return n ? (void *)n->stream : nullptr; }

int LBM_WarmNetSetGradClip(LBMWarmNet *n, float maxNorm) {
    if (!n || !(maxNorm >= 0.f)) return LBM_ERR_INVALID_ARGUMENT;
    n->clip = maxNorm;
    return LBM_OK;
}

int LBM_WarmNetSetOutputScaling(LBMWarmNet *n, const float *scale4, const float *shift4) {
    if (!n || !scale4 || !shift4) return LBM_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 4; k++) {
        n->out_scale.scale[k] = scale4[k];
        n->out_scale.shift[k] = shift4[k];
    }
    return LBM_OK;
}

int LBM_WarmNetGridFeatures(LBMGrid *grid, int factor, float U, float Re, float *featDev) {
    if (!grid || !grid->impl || factor <= 0 || !featDev) return LBM_ERR_INVALID_ARGUMENT;
    GridImpl &I = *static_cast<GridImpl *>(grid->impl);
    if (I.nx % factor || I.ny % factor || I.nz % factor) return LBM_ERR_INVALID_ARGUMENT;
    const long long m = (long long)(I.nx / factor) * (I.ny / factor) * (I.nz / factor);
    k_grid_features<<<nblk(m), 256, 0, I.stream>>>(I.solid, I.nx, I.ny, I.nz, factor, U, Re,
                                                   featDev);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(I.stream) != cudaSuccess)
        return LBM_ERR_CUDA;
    return LBM_OK;
}

int LBM_WarmNetGridTargets(LBMGrid *grid, int factor, float U, float *targetDev) {
    if (!grid || !grid->impl || factor <= 0 || !targetDev || !(U > 0.f))
        return LBM_ERR_INVALID_ARGUMENT;
    GridImpl &I = *static_cast<GridImpl *>(grid->impl);
    if (I.nx % factor || I.ny % factor || I.nz % factor) return LBM_ERR_INVALID_ARGUMENT;
    const float4 *vel = static_cast<const float4 *>(LBM_GetVelocityBuffer(grid));
    if (!vel) return LBM_ERR_CUDA;
    const long long m = (long long)(I.nx / factor) * (I.ny / factor) * (I.nz / factor);
    k_grid_targets<<<nblk(m), 256, 0, I.stream>>>(vel, I.solid, I.nx, I.ny, I.nz, factor, U,
                                                  targetDev);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(I.stream) != cudaSuccess)
        return LBM_ERR_CUDA;
    return LBM_OK;
}

int LBM_InitializeFromWarmNet(LBMGrid *grid, LBMWarmNet *n, float U, float Re, int flags) {
    if (!grid || !grid->impl || !n || !(U > 0.f) || !(Re > 0.f)) return LBM_ERR_INVALID_ARGUMENT;
    GridImpl &I = *static_cast<GridImpl *>(grid->impl);
    if (I.nx % n->nx || I.nx / n->nx != I.ny / n->ny || I.nx / n->nx != I.nz / n->nz ||
        I.ny % n->ny || I.nz % n->nz)
        return LBM_ERR_INVALID_ARGUMENT;
    const int f = I.nx / n->nx;
    int rc = LBM_WarmNetGridFeatures(grid, f, U, Re, n->feat);
    if (rc != LBM_OK) return rc;
    rc = LBM_WarmNetForwardDevice(n, n->feat, 1, n->pred32);
    if (rc != LBM_OK) return rc;
    float *d = nullptr;
    if (cudaMallocAsync(&d, sizeof(float) * 4 * (size_t)I.n, I.stream) != cudaSuccess)
        return LBM_ERR_OUT_OF_MEMORY;
    k_decode_upsample<<<nblk(I.n), 256, 0, I.stream>>>(n->pred32, n->nx, n->ny, n->nz, f, U,
                                                       I.solid, I.nx, I.ny, I.nz, d, d + I.n,
                                                       (flags & LBM_WARM_UNIFORM_DENSITY) ? 0 : 1);
    bool good = cudaGetLastError() == cudaSuccess;
    if (good && (flags & LBM_WARM_FLUX_CORRECT)) {
        double *sums = nullptr;
        good = cudaMallocAsync(&sums, sizeof(double) * 3 * I.nx, I.stream) == cudaSuccess;
        if (good) {
            k_plane_sums<<<I.nx, 256, 0, I.stream>>>(d, d + I.n, I.solid, I.nx, I.ny, I.nz, sums);
            k_flux_correct<<<nblk(I.n), 256, 0, I.stream>>>(d, d + I.n, I.solid, I.nx, I.ny,
                                                            I.nz, U, sums);
            good = cudaGetLastError() == cudaSuccess;
            cudaFreeAsync(sums, I.stream);
        }
    }
    rc = good && grid_init_from_device(grid, d, d + I.n) ? LBM_OK : LBM_ERR_CUDA;
    cudaFreeAsync(d, I.stream);
    cudaStreamSynchronize(I.stream);
    return rc;
}

}  // extern "C"
