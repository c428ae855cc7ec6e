// Super-resolution upscaling of the velocity field (the reference's SR_*
// path: simulation/src/superres.c, simulation/shaders/superres_upscale.comp)
// as one persistent tensor-core kernel.
//
// Per coarse cell (superres_upscale.comp:160-216): the 3x3x3 neighbourhood of
// vec4 (ux, uy, uz, rho), clamped at the grid faces and normalised by the
// channel mean and std, is the 108-wide input of an MLP 108 -> 128 -> 128 ->
// 128 -> 32 with ReLU after the first three layers; its 32 outputs correct a
// trilinear estimate ("skip") of the 8 fine cells x 4 channels; skip +
// correction is denormalised and written to the fine field.
//
// Layout on the device: each CTA keeps the four weight matrices in shared
// memory as BF16 (K-major, no-swizzle core matrices, K padded to 128 with
// zeros) for its whole life and walks tiles of 128 coarse cells.  Per tile
// its 128 threads gather one cell each into the A operand (BF16, row = cell),
// one thread issues the layer's tcgen05.mma (M = 128, N = 128 or 32, K = 16
// per instruction, FP32 accumulator in tensor memory), and the epilogue --
// thread t reads accumulator row t, adds the bias, applies ReLU and writes
// the BF16 activations back into A -- feeds the next layer.  The last
// epilogue adds the skip, computed in FP32 from the coarse field exactly as
// the shader does, and writes the 8 fine cells.  No TMA and no multicast.
//
// Every wait is bounded; when one gives up the CTA stops issuing, drains
// the MMAs it committed (bounded), writes no output, sets the error word and
// frees its tensor memory.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <new>
#include <vector>

#include <cuda_bf16.h>

#include "lbm_internal.h"
#include "tc05.cuh"

namespace lbm {
namespace sr {

constexpr int H = 128;        // hidden width
constexpr int KIN = 108;      // 27 cells x 4 channels
constexpr int NOUT = 32;      // 8 fine cells x 4 channels
constexpr int KS = 128;       // K extent of every operand in shared memory
constexpr int NWEIGHTS = H + H * KIN + H + H * H + H + H * H + NOUT + NOUT * H;  // 51,104
constexpr uint32_t WAIT_LIMIT = 1u << 24;

// bytes of one operand of `rows` rows in shared memory
constexpr int op_bytes(int rows) { return rows * KS * 2; }
constexpr int OFF_W0 = 0;
constexpr int OFF_W1 = OFF_W0 + op_bytes(H);
constexpr int OFF_W2 = OFF_W1 + op_bytes(H);
constexpr int OFF_W3 = OFF_W2 + op_bytes(H);
constexpr int OFF_A = OFF_W3 + op_bytes(NOUT);
constexpr int OFF_BIAS = OFF_A + op_bytes(H);           // b0, b1, b2 (128 each), b3 (32)
constexpr int OFF_BAR = OFF_BIAS + (3 * H + NOUT) * 4;  // one mbarrier
constexpr int OFF_TSLOT = OFF_BAR + 8;
constexpr int SMEM_BYTES = OFF_TSLOT + 8 + 1024;        // + alignment slack
constexpr int WEIGHT_BYTES = OFF_A;                      // the packed weights in global memory

// byte offset of element (row r, k) in a K-major no-swizzle operand whose
// 8-row groups are KS / 8 core matrices of 8 x 16 bytes apart
__host__ __device__ constexpr int elem_off(int r, int k) {
    return ((r >> 3) * (KS / 8) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

struct Params {
    const float4 *coarse;
    float4 *fine;
    const uint8_t *weights;   // WEIGHT_BYTES, the packed BF16 operands
    const float *bias;        // 3 * H + NOUT
    float4 mean, stdv;
    int cx, cy, cz;
    long long ncells;
    int *err;
};

__device__ __forceinline__ float4 norm4(float4 v, float4 m, float4 s) {
    // (v - normMean) / normStd, componentwise (superres_upscale.comp:58-60)
    return make_float4((v.x - m.x) / s.x, (v.y - m.y) / s.y, (v.z - m.z) / s.z,
                       (v.w - m.w) / s.w);
}

__device__ __forceinline__ float4 sample(const Params &p, int x, int y, int z) {
    x = min(max(x, 0), p.cx - 1);
    y = min(max(y, 0), p.cy - 1);
    z = min(max(z, 0), p.cz - 1);
    return __ldg(p.coarse + (long long)x + (long long)p.cx * ((long long)y + (long long)p.cy * z));
}

__global__ void __launch_bounds__(128, 1) k_superres(const Params p) {
    extern __shared__ __align__(1024) uint8_t sm_raw[];
    uint8_t *sm = sm_raw + ((1024 - (reinterpret_cast<uintptr_t>(sm_raw) & 1023)) & 1023);
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t bar = tc::smem_addr(sm + OFF_BAR);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + OFF_TSLOT);
    float *bias = reinterpret_cast<float *>(sm + OFF_BIAS);

    // weights and biases into shared memory, once per CTA
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(p.weights);
        uint4 *dst = reinterpret_cast<uint4 *>(sm);
        for (int k = tid; k < WEIGHT_BYTES / 16; k += 128) dst[k] = __ldg(src + k);
        for (int k = tid; k < 3 * H + NOUT; k += 128) bias[k] = __ldg(p.bias + k);
    }
    if (warp == 0) {
        tc::tmem_alloc(tc::smem_addr(tslot), 128);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        tc::mbar_init_fence();
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t a_addr = tc::smem_addr(sm + OFF_A);
    const uint32_t w_addr[4] = {tc::smem_addr(sm + OFF_W0), tc::smem_addr(sm + OFF_W1),
                                tc::smem_addr(sm + OFF_W2), tc::smem_addr(sm + OFF_W3)};
    uint8_t *A = sm + OFF_A;
    uint32_t phase = 0;  // completed commits on the barrier
    bool ok = true;      // block-uniform

    // one layer: K / 16 MMAs of the A operand against weights w, then wait
    auto layer = [&](int w, int ksteps, int n) -> bool {
        tc::fence_async_smem();  // A written by the generic proxy
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t idesc = tc::idesc_bf16_f32(128, n);
            for (int j = 0; j < ksteps; j++) {
                const uint64_t ad = tc::kmajor_desc(a_addr + j * 256, 128, KS * 16);
                const uint64_t bd = tc::kmajor_desc(w_addr[w] + j * 256, 128, KS * 16);
                tc::mma_bf16(tmem, ad, bd, idesc, j != 0);
            }
            tc::mma_commit(bar);
        }
        const bool got = tc::mbar_wait(bar, phase & 1u, WAIT_LIMIT);
        phase++;
        if (!__syncthreads_and(got)) {
            // drain: a second bounded wait for the same commit
            const bool again = tc::mbar_wait(bar, (phase - 1) & 1u, WAIT_LIMIT);
            const int drained = __syncthreads_and(again);
            if (tid == 0) atomicOr(p.err, drained ? 1 : 3);
            return false;
        }
        tc::fence_after_sync();
        return true;
    };
    // accumulator row tid, columns [c, c + 8)
    auto acc8 = [&](int c, float (&v)[8]) {
        tc::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
        tc::tmem_wait_ld();
    };
    // bias + ReLU of accumulator row tid into A row tid (BF16)
    auto hidden_epilogue = [&](const float *b) {
#pragma unroll 1
        for (int c = 0; c < H; c += 8) {
            float v[8];
            acc8(c, v);
            __align__(16) __nv_bfloat16 h[8];
#pragma unroll
            for (int i = 0; i < 8; i++) h[i] = __float2bfloat16_rn(fmaxf(v[i] + b[c + i], 0.0f));
            *reinterpret_cast<uint4 *>(A + elem_off(tid, c)) = *reinterpret_cast<const uint4 *>(h);
        }
    };

    const long long ntiles = (p.ncells + 127) / 128;
    for (long long tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x) {
        const long long m = tile * 128 + tid;
        const bool valid = m < p.ncells;
        int x = 0, y = 0, z = 0;
        if (valid) {
            x = (int)(m % p.cx);
            const long long r = m / p.cx;
            y = (int)(r % p.cy);
            z = (int)(r / p.cy);
        }
        // gatherPatch (:76-92): [dz][dy][dx][channel], x fastest, as BF16
        {
            __align__(16) __nv_bfloat16 row[KS];
            int k = 0;
#pragma unroll
            for (int dz = -1; dz <= 1; dz++)
#pragma unroll
                for (int dy = -1; dy <= 1; dy++)
#pragma unroll
                    for (int dx = -1; dx <= 1; dx++) {
                        const float4 v = valid ? norm4(sample(p, x + dx, y + dy, z + dz), p.mean,
                                                       p.stdv)
                                               : make_float4(0.f, 0.f, 0.f, 0.f);
                        row[k++] = __float2bfloat16_rn(v.x);
                        row[k++] = __float2bfloat16_rn(v.y);
                        row[k++] = __float2bfloat16_rn(v.z);
                        row[k++] = __float2bfloat16_rn(v.w);
                    }
#pragma unroll
            for (; k < KS; k++) row[k] = __float2bfloat16_rn(0.0f);
#pragma unroll
            for (int c = 0; c < KS; c += 8)
                *reinterpret_cast<uint4 *>(A + elem_off(tid, c)) =
                    *reinterpret_cast<const uint4 *>(row + c);
        }
        // the MLP (:168-191): three hidden layers, then 32 outputs
        if (!(ok = layer(0, 7, H))) break;   // K = 108 padded to 112
        hidden_epilogue(bias);
        if (!(ok = layer(1, 8, H))) break;
        hidden_epilogue(bias + H);
        if (!(ok = layer(2, 8, H))) break;
        hidden_epilogue(bias + 2 * H);
        if (!(ok = layer(3, 8, NOUT))) break;
        float corr[NOUT];
#pragma unroll
        for (int c = 0; c < NOUT; c += 8) {
            float v[8];
            acc8(c, v);
#pragma unroll
            for (int i = 0; i < 8; i++) corr[c + i] = v[i] + bias[3 * H + c + i];
        }
        tc::fence_before_sync();
        if (valid) {
            // trilinearSkip (:95-129) in FP32 from the normalised coarse
            // field: sub-cell (dx, dy, dz) interpolates the centre cell and
            // its +1 neighbours with weights (1 - f) and f, f = 0.25 + 0.5 d
            float4 pc[8];
#pragma unroll
            for (int c = 0; c < 8; c++)
                pc[c] = norm4(sample(p, x + (c & 1), y + ((c >> 1) & 1), z + (c >> 2)), p.mean,
                              p.stdv);
#pragma unroll
            for (int s = 0; s < 8; s++) {
                const int dx = s & 1, dy = (s >> 1) & 1, dz = s >> 2;
                const float fx = 0.25f + 0.5f * (float)dx, fy = 0.25f + 0.5f * (float)dy,
                            fz = 0.25f + 0.5f * (float)dz;
                float4 val = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int c = 0; c < 8; c++) {
                    const int ccx = c & 1, ccy = (c >> 1) & 1, ccz = c >> 2;
                    const float wz = ccz ? fz : 1.0f - fz;
                    const float wy = ccy ? fy : 1.0f - fy;
                    const float wx = ccx ? fx : 1.0f - fx;
                    const float w = wz * wy * wx;
                    val.x = val.x + w * pc[c].x;
                    val.y = val.y + w * pc[c].y;
                    val.z = val.z + w * pc[c].z;
                    val.w = val.w + w * pc[c].w;
                }
                // (skip + correction) * std + mean (:193-214)
                const float4 o = make_float4((val.x + corr[4 * s]) * p.stdv.x + p.mean.x,
                                             (val.y + corr[4 * s + 1]) * p.stdv.y + p.mean.y,
                                             (val.z + corr[4 * s + 2]) * p.stdv.z + p.mean.z,
                                             (val.w + corr[4 * s + 3]) * p.stdv.w + p.mean.w);
                const long long fxi = 2 * x + dx, fyi = 2 * y + dy, fzi = 2 * z + dz;
                const long long fcx = 2ll * p.cx, fcy = 2ll * p.cy;
                p.fine[fxi + fcx * (fyi + fcy * fzi)] = o;
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 128);
}

// The LTWS parameter file of the reference (superres.c:43-101): magic
// "LTWS", version, parameter count, then per parameter its rank, its
// extents and its FP32 values; the values of all parameters concatenated.
bool read_ltws(const char *path, std::vector<float> &out) {
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    uint32_t hdr[3];
    bool good = fread(hdr, 4, 3, f) == 3 && hdr[0] == 0x4C545753u;
    for (uint32_t k = 0; good && k < hdr[2]; k++) {
        uint32_t rank = 0;
        good = fread(&rank, 4, 1, f) == 1 && rank <= 8;
        long long numel = 1;
        for (uint32_t d = 0; good && d < rank; d++) {
            uint32_t e = 0;
            good = fread(&e, 4, 1, f) == 1;
            numel *= e;
        }
        good = good && numel >= 0 && numel <= (1ll << 28);
        if (good) {
            const size_t at = out.size();
            out.resize(at + (size_t)numel);
            good = fread(out.data() + at, 4, (size_t)numel, f) == (size_t)numel;
        }
    }
    fclose(f);
    return good;
}

}  // namespace sr
}  // namespace lbm

using namespace lbm;

struct LBMSuperRes {
    int cx = 0, cy = 0, cz = 0;
    float mean[4] = {0, 0, 0, 0}, stdv[4] = {1, 1, 1, 1};
    uint8_t *weights = nullptr;
    float *bias = nullptr;
    float4 *fine = nullptr;
    int *err = nullptr;
    int grid = 0;
};

extern "C" {

LBMSuperRes *LBM_SuperResCreateFromArrays(int coarseX, int coarseY, int coarseZ,
                                          const float *w, long long count, const float *mean,
                                          const float *stdv) {
    using namespace sr;
    if (coarseX <= 0 || coarseY <= 0 || coarseZ <= 0 || !w || count != NWEIGHTS || !mean ||
        !stdv)
        return nullptr;
    LBMSuperRes *r = new (std::nothrow) LBMSuperRes();
    if (!r) return nullptr;
    r->cx = coarseX;
    r->cy = coarseY;
    r->cz = coarseZ;
    for (int c = 0; c < 4; c++) r->mean[c] = mean[c], r->stdv[c] = stdv[c];
    // the file's order (superres.c:130-166): b0, W0 [128][108], b1, W1, b2,
    // W2, b3, W3 [32][128]; each W packed as the K-major BF16 operand
    std::vector<uint8_t> packed(WEIGHT_BYTES, 0);
    std::vector<float> bias(3 * H + NOUT);
    auto put = [&](int base, const float *W, int rows, int k) {
        for (int n = 0; n < rows; n++)
            for (int j = 0; j < k; j++) {
                const __nv_bfloat16 b = __float2bfloat16_rn(W[(long long)n * k + j]);
                memcpy(&packed[base + elem_off(n, j)], &b, 2);
            }
    };
    long long off = 0;
    memcpy(&bias[0], w + off, H * 4), off += H;
    put(OFF_W0, w + off, H, KIN), off += (long long)H * KIN;
    memcpy(&bias[H], w + off, H * 4), off += H;
    put(OFF_W1, w + off, H, H), off += (long long)H * H;
    memcpy(&bias[2 * H], w + off, H * 4), off += H;
    put(OFF_W2, w + off, H, H), off += (long long)H * H;
    memcpy(&bias[3 * H], w + off, NOUT * 4), off += NOUT;
    put(OFF_W3, w + off, NOUT, H), off += (long long)NOUT * H;
    const long long fine = 8ll * coarseX * coarseY * coarseZ;
    bool good = cudaMalloc(&r->weights, WEIGHT_BYTES) == cudaSuccess &&
                cudaMalloc(&r->bias, bias.size() * 4) == cudaSuccess &&
                cudaMalloc(&r->fine, (size_t)fine * sizeof(float4)) == cudaSuccess &&
                cudaMalloc(&r->err, sizeof(int)) == cudaSuccess;
    good = good && cudaMemcpy(r->weights, packed.data(), WEIGHT_BYTES, cudaMemcpyHostToDevice) ==
                       cudaSuccess;
    good = good &&
           cudaMemcpy(r->bias, bias.data(), bias.size() * 4, cudaMemcpyHostToDevice) == cudaSuccess;
    good = good && cudaMemset(r->err, 0, sizeof(int)) == cudaSuccess;
    good = good && cudaFuncSetAttribute(k_superres, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        SMEM_BYTES) == cudaSuccess;
    int dev = 0, sms = 0;
    good = good && cudaGetDevice(&dev) == cudaSuccess &&
           cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess;
    if (!good) {
        cudaGetLastError();
        LBM_SuperResFree(r);
        return nullptr;
    }
    const long long tiles = ((long long)coarseX * coarseY * coarseZ + 127) / 128;
    r->grid = (int)(tiles < sms ? tiles : sms);
    return r;
}

LBMSuperRes *LBM_SuperResCreate(int coarseX, int coarseY, int coarseZ, const char *weightsPath,
                                const char *normPath) {
    if (!weightsPath) return nullptr;
    std::vector<float> w;
    if (!sr::read_ltws(weightsPath, w)) {
        fprintf(stderr, "LBM_SuperResCreate: cannot read LTWS weights from %s\n", weightsPath);
        return nullptr;
    }
    float mean[4] = {0, 0, 0, 0}, stdv[4] = {1, 1, 1, 1};
    if (normPath) {
        FILE *f = fopen(normPath, "rb");
        if (f) {
            float v[8];
            if (fread(v, 4, 8, f) == 8) {
                for (int c = 0; c < 4; c++) mean[c] = v[c], stdv[c] = v[4 + c];
            }
            fclose(f);
        }
    }
    return LBM_SuperResCreateFromArrays(coarseX, coarseY, coarseZ, w.data(), (long long)w.size(),
                                        mean, stdv);
}

void LBM_SuperResFree(LBMSuperRes *r) {
    if (!r) return;
    cudaFree(r->weights);
    cudaFree(r->bias);
    cudaFree(r->fine);
    cudaFree(r->err);
    delete r;
}

int LBM_SuperResUpscale(LBMSuperRes *r, const float *coarse, void *stream) {
    if (!r || !coarse) return LBM_ERR_INVALID_ARGUMENT;
    sr::Params p;
    p.coarse = reinterpret_cast<const float4 *>(coarse);
    p.fine = r->fine;
    p.weights = r->weights;
    p.bias = r->bias;
    p.mean = make_float4(r->mean[0], r->mean[1], r->mean[2], r->mean[3]);
    p.stdv = make_float4(r->stdv[0], r->stdv[1], r->stdv[2], r->stdv[3]);
    p.cx = r->cx;
    p.cy = r->cy;
    p.cz = r->cz;
    p.ncells = (long long)r->cx * r->cy * r->cz;
    p.err = r->err;
    void *args[] = {&p};
    return cudaLaunchKernel((const void *)sr::k_superres, dim3(r->grid), dim3(128), args,
                            sr::SMEM_BYTES, static_cast<cudaStream_t>(stream)) == cudaSuccess
               ? LBM_OK
               : LBM_ERR_CUDA;
}

const float *LBM_SuperResGetFineVelocity(LBMSuperRes *r) {
    return r ? reinterpret_cast<const float *>(r->fine) : nullptr;
}

void LBM_SuperResGetFineSize(LBMSuperRes *r, int *fx, int *fy, int *fz) {
    if (!r) return;
    if (fx) *fx = 2 * r->cx;
    if (fy) *fy = 2 * r->cy;
    if (fz) *fz = 2 * r->cz;
}

int LBM_SuperResCopyFine(LBMSuperRes *r, float *host) {
    if (!r || !host) return LBM_ERR_INVALID_ARGUMENT;
    if (cudaDeviceSynchronize() != cudaSuccess) return LBM_ERR_CUDA;
    int e = 0;
    if (cudaMemcpy(&e, r->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return LBM_ERR_CUDA;
    if (e) {
        cudaMemset(r->err, 0, sizeof(int));
        return LBM_ERR_TIMEOUT;
    }
    const size_t bytes = 8ull * r->cx * r->cy * r->cz * sizeof(float4);
    return cudaMemcpy(host, r->fine, bytes, cudaMemcpyDeviceToHost) == cudaSuccess ? LBM_OK
                                                                                   : LBM_ERR_CUDA;
}

}  // extern "C"
