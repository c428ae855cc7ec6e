// Storage-format dispatch of the step kernels.  The kernels are
// instantiated in lbm_step_{f32,f64,f16,bf16}.cu and lbm_step_fast_*.cu,
// each of which exports a StepOps table; this unit sees only the tables.
#include <cudaTypedefs.h>
#include <stdlib.h>

#include "lbm_internal.h"

namespace lbm {

static const StepOps *ops_of(int storage) {
    switch (storage) {
        case LBM_STORAGE_FP32: return &step_ops_f32;
        case LBM_STORAGE_FP64: return &step_ops_f64;
        case LBM_STORAGE_FP16: return &step_ops_f16;
        case LBM_STORAGE_BF16: return &step_ops_bf16;
        default: return nullptr;
    }
}

static const StepOps *fast_ops_of(int storage) {
    switch (storage) {
        case LBM_STORAGE_FP32: return &step_ops_fast_f32;
        case LBM_STORAGE_FP16: return &step_ops_fast_f16;
        case LBM_STORAGE_BF16: return &step_ops_fast_bf16;
        default: return nullptr;
    }
}

#define LBM_DISPATCH(storage, CALL)                   \
    do {                                              \
        const StepOps *ops_ = ops_of(storage);        \
        if (!ops_) return cudaErrorInvalidValue;      \
        return ops_->CALL;                            \
    } while (0)

cudaError_t launch_step(const GridImpl &g, const StepArgs &a, bool fused, int op, bool smag,
                        bool fast_arith, cudaStream_t s) {
    if (fast_arith && g.storage != LBM_STORAGE_FP64) {
        const StepOps *f = fast_ops_of(g.storage);
        if (!f) return cudaErrorInvalidValue;
        return f->step(g, a, fused, op, smag, s);
    }
    LBM_DISPATCH(g.storage, step(g, a, fused, op, smag, s));
}

cudaError_t launch_step_batch(int storage, const BatchLaunchParams &p, int set, cudaStream_t s) {
    LBM_DISPATCH(storage, batch(p, set, s));
}

cudaError_t launch_step_batch_pair(int storage, const BatchPairParams &p, int set,
                                   cudaStream_t s) {
    LBM_DISPATCH(storage, batch_pair(p, set, s));
}

// the driver's tensor-map encoder, looked up once through the runtime
static PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// Each population buffer as a rank-4 tensor (x, y, z, direction) with boxes
// of tma_box_x x TMA_BOX_Y x 1 x 1 elements, zero fill outside the grid.
void setup_tma(GridImpl &g, bool force) {
    g.tma = false;
    const char *env = getenv("LBM_TMA");
    if (!force && !(env && atoi(env) == 1)) return;
    CUtensorMapDataType dt;
    switch (g.storage) {
        case LBM_STORAGE_FP32: dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32; break;
        case LBM_STORAGE_FP16: dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT16; break;
        case LBM_STORAGE_BF16: dt = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16; break;
        default: return;
    }
    const size_t es = g.elem;
    if (((size_t)g.nx * es) % 16 != 0 || !g.pop[0] || !g.pop[1]) return;
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tma_encoder();
    if (!enc) return;
    const cuuint64_t dims[4] = {(cuuint64_t)g.nx, (cuuint64_t)g.ny, (cuuint64_t)g.nz, 19};
    const cuuint64_t strides[3] = {(cuuint64_t)g.nx * es, (cuuint64_t)g.nx * g.ny * es,
                                   (cuuint64_t)g.n * es};
    const cuuint32_t box[4] = {(cuuint32_t)tma_box_x(es), (cuuint32_t)TMA_BOX_Y, 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    for (int k = 0; k < 2; k++) {
        if (enc(&g.tmap[k], dt, 4, g.pop[k], dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return;
    }
    const StepOps *ops = ops_of(g.storage), *fops = fast_ops_of(g.storage);
    cudaError_t e = (ops && fops) ? ops->tma_prepare() : cudaErrorNotSupported;
    if (e == cudaSuccess) e = fops->tma_prepare();
    if (e != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    g.tma = true;
}

static StepArgs stream_args(const GridImpl &g, const void *src, void *dst, int periodic) {
    StepArgs a{};
    a.src = src;
    a.dst = dst;
    a.flags = g.flags;
    a.slot = g.slot;
    a.bmask = g.links.bmask;
    a.bfirst = g.links.bfirst;
    a.lq = g.links.lq;
    a.nx = g.nx;
    a.ny = g.ny;
    a.nz = g.nz;
    a.n = g.n;
    a.periodic = periodic;
    return a;
}

cudaError_t launch_stream_only(const GridImpl &g, const void *src, void *dst, int periodic,
                               cudaStream_t s) {
    StepArgs a = stream_args(g, src, dst, periodic);
    LBM_DISPATCH(g.storage, stream_only(g, a, s));
}

cudaError_t launch_velocity(const GridImpl &g, const void *src, int kind, int periodic,
                            float inX, float inY, float inZ, float4 *vel, double4 *vel64,
                            cudaStream_t s) {
    StepArgs a = stream_args(g, src, nullptr, periodic);
    a.inX = inX;
    a.inY = inY;
    a.inZ = inZ;
    LBM_DISPATCH(g.storage, velocity(g, a, kind, vel, vel64, s));
}

cudaError_t launch_init_uniform(const GridImpl &g, void *a, void *b, float ux, float uy,
                                float uz, cudaStream_t s) {
    LBM_DISPATCH(g.storage, init_uniform(g, a, b, ux, uy, uz, s));
}

cudaError_t launch_init_field(const GridImpl &g, void *a, void *b, const float *rho,
                              const float *u, cudaStream_t s) {
    LBM_DISPATCH(g.storage, init_field(g, a, b, rho, u, s));
}

cudaError_t launch_export_aos(const GridImpl &g, const void *src, void *dst, bool as_double,
                              cudaStream_t s) {
    LBM_DISPATCH(g.storage, export_aos(g, src, dst, as_double, s));
}

cudaError_t launch_import_aos(const GridImpl &g, const float *src, void *dst, cudaStream_t s) {
    LBM_DISPATCH(g.storage, import_aos(g, src, dst, s));
}

cudaError_t launch_mass_momentum(const GridImpl &g, const void *f, double *out4, cudaStream_t s) {
    LBM_DISPATCH(g.storage, mass_momentum(g, f, out4, s));
}

}  // namespace lbm
