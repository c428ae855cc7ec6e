// C ABI of the solver (include/lattice_lbm.h): grid lifetime, the
// population-buffer state machine, geometry set-up, readbacks.
//
// Reference behaviour being replaced: simulation/src/lbm.c (all LBM_*
// functions) and simulation/src/vti_export.c (writeVTI).
//
// State machine.  The reference keeps two population arrays, f (post
// stream) and f_new (post collision), and runs collide then stream every
// step.  This library runs ONE fused stream+collide kernel per step over
// two ping-pong buffers, so after a step only the post-collision field g
// is stored and the post-stream f is implicit (f = Stream(g)).  Whatever
// needs the reference's f (population readback, geometry edits, the FP64
// mass sum) first materialises it with a stream-only kernel.  The
// velocity field of a step is likewise derived on demand from the step's
// input buffer, which stays intact until the next step, so the hot loop
// moves only the 2 x 19 populations per cell.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <new>
#include <vector>

#include "lbm_internal.h"

using namespace lbm;

struct LBMParticles {
    int n = 0;
    uint32_t seed = 0;
    LBMParticle *dev = nullptr;
    cudaEvent_t done = nullptr;  // recorded after each step on the grid's stream
};

namespace {

inline GridImpl *IMPL(LBMGrid *g) { return g ? static_cast<GridImpl *>(g->impl) : nullptr; }

inline bool ok(LBMGrid *g, cudaError_t e) {
    if (e != cudaSuccess) {
        if (g) g->lastError = (e == cudaErrorMemoryAllocation) ? LBM_ERR_OUT_OF_MEMORY : LBM_ERR_CUDA;
        return false;
    }
    return true;
}

size_t elem_size(int storage) {
    switch (storage) {
        case LBM_STORAGE_FP32: return 4;
        case LBM_STORAGE_FP64: return 8;
        case LBM_STORAGE_FP16:
        case LBM_STORAGE_BF16: return 2;
        default: return 0;
    }
}

// Step launch shape.  FP32 / FP16 / BF16 grids with an even NX run the
// paired kernel (two cells per thread, cpt = 2; 128-thread blocks of 32 x 4
// threads, 64 x 4 cells).  Otherwise (FP64, odd NX, or LBM_CPT=1): 256-thread
// blocks of 32 x 8 cells (a warp spans 32 consecutive x), at least 4 blocks
// resident per SM (<= 64 registers), measured on B200 at 256x128x128 against
// 64x4 / 128x2 / 256x1 shapes and an unconstrained register budget.
// LBM_BLOCK=<bx>x<by>, LBM_MINB=1|4, LBM_CPT=1|2 and LBM_PBX=32|64|128
// (threads along x of a paired block) override it.
void default_block(GridImpl &I) {
    I.bx = 32;
    I.by = 8;
    I.cpt = 2;
    I.pbx = 32;
    I.minb = 4;
    const char *cenv = getenv("LBM_CPT");
    if (cenv) I.cpt = atoi(cenv) == 2 ? 2 : 1;
    const char *penv = getenv("LBM_PBX");
    if (penv) {
        const int v = atoi(penv);
        if (v == 32 || v == 64 || v == 128) I.pbx = v;
    }
    const char *menv = getenv("LBM_MINB");
    if (menv) I.minb = atoi(menv) == 1 ? 1 : 4;
    const char *env = getenv("LBM_BLOCK");
    if (env) {
        int a = 0, b = 0;
        if (sscanf(env, "%dx%d", &a, &b) == 2 && a > 0 && b > 0 && a * b <= 256 && a % 32 == 0) {
            I.bx = a;
            I.by = b;
        }
    }
}

__global__ void k_fill_vel(float4 *v, double4 *v64, long long n, float4 val) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    v[i] = val;
    if (v64) v64[i] = make_double4(val.x, val.y, val.z, val.w);
}

__global__ void k_vel_from_field(float4 *v, double4 *v64, long long n, const float *rho,
                                 const float *u) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    v[i] = make_float4(u[3 * i], u[3 * i + 1], u[3 * i + 2], rho[i]);
    if (v64) v64[i] = make_double4(u[3 * i], u[3 * i + 1], u[3 * i + 2], rho[i]);
}

void drop_graph(GridImpl &I) {
    for (int k = 0; k < 2; k++) {
        if (I.graph[k]) {
            cudaGraphExecDestroy(I.graph[k]);
            I.graph[k] = nullptr;
        }
    }
}

// Derive the velocity field of the last step from its input buffer.
bool ensure_vel(LBMGrid *grid) {
    GridImpl &I = *IMPL(grid);
    if (I.vel_valid) return true;
    if (!ok(grid, launch_velocity(I, I.pop[I.vin], I.vin_kind, I.vin_periodic, I.vin_inlet[0],
                                  I.vin_inlet[1], I.vin_inlet[2], I.vel, I.vel64, I.stream)))
        return false;
    I.vel_valid = true;
    return true;
}

// Make the post-stream populations explicit in buffer fbuf.
bool materialize_f(LBMGrid *grid) {
    GridImpl &I = *IMPL(grid);
    if (I.fbuf >= 0) return true;
    if (!ensure_vel(grid)) return false;
    const int dst = 1 - I.gbuf;
    if (!ok(grid, launch_stream_only(I, I.pop[I.gbuf], I.pop[dst], I.stream_periodic, I.stream)))
        return false;
    I.fbuf = dst;
    return true;
}

StepArgs step_args(LBMGrid *grid, GridImpl &I, float inX, float inY, float inZ) {
    StepArgs a{};
    a.flags = I.flags;
    a.slot = I.slot;
    a.bmask = I.links.bmask;
    a.bfirst = I.links.bfirst;
    a.lq = I.links.lq;
    a.nx = I.nx;
    a.ny = I.ny;
    a.nz = I.nz;
    a.n = I.n;
    a.tau = grid->tau;
    // lbm_collide.comp:480-486 in each arithmetic precision
    a.omega = 1.0f / grid->tau;
    a.smag18 = 18.0f * (grid->smagorinskyCs * grid->smagorinskyCs);
    a.omega_d = 1.0 / (double)grid->tau;
    a.smag18_d = 18.0 * ((double)grid->smagorinskyCs * (double)grid->smagorinskyCs);
    a.inX = inX;
    a.inY = inY;
    a.inZ = inZ;
    a.guard = I.guard;
    a.err = I.err_flag;
    return a;
}

int op_of(LBMGrid *grid) {
    // lbm_collide.comp:488, :544, :618 -- regularized wins over MRT
    if (grid->useRegularized == 1) return OP_REG;
    if (grid->useMRT == 1) return OP_MRT;
    return OP_BGK;
}

// Enqueue one step; updates the state machine.
bool enqueue_step(LBMGrid *grid, float inX, float inY, float inZ) {
    GridImpl &I = *IMPL(grid);
    StepArgs a = step_args(grid, I, inX, inY, inZ);
    const int op = op_of(grid);
    const bool smag = grid->useSmagorinsky == 1;
    if (I.fbuf >= 0) {
        a.src = I.pop[I.fbuf];
        a.dst = I.pop[I.gbuf];
        a.periodic = I.stream_periodic;
        if (!ok(grid, launch_step(I, a, false, op, smag, grid->arithmetic == LBM_ARITH_FAST,
                                  I.stream)))
            return false;
        I.vin = I.fbuf;
        I.vin_kind = IN_EXPLICIT_F;
        I.fbuf = -1;
    } else {
        const int src = I.gbuf, dst = 1 - I.gbuf;
        a.src = I.pop[src];
        a.dst = I.pop[dst];
        a.periodic = I.stream_periodic;
        if (!ok(grid, launch_step(I, a, true, op, smag, grid->arithmetic == LBM_ARITH_FAST,
                                  I.stream)))
            return false;
        I.vin = src;
        I.vin_kind = IN_POST_COLLISION;
        I.vin_periodic = I.stream_periodic;
        I.gbuf = dst;
    }
    I.vin_inlet[0] = inX;
    I.vin_inlet[1] = inY;
    I.vin_inlet[2] = inZ;
    I.vel_valid = false;
    I.stream_periodic = grid->periodicYZ;
    return true;
}

// Geometry edits need the reference's explicit f and velocity, and a
// transient dense q table.
float *begin_geometry(LBMGrid *grid, bool load_links) {
    GridImpl &I = *IMPL(grid);
    drop_graph(I);
    if (I.initialized) {
        if (!ensure_vel(grid) || !materialize_f(grid)) return nullptr;
    }
    float *qd = nullptr;
    if (!ok(grid, cudaMallocAsync(&qd, sizeof(float) * 19 * (size_t)I.n, I.stream))) return nullptr;
    if (load_links) {
        if (!ok(grid, geo_links_to_dense(I, qd, I.stream))) {
            cudaFreeAsync(qd, I.stream);
            return nullptr;
        }
    }
    return qd;
}

void end_geometry(LBMGrid *grid, float *qd, bool launched_ok) {
    GridImpl &I = *IMPL(grid);
    if (launched_ok) ok(grid, geo_compact(I, qd, I.stream));
    cudaFreeAsync(qd, I.stream);
    ok(grid, cudaStreamSynchronize(I.stream));
}

bool sync(LBMGrid *grid) { return ok(grid, cudaStreamSynchronize(IMPL(grid)->stream)); }

}  // namespace

namespace lbm {
StepArgs grid_step_args(LBMGrid *grid, float inX, float inY, float inZ) {
    return step_args(grid, *IMPL(grid), inX, inY, inZ);
}
int grid_op(LBMGrid *grid) { return op_of(grid); }
bool grid_enqueue_step(LBMGrid *grid, float inX, float inY, float inZ) {
    return enqueue_step(grid, inX, inY, inZ);
}
bool grid_ok(LBMGrid *grid, cudaError_t e) { return ok(grid, e); }
bool grid_ensure_velocity(LBMGrid *grid) { return ensure_vel(grid); }
void grid_note_fused_steps(LBMGrid *grid, int k, float inX, float inY, float inZ) {
    GridImpl &I = *IMPL(grid);
    if (k <= 0) return;
    // k fused steps from buffer gbuf: the last one read 1 - final gbuf
    I.gbuf ^= (k & 1);
    I.vin = 1 - I.gbuf;
    I.vin_kind = IN_POST_COLLISION;
    I.vin_periodic = I.stream_periodic;
    I.vin_inlet[0] = inX;
    I.vin_inlet[1] = inY;
    I.vin_inlet[2] = inZ;
    I.vel_valid = false;
    I.stream_periodic = grid->periodicYZ;
}
}  // namespace lbm

extern "C" {

const char *LBM_GetErrorString(int code) {
    switch (code) {
        case LBM_OK: return "ok";
        case LBM_ERR_INVALID_ARGUMENT: return "invalid argument";
        case LBM_ERR_OUT_OF_MEMORY: return "out of device memory";
        case LBM_ERR_CUDA: return "CUDA error";
        case LBM_ERR_NOT_INITIALIZED: return "not initialized";
        case LBM_ERR_UNSUPPORTED: return "unsupported";
        case LBM_ERR_DIVERGED: return "diverged";
        case LBM_ERR_TIMEOUT: return "timeout";
        default: return "unknown error";
    }
}

int LBM_GetLastError(LBMGrid *grid) { return grid ? grid->lastError : LBM_ERR_INVALID_ARGUMENT; }

LBMGrid *LBM_CreateEx(int sizeX, int sizeY, int sizeZ, float viscosity, int storage) {
    if (sizeX <= 0 || sizeY <= 0 || sizeZ <= 0) return nullptr;
    const long long n = (long long)sizeX * sizeY * sizeZ;
    if (n > 0x7fffffffLL || elem_size(storage) == 0) return nullptr;
    LBMGrid *grid = (LBMGrid *)calloc(1, sizeof(LBMGrid));
    if (!grid) return nullptr;
    GridImpl *I = new (std::nothrow) GridImpl();
    if (!I) {
        free(grid);
        return nullptr;
    }
    grid->impl = I;
    grid->sizeX = sizeX;
    grid->sizeY = sizeY;
    grid->sizeZ = sizeZ;
    grid->totalCells = (int)n;
    // lbm.c:56-60
    grid->tau = 0.5f + 3.0f * viscosity;
    if (grid->tau < 0.52f) grid->tau = 0.52f;
    if (grid->tau > 2.0f) grid->tau = 2.0f;
    // lbm.c:272-276
    grid->useRegularized = 0;
    grid->useMRT = 0;
    grid->useSmagorinsky = 0;
    grid->smagorinskyCs = 0.1f;
    grid->periodicYZ = 0;
    grid->storage = storage;
    grid->arithmetic = LBM_ARITH_EXACT;
    grid->lastError = LBM_OK;

    I->nx = sizeX;
    I->ny = sizeY;
    I->nz = sizeZ;
    I->n = n;
    I->storage = storage;
    I->elem = elem_size(storage);
    default_block(*I);

    bool good = ok(grid, cudaStreamCreateWithFlags(&I->stream, cudaStreamNonBlocking));
    const size_t popBytes = 19 * (size_t)n * I->elem;
    good = good && ok(grid, cudaMalloc(&I->pop[0], popBytes));
    good = good && ok(grid, cudaMalloc(&I->pop[1], popBytes));
    good = good && ok(grid, cudaMalloc(&I->vel, sizeof(float4) * (size_t)n));
    if (storage == LBM_STORAGE_FP64)
        good = good && ok(grid, cudaMalloc(&I->vel64, sizeof(double4) * (size_t)n));
    good = good && ok(grid, cudaMalloc(&I->solid, sizeof(int32_t) * (size_t)n));
    good = good && ok(grid, cudaMalloc(&I->flags, (size_t)n));
    good = good && ok(grid, cudaMalloc(&I->slot, sizeof(int32_t) * (size_t)n));
    // one block: 8 integer sums, then 8 FP64 sums, zeroed and read back
    // with one call each
    good = good && ok(grid, cudaMalloc(&I->force_i64, sizeof(long long) * 16));
    if (good) {
        I->force_f64 = reinterpret_cast<double *>(I->force_i64 + 8);
        I->force_ticket = reinterpret_cast<unsigned *>(I->force_i64 + 15);
    }
    good = good && ok(grid, cudaMalloc(&I->sums_f64, sizeof(double) * 4));
    good = good && ok(grid, cudaMalloc(&I->guard, sizeof(unsigned long long)));
    good = good && ok(grid, cudaMalloc(&I->err_flag, sizeof(int)));
    good = good && ok(grid, cudaMallocHost(&I->host_pinned, 256));
    if (good) {
        // lbm.c:145-250: every buffer starts zeroed
        cudaStream_t s = I->stream;
        good = good && ok(grid, cudaMemsetAsync(I->pop[0], 0, popBytes, s));
        good = good && ok(grid, cudaMemsetAsync(I->pop[1], 0, popBytes, s));
        good = good && ok(grid, cudaMemsetAsync(I->vel, 0, sizeof(float4) * (size_t)n, s));
        good = good && ok(grid, cudaMemsetAsync(I->solid, 0, sizeof(int32_t) * (size_t)n, s));
        good = good && ok(grid, cudaMemsetAsync(I->flags, 0, (size_t)n, s));
        good = good && ok(grid, cudaMemsetAsync(I->slot, 0xff, sizeof(int32_t) * (size_t)n, s));
        good = good && ok(grid, cudaMemsetAsync(I->guard, 0, sizeof(unsigned long long), s));
        good = good && ok(grid, cudaMemsetAsync(I->err_flag, 0, sizeof(int), s));
        good = good && ok(grid, cudaMemsetAsync(I->force_i64, 0, sizeof(long long) * 16, s));
        good = good && ok(grid, cudaStreamSynchronize(s));
    }
    if (!good) {
        LBM_Free(grid);
        return nullptr;
    }
    setup_tma(*I, false);
    I->fbuf = 0;
    I->gbuf = 1;
    I->vel_valid = true;
    I->stream_periodic = 0;
    return grid;
}

LBMGrid *LBM_Create(int sizeX, int sizeY, int sizeZ, float viscosity) {
    return LBM_CreateEx(sizeX, sizeY, sizeZ, viscosity, LBM_STORAGE_FP32);
}

void LBM_Free(LBMGrid *grid) {
    if (!grid) return;
    GridImpl *I = IMPL(grid);
    if (I) {
        if (I->stream) cudaStreamSynchronize(I->stream);
        drop_graph(*I);
        cudaFree(I->pop[0]);
        cudaFree(I->pop[1]);
        cudaFree(I->vel);
        cudaFree(I->vel64);
        cudaFree(I->solid);
        cudaFree(I->flags);
        cudaFree(I->slot);
        cudaFree(I->force_i64);  // force_f64 and force_ticket live in the same block
        cudaFree(I->force_part);
        cudaFree(I->sums_f64);
        cudaFree(I->guard);
        cudaFree(I->err_flag);
        if (I->host_pinned) cudaFreeHost(I->host_pinned);
        geo_free_links(I->links);
        if (I->stream) cudaStreamDestroy(I->stream);
        delete I;
    }
    free(grid);
}

void LBM_SetSolidAABB(LBMGrid *grid, float minX, float minY, float minZ, float maxX, float maxY,
                      float maxZ) {
    if (!IMPL(grid)) return;
    float *qd = begin_geometry(grid, false);
    if (!qd) return;
    GridImpl &I = *IMPL(grid);
    bool good = ok(grid, geo_aabb(I, qd, minX, minY, minZ, maxX, maxY, maxZ, I.stream));
    end_geometry(grid, qd, good);
}

static void set_sphere(LBMGrid *grid, float cx, float cy, float cz, float r, bool halfway) {
    if (!IMPL(grid)) return;
    float *qd = begin_geometry(grid, false);
    if (!qd) return;
    GridImpl &I = *IMPL(grid);
    bool good = ok(grid, geo_sphere(I, qd, cx, cy, cz, r, halfway, I.stream));
    end_geometry(grid, qd, good);
}

void LBM_SetSolidSphere(LBMGrid *grid, float cx, float cy, float cz, float radius) {
    set_sphere(grid, cx, cy, cz, radius, false);
}

void LBM_SetSolidSphereHalfway(LBMGrid *grid, float cx, float cy, float cz, float radius) {
    set_sphere(grid, cx, cy, cz, radius, true);
}

void LBM_AddGroundPlane(LBMGrid *grid, float worldZ) {
    if (!IMPL(grid)) return;
    float *qd = begin_geometry(grid, true);
    if (!qd) return;
    GridImpl &I = *IMPL(grid);
    bool good = ok(grid, geo_ground(I, qd, worldZ, I.stream));
    end_geometry(grid, qd, good);
}

void LBM_SetSolidMesh(LBMGrid *grid, float *triangles, int numTriangles, float minX, float minY,
                      float minZ, float maxX, float maxY, float maxZ) {
    if (!IMPL(grid)) return;
    if (numTriangles < 0 || (numTriangles > 0 && !triangles)) {
        grid->lastError = LBM_ERR_INVALID_ARGUMENT;
        return;
    }
    float *qd = begin_geometry(grid, false);
    if (!qd) return;
    GridImpl &I = *IMPL(grid);
    float *tris = nullptr;
    const size_t bytes = sizeof(float) * 12 * (size_t)(numTriangles > 0 ? numTriangles : 1);
    bool good = ok(grid, cudaMallocAsync(&tris, bytes, I.stream));
    if (good && numTriangles > 0)
        good = ok(grid, cudaMemcpyAsync(tris, triangles, sizeof(float) * 12 * (size_t)numTriangles,
                                        cudaMemcpyHostToDevice, I.stream));
    const float bbox[6] = {minX, minY, minZ, maxX, maxY, maxZ};
    if (good) good = ok(grid, geo_mesh(I, qd, tris, numTriangles, bbox, I.stream));
    if (tris) cudaFreeAsync(tris, I.stream);
    end_geometry(grid, qd, good);
}

float LBM_ComputeProjectedArea(LBMGrid *grid, int axis) {
    GridImpl *I = IMPL(grid);
    if (!I) return 0.0f;
    int *dcount = nullptr;
    if (!ok(grid, cudaMallocAsync(&dcount, sizeof(int), I->stream))) return 0.0f;
    int host = 0;
    bool good = ok(grid, geo_projected_area(*I, axis, dcount, I->stream));
    good = good && ok(grid, cudaMemcpyAsync(&host, dcount, sizeof(int), cudaMemcpyDeviceToHost,
                                            I->stream));
    cudaFreeAsync(dcount, I->stream);
    good = good && sync(grid);
    return good ? (float)host : 0.0f;
}

int LBM_InitializeFlow(LBMGrid *grid, float ux, float uy, float uz) {
    GridImpl *I = IMPL(grid);
    if (!I) return 0;
    drop_graph(*I);
    bool good = ok(grid, launch_init_uniform(*I, I->pop[0], I->pop[1], ux, uy, uz, I->stream));
    k_fill_vel<<<(unsigned)((I->n + 255) / 256), 256, 0, I->stream>>>(
        I->vel, I->vel64, I->n, make_float4(ux, uy, uz, 1.0f));
    good = good && ok(grid, cudaGetLastError());
    good = good && ok(grid, cudaMemsetAsync(I->guard, 0, sizeof(unsigned long long), I->stream));
    good = good && sync(grid);
    if (!good) return 0;
    I->fbuf = 0;
    I->gbuf = 1;
    I->vel_valid = true;
    I->stream_periodic = grid->periodicYZ;
    I->initialized = true;
    return 1;
}

}  // extern "C"

namespace lbm {
// f = f_new = feq(rho, u) from device fields; the state machine restarts
// from an explicit f (shared by LBM_InitializeFromField and the warm start)
int grid_init_from_device(LBMGrid *grid, const float *drho, const float *du) {
    GridImpl *I = IMPL(grid);
    drop_graph(*I);
    bool good = ok(grid, launch_init_field(*I, I->pop[0], I->pop[1], drho, du, I->stream));
    if (good) {
        k_vel_from_field<<<(unsigned)((I->n + 255) / 256), 256, 0, I->stream>>>(
            I->vel, I->vel64, I->n, drho, du);
        good = ok(grid, cudaGetLastError());
    }
    good = good && ok(grid, cudaMemsetAsync(I->guard, 0, sizeof(unsigned long long), I->stream));
    good = good && sync(grid);
    if (!good) return 0;
    I->fbuf = 0;
    I->gbuf = 1;
    I->vel_valid = true;
    I->stream_periodic = grid->periodicYZ;
    I->initialized = true;
    return 1;
}
}  // namespace lbm

extern "C" {

int LBM_InitializeFromField(LBMGrid *grid, const float *rho, const float *u) {
    GridImpl *I = IMPL(grid);
    if (!I || !rho || !u) {
        if (grid) grid->lastError = LBM_ERR_INVALID_ARGUMENT;
        return 0;
    }
    drop_graph(*I);
    float *d = nullptr;
    bool good = ok(grid, cudaMallocAsync(&d, sizeof(float) * 4 * (size_t)I->n, I->stream));
    if (!good) return 0;
    float *drho = d, *du = d + I->n;
    good = ok(grid, cudaMemcpyAsync(drho, rho, sizeof(float) * (size_t)I->n, cudaMemcpyHostToDevice,
                                    I->stream));
    good = good && ok(grid, cudaMemcpyAsync(du, u, sizeof(float) * 3 * (size_t)I->n,
                                            cudaMemcpyHostToDevice, I->stream));
    const int r = good ? grid_init_from_device(grid, drho, du) : 0;
    cudaFreeAsync(d, I->stream);
    sync(grid);
    return r;
}

void LBM_Step(LBMGrid *grid, float inletVelX, float inletVelY, float inletVelZ) {
    if (!IMPL(grid)) return;
    enqueue_step(grid, inletVelX, inletVelY, inletVelZ);
}

void LBM_StepN(LBMGrid *grid, int nSteps, float inX, float inY, float inZ) {
    GridImpl *I = IMPL(grid);
    if (!I || nSteps <= 0) return;
    // The first step out of an explicit-f state is a collide-only launch.
    if (I->fbuf >= 0) {
        if (!enqueue_step(grid, inX, inY, inZ)) return;
        nSteps--;
    }
    // Periodic flag of the stream is the caller's current one from here on.
    if (I->stream_periodic != grid->periodicYZ && nSteps > 0) {
        if (!enqueue_step(grid, inX, inY, inZ)) return;
        nSteps--;
    }
    const int chunk = 32;  // even: the buffer parity repeats after a replay
    if (nSteps >= chunk) {
        union {
            float f;
            int i;
        } cv[5];
        cv[0].f = grid->tau;
        cv[1].f = grid->smagorinskyCs;
        cv[2].f = inX;
        cv[3].f = inY;
        cv[4].f = inZ;
        const int key[8] = {op_of(grid) * 8 + (grid->useSmagorinsky == 1) * 4 +
                                grid->periodicYZ * 2 + (grid->arithmetic == LBM_ARITH_FAST),
                            cv[0].i, cv[1].i, cv[2].i, cv[3].i, cv[4].i, chunk, 1};
        const int par = I->gbuf;
        if (!I->graph[par] || memcmp(key, I->graph_key[par], sizeof(key)) != 0) {
            if (I->graph[par]) {
                cudaGraphExecDestroy(I->graph[par]);
                I->graph[par] = nullptr;
            }
            // capture `chunk` steps; capturing does not execute, so the
            // state machine is restored afterwards
            GridImpl saved = *I;
            cudaGraph_t graph = nullptr;
            bool good = ok(grid, cudaStreamBeginCapture(I->stream, cudaStreamCaptureModeThreadLocal));
            for (int k = 0; good && k < chunk; k++) good = enqueue_step(grid, inX, inY, inZ);
            cudaError_t e = cudaStreamEndCapture(I->stream, &graph);
            good = good && ok(grid, e);
            cudaGraphExec_t exec = nullptr;
            if (good) good = ok(grid, cudaGraphInstantiate(&exec, graph, 0));
            if (graph) cudaGraphDestroy(graph);
            *I = saved;
            if (!good) return;
            I->graph[par] = exec;
            memcpy(I->graph_key[par], key, sizeof(key));
        }
        while (nSteps >= chunk) {
            if (!ok(grid, cudaGraphLaunch(I->graph[I->gbuf], I->stream))) return;
            // replicate the state transition of `chunk` fused steps
            I->vin = 1 - I->gbuf;  // chunk is even: gbuf unchanged
            I->vin_kind = IN_POST_COLLISION;
            I->vin_periodic = I->stream_periodic;
            I->vin_inlet[0] = inX;
            I->vin_inlet[1] = inY;
            I->vin_inlet[2] = inZ;
            I->vel_valid = false;
            I->stream_periodic = grid->periodicYZ;
            nSteps -= chunk;
        }
    }
    while (nSteps-- > 0)
        if (!enqueue_step(grid, inX, inY, inZ)) return;
}

const void *LBM_GetVelocityBuffer(LBMGrid *grid) {
    GridImpl *I = IMPL(grid);
    if (!I) return nullptr;
    if (!ensure_vel(grid) || !sync(grid)) return nullptr;
    return I->vel;
}

void LBM_ComputeDragForceDecomposed(LBMGrid *grid, float *forceX, float *forceY, float *forceZ,
                                    float *pressureX, float *pressureY, float *pressureZ) {
    // lbm.c:842-850
    if (forceX) *forceX = 0.0f;
    if (forceY) *forceY = 0.0f;
    if (forceZ) *forceZ = 0.0f;
    if (pressureX) *pressureX = 0.0f;
    if (pressureY) *pressureY = 0.0f;
    if (pressureZ) *pressureZ = 0.0f;
    long long raw[7];
    double f64[6];
    if (!LBM_ComputeDragForceF64(grid, f64, raw)) return;
    // lbm.c:909-917 (the reference accumulates in int32)
    if (forceX) *forceX = (float)(int32_t)raw[0] / 10000.0f;
    if (forceY) *forceY = (float)(int32_t)raw[1] / 10000.0f;
    if (forceZ) *forceZ = (float)(int32_t)raw[2] / 10000.0f;
    if (pressureX) *pressureX = (float)(int32_t)raw[4] / 10000.0f;
    if (pressureY) *pressureY = (float)(int32_t)raw[5] / 10000.0f;
    if (pressureZ) *pressureZ = (float)(int32_t)raw[6] / 10000.0f;
}

int LBM_ComputeDragForceF64(LBMGrid *grid, double *out6, long long *raw7) {
    GridImpl *I = IMPL(grid);
    if (!I) return 0;
    const void *fexp = I->fbuf >= 0 ? I->pop[I->fbuf] : nullptr;
    const float4 *vel = I->vel_valid ? I->vel : nullptr;
    const int blocks = force_blocks(I->links.nb);
    if (blocks > I->force_part_blocks) {
        // partial sums of the force kernel's blocks; grows with the link list
        if (!ok(grid, cudaStreamSynchronize(I->stream))) return 0;
        cudaFree(I->force_part);
        I->force_part = nullptr;
        I->force_part_blocks = 0;
        if (!ok(grid, cudaMalloc(&I->force_part, sizeof(long long) * 16 * (size_t)blocks)))
            return 0;
        I->force_part_blocks = blocks;
    }
    bool good = ok(grid, launch_force(*I, I->pop[I->gbuf], fexp, I->stream_periodic, vel,
                                      I->vel64, I->pop[I->vin], I->vin_kind, I->vin_periodic, I->vin_inlet,
                                      I->force_i64, I->force_f64, I->force_part, I->force_ticket,
                                      I->stream));
    long long *h = I->host_pinned;  // h[0..6] integer sums, h[8..13] FP64 sums
    good = good && ok(grid, cudaMemcpyAsync(h, I->force_i64, sizeof(long long) * 14,
                                            cudaMemcpyDeviceToHost, I->stream));
    good = good && sync(grid);
    if (!good) return 0;
    if (raw7)
        for (int k = 0; k < 7; k++) raw7[k] = h[k];
    if (out6) memcpy(out6, h + 8, sizeof(double) * 6);
    return 1;
}

void LBM_ComputeDragForce(LBMGrid *grid, float *forceX, float *forceY, float *forceZ) {
    LBM_ComputeDragForceDecomposed(grid, forceX, forceY, forceZ, nullptr, nullptr, nullptr);
}

float LBM_ComputeDragCoefficient(LBMGrid *grid, float inletVelocity, float refArea) {
    float fx, fy, fz;
    LBM_ComputeDragForce(grid, &fx, &fy, &fz);
    const float dragForce = fabsf(fx);
    const float rho = 1.0f;
    const float dynamicPressure = 0.5f * rho * inletVelocity * inletVelocity;
    if (dynamicPressure * refArea < 1e-10f) return 0.0f;
    return dragForce / (dynamicPressure * refArea);
}

float LBM_ComputeLiftCoefficient(LBMGrid *grid, float inletVelocity, float refArea) {
    float fx, fy, fz;
    LBM_ComputeDragForce(grid, &fx, &fy, &fz);
    const float liftForce = fabsf(fy);
    const float rho = 1.0f;
    const float dynamicPressure = 0.5f * rho * inletVelocity * inletVelocity;
    if (dynamicPressure * refArea < 1e-10f) return 0.0f;
    return liftForce / (dynamicPressure * refArea);
}

int LBM_ComputeMassMomentum(LBMGrid *grid, double *out4) {
    GridImpl *I = IMPL(grid);
    if (!I || !out4) return 0;
    if (!materialize_f(grid)) return 0;
    bool good = ok(grid, cudaMemsetAsync(I->sums_f64, 0, sizeof(double) * 4, I->stream));
    good = good && ok(grid, launch_mass_momentum(*I, I->pop[I->fbuf], I->sums_f64, I->stream));
    good = good && ok(grid, cudaMemcpyAsync(out4, I->sums_f64, sizeof(double) * 4,
                                            cudaMemcpyDeviceToHost, I->stream));
    return good && sync(grid) ? 1 : 0;
}

long long LBM_GetGuardResetCount(LBMGrid *grid) {
    GridImpl *I = IMPL(grid);
    if (!I) return -1;
    unsigned long long v = 0;
    if (!ok(grid, cudaMemcpyAsync(&v, I->guard, sizeof(v), cudaMemcpyDeviceToHost, I->stream)) ||
        !sync(grid))
        return -1;
    return (long long)v;
}

int LBM_CopyVelocity(LBMGrid *grid, float *host) {
    GridImpl *I = IMPL(grid);
    if (!I || !host) return 0;
    if (!ensure_vel(grid)) return 0;
    bool good = ok(grid, cudaMemcpyAsync(host, I->vel, sizeof(float4) * (size_t)I->n,
                                         cudaMemcpyDeviceToHost, I->stream));
    return good && sync(grid) ? 1 : 0;
}

int LBM_CopySolid(LBMGrid *grid, int32_t *host) {
    GridImpl *I = IMPL(grid);
    if (!I || !host) return 0;
    bool good = ok(grid, cudaMemcpyAsync(host, I->solid, sizeof(int32_t) * (size_t)I->n,
                                         cudaMemcpyDeviceToHost, I->stream));
    return good && sync(grid) ? 1 : 0;
}

static int copy_pop(LBMGrid *grid, int which, void *host, bool as_double) {
    GridImpl *I = IMPL(grid);
    if (!I || !host) return 0;
    int buf;
    if (which == 0) {
        if (!materialize_f(grid)) return 0;
        buf = I->fbuf;
    } else {
        buf = I->gbuf;
    }
    const size_t bytes = 19 * (size_t)I->n * (as_double ? 8 : 4);
    void *tmp = nullptr;
    bool good = ok(grid, cudaMallocAsync(&tmp, bytes, I->stream));
    if (!good) return 0;
    good = ok(grid, launch_export_aos(*I, I->pop[buf], tmp, as_double, I->stream));
    good = good && ok(grid, cudaMemcpyAsync(host, tmp, bytes, cudaMemcpyDeviceToHost, I->stream));
    cudaFreeAsync(tmp, I->stream);
    return good && sync(grid) ? 1 : 0;
}

int LBM_CopyPopulations(LBMGrid *grid, float *host) { return copy_pop(grid, 0, host, false); }
int LBM_CopyPostCollision(LBMGrid *grid, float *host) { return copy_pop(grid, 1, host, false); }
int LBM_CopyPopulationsF64(LBMGrid *grid, double *host) { return copy_pop(grid, 0, host, true); }
int LBM_CopyPostCollisionF64(LBMGrid *grid, double *host) { return copy_pop(grid, 1, host, true); }

int LBM_LoadPopulations(LBMGrid *grid, const float *host) {
    GridImpl *I = IMPL(grid);
    if (!I || !host) return 0;
    drop_graph(*I);
    const size_t bytes = 19 * (size_t)I->n * 4;
    float *tmp = nullptr;
    bool good = ok(grid, cudaMallocAsync(&tmp, bytes, I->stream));
    if (!good) return 0;
    good = ok(grid, cudaMemcpyAsync(tmp, host, bytes, cudaMemcpyHostToDevice, I->stream));
    good = good && ok(grid, launch_import_aos(*I, tmp, I->pop[0], I->stream));
    good = good && ok(grid, launch_import_aos(*I, tmp, I->pop[1], I->stream));
    cudaFreeAsync(tmp, I->stream);
    good = good && sync(grid);
    if (!good) return 0;
    I->fbuf = 0;
    I->gbuf = 1;
    I->vin = 0;
    I->vin_kind = IN_EXPLICIT_F;
    I->vel_valid = false;
    I->stream_periodic = grid->periodicYZ;
    I->initialized = true;
    return 1;
}

int LBM_CopyQ(LBMGrid *grid, float *host) {
    GridImpl *I = IMPL(grid);
    if (!I || !host) return 0;
    float *qd = nullptr;
    const size_t bytes = sizeof(float) * 19 * (size_t)I->n;
    bool good = ok(grid, cudaMallocAsync(&qd, bytes, I->stream));
    if (!good) return 0;
    good = ok(grid, geo_links_to_dense(*I, qd, I->stream));
    good = good && ok(grid, cudaMemcpyAsync(host, qd, bytes, cudaMemcpyDeviceToHost, I->stream));
    cudaFreeAsync(qd, I->stream);
    return good && sync(grid) ? 1 : 0;
}

long long LBM_GetBoundaryLinkCount(LBMGrid *grid) {
    GridImpl *I = IMPL(grid);
    return I ? I->links.nl : -1;
}

int LBM_CopyBoundaryLinks(LBMGrid *grid, int32_t *cell, int32_t *dir, float *q) {
    GridImpl *I = IMPL(grid);
    if (!I) return 0;
    const size_t nl = (size_t)I->links.nl;
    bool good = true;
    if (nl && cell)
        good = good && ok(grid, cudaMemcpyAsync(cell, I->links.lcell, 4 * nl,
                                                cudaMemcpyDeviceToHost, I->stream));
    if (nl && dir)
        good = good && ok(grid, cudaMemcpyAsync(dir, I->links.ldir, 4 * nl, cudaMemcpyDeviceToHost,
                                                I->stream));
    if (nl && q)
        good = good && ok(grid, cudaMemcpyAsync(q, I->links.lq, 4 * nl, cudaMemcpyDeviceToHost,
                                                I->stream));
    return good && sync(grid) ? 1 : 0;
}

void *LBM_GetStream(LBMGrid *grid) {
    GridImpl *I = IMPL(grid);
    return I ? (void *)I->stream : nullptr;
}

int LBM_BytesPerUpdate(LBMGrid *grid) {
    GridImpl *I = IMPL(grid);
    return I ? (int)(38 * I->elem) : 0;
}

int LBM_SetTMAStaging(LBMGrid *grid, int enable) {
    GridImpl *I = IMPL(grid);
    if (!I) return 0;
    if (!enable) {
        I->tma = false;
    } else if (!I->tma) {
        setup_tma(*I, true);
    }
    drop_graph(*I);  // captured steps name the kernel
    return I->tma ? 1 : 0;
}

// vti_export.c:10-116
void writeVTI(LBMGrid *grid, const char *path, int step) {
    GridImpl *I = IMPL(grid);
    if (!I || !path) return;
    char filename[512];
    snprintf(filename, sizeof(filename), "%s/field_%06d.vti", path, step);
    const int nx = grid->sizeX, ny = grid->sizeY, nz = grid->sizeZ;
    const size_t total = (size_t)nx * ny * nz;
    std::vector<float> vel;
    std::vector<int32_t> solid;
    try {
        vel.resize(total * 4);
        solid.resize(total);
    } catch (...) {
        return;
    }
    if (!LBM_CopyVelocity(grid, vel.data()) || !LBM_CopySolid(grid, solid.data())) return;
    FILE *f = fopen(filename, "wb");
    if (!f) return;
    const size_t rhoOffset = sizeof(uint64_t) + total * 3 * sizeof(float);
    const size_t solidOffset = rhoOffset + sizeof(uint64_t) + total * sizeof(float);
    fprintf(f,
            "<?xml version=\"1.0\"?>\n"
            "<VTKFile type=\"ImageData\" version=\"1.0\""
            " byte_order=\"LittleEndian\" header_type=\"UInt64\">\n"
            "  <ImageData WholeExtent=\"0 %d 0 %d 0 %d\""
            " Origin=\"0 0 0\" Spacing=\"1 1 1\">\n"
            "    <Piece Extent=\"0 %d 0 %d 0 %d\">\n"
            "      <PointData Vectors=\"velocity\" Scalars=\"rho\">\n"
            "        <DataArray type=\"Float32\" Name=\"velocity\""
            " NumberOfComponents=\"3\" format=\"appended\""
            " offset=\"0\"/>\n"
            "        <DataArray type=\"Float32\" Name=\"rho\""
            " format=\"appended\" offset=\"%lu\"/>\n"
            "        <DataArray type=\"Int32\" Name=\"solid\""
            " format=\"appended\" offset=\"%lu\"/>\n"
            "      </PointData>\n"
            "    </Piece>\n"
            "  </ImageData>\n"
            "  <AppendedData encoding=\"raw\">\n_",
            nx, ny, nz, nx, ny, nz, (unsigned long)rhoOffset, (unsigned long)solidOffset);
    // velocity (xyz of each vec4), rho (w), solid -- each with a uint64 size
    std::vector<float> buf(total * 3);
    for (size_t i = 0; i < total; i++) {
        buf[3 * i] = vel[4 * i];
        buf[3 * i + 1] = vel[4 * i + 1];
        buf[3 * i + 2] = vel[4 * i + 2];
    }
    bool w = true;
    uint64_t sz = (uint64_t)total * 3 * sizeof(float);
    w = w && fwrite(&sz, sizeof(uint64_t), 1, f) == 1;
    w = w && fwrite(buf.data(), sizeof(float), total * 3, f) == total * 3;
    for (size_t i = 0; i < total; i++) buf[i] = vel[4 * i + 3];
    sz = (uint64_t)total * sizeof(float);
    w = w && fwrite(&sz, sizeof(uint64_t), 1, f) == 1;
    w = w && fwrite(buf.data(), sizeof(float), total, f) == total;
    sz = (uint64_t)total * sizeof(int32_t);
    w = w && fwrite(&sz, sizeof(uint64_t), 1, f) == 1;
    w = w && fwrite(solid.data(), sizeof(int32_t), total, f) == total;
    if (!w) {
        fprintf(stderr, "VTK: write error for %s\n", filename);
        fclose(f);
        return;
    }
    fprintf(f, "\n  </AppendedData>\n</VTKFile>\n");
    fclose(f);
    printf("VTK: wrote %s\n", filename);
}

// ---------------------------------------------------------------------
// particles
// ---------------------------------------------------------------------
LBMParticles *LBM_ParticlesCreate(int n, unsigned int seed) {
    if (n <= 0) return nullptr;
    LBMParticles *p = new (std::nothrow) LBMParticles();
    if (!p) return nullptr;
    p->n = n;
    p->seed = seed;
    std::vector<LBMParticle> h((size_t)n);
    particles_seed_host(h.data(), n, seed);
    if (cudaEventCreateWithFlags(&p->done, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&p->dev, sizeof(LBMParticle) * (size_t)n) != cudaSuccess ||
        cudaMemcpy(p->dev, h.data(), sizeof(LBMParticle) * (size_t)n, cudaMemcpyHostToDevice) !=
            cudaSuccess) {
        if (p->done) cudaEventDestroy(p->done);
        cudaFree(p->dev);
        delete p;
        return nullptr;
    }
    return p;
}

void LBM_ParticlesFree(LBMParticles *p) {
    if (!p) return;
    if (p->done) {
        cudaEventSynchronize(p->done);
        cudaEventDestroy(p->done);
    }
    cudaFree(p->dev);
    delete p;
}

int LBM_ParticlesStep(LBMParticles *p, LBMGrid *grid, float dt) {
    GridImpl *I = IMPL(grid);
    if (!p || !I) return 0;
    if (!ensure_vel(grid)) return 0;
    if (!ok(grid, launch_particles(p->dev, p->n, I->vel, I->nx, I->ny, I->nz, dt, p->seed,
                                   I->stream)))
        return 0;
    return ok(grid, cudaEventRecord(p->done, I->stream)) ? 1 : 0;
}

int LBM_ParticlesCopy(LBMParticles *p, LBMParticle *host) {
    if (!p || !host) return 0;
    if (cudaEventSynchronize(p->done) != cudaSuccess) return 0;
    return cudaMemcpy(host, p->dev, sizeof(LBMParticle) * (size_t)p->n, cudaMemcpyDeviceToHost) ==
                   cudaSuccess
               ? 1
               : 0;
}

int LBM_ParticlesLoad(LBMParticles *p, const LBMParticle *host) {
    if (!p || !host) return 0;
    if (cudaEventSynchronize(p->done) != cudaSuccess) return 0;
    return cudaMemcpy(p->dev, host, sizeof(LBMParticle) * (size_t)p->n, cudaMemcpyHostToDevice) ==
                   cudaSuccess
               ? 1
               : 0;
}

void *LBM_ParticlesDevice(LBMParticles *p) { return p ? p->dev : nullptr; }

}  // extern "C"
