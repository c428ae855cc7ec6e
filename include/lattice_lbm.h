/*
 * lattice_lbm.h -- C ABI of the B200 (sm_100a) D3Q19 wind-tunnel solver.
 *
 * Drop-in replacement for the solver API of Lattice
 * (MarcosAsh/Lattice_Fluid_Dynamics, simulation/lib/lbm.h).  Every function
 * the reference declares keeps its name, argument order and meaning; the
 * one GL type in that API (the GLuint returned by LBM_GetVelocityBuffer)
 * becomes a CUDA device pointer.  A C caller written against lbm.h links
 * this library in place of simulation/src/lbm.c; code that pokes the
 * public LBMGrid fields (simulation/src/main.c:503-516,
 * simulation/test/test_lbm.c:373,391-393) keeps compiling because those
 * fields keep their names.
 *
 * Threading: one CUDA stream per grid.  LBM_Step only enqueues work; every
 * function that returns data to the host synchronises that stream.  All
 * functions are safe to call from one host thread per grid.
 *
 * Errors: functions keep the reference's return conventions (LBM_Create
 * returns NULL, LBM_InitializeFlow returns 0, the void functions fail
 * silently) and additionally record an LBM_ERR_* code readable with
 * LBM_GetLastError.  No function traps the device.
 */
#ifndef LATTICE_LBM_H
#define LATTICE_LBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Population storage formats (LBM_CreateEx).  FP16 and BF16 store the
 * shifted deviation f_i - w_i and collide in FP32; FP64 stores and
 * collides in double. */
enum {
    LBM_STORAGE_FP32 = 0,
    LBM_STORAGE_FP16 = 1,
    LBM_STORAGE_BF16 = 2,
    LBM_STORAGE_FP64 = 3
};

/* Arithmetic of the step kernel (LBMGrid.arithmetic).  EXACT performs the
 * reference shaders' operations as separately rounded IEEE single (or
 * double) operations, bit-identical to the CPU oracle.  FAST contracts
 * multiply-adds and uses hardware-approximate division and square root;
 * its results stay within the parity tolerances of the tests but are not
 * bit-identical.  FP64 storage always runs EXACT. */
enum {
    LBM_ARITH_EXACT = 0,
    LBM_ARITH_FAST = 1
};

enum {
    LBM_OK = 0,
    LBM_ERR_INVALID_ARGUMENT = 1,
    LBM_ERR_OUT_OF_MEMORY = 2,
    LBM_ERR_CUDA = 3,
    LBM_ERR_NOT_INITIALIZED = 4,
    LBM_ERR_UNSUPPORTED = 5,
    LBM_ERR_DIVERGED = 6,
    LBM_ERR_TIMEOUT = 7
};

/* Grid handle.  The first fields are the public scalars of the reference
 * struct (simulation/lib/lbm.h:6-56) under the same names; callers may set
 * tau and the operator flags between steps exactly as with the reference.
 * The GL buffer/program/uniform fields of the reference have no
 * counterpart; device state lives behind `impl`. */
typedef struct LBMGrid {
    int sizeX, sizeY, sizeZ;
    int totalCells;
    float tau;
    int useRegularized;  /* 0 = BGK, 1 = regularized            */
    int useMRT;          /* 1 = MRT (d'Humieres 2002) collision  */
    int useSmagorinsky;  /* 1 = Smagorinsky SGS tau_eff          */
    float smagorinskyCs; /* Smagorinsky constant                 */
    int periodicYZ;      /* 0 = clamp, 1 = periodic y/z          */
    /* extensions of this library */
    int storage;         /* LBM_STORAGE_*, fixed at creation     */
    int arithmetic;      /* LBM_ARITH_*, may change between steps */
    int lastError;       /* last LBM_ERR_* code                  */
    void *impl;          /* opaque device state                  */
} LBMGrid;

/* Particle record of the reference (simulation/lib/particle_system.h:12-17,
 * shader struct particle_lbm.comp:4-9): 32 bytes. */
typedef struct LBMParticle {
    float x, y, z, pad;
    float vx, vy, vz, life;
} LBMParticle;

/* ---------------------------------------------------------------------
 * Reference API (simulation/lib/lbm.h:58-129)
 * ------------------------------------------------------------------- */

/* lbm.h:59 / lbm.c:46-318.  tau = 0.5 + 3*viscosity clamped to [0.52, 2];
 * FP32 storage.  NULL on failure. */
LBMGrid *LBM_Create(int sizeX, int sizeY, int sizeZ, float viscosity);

/* lbm.h:62 / lbm.c:320-344.  Accepts NULL. */
void LBM_Free(LBMGrid *grid);

/* lbm.h:65-71 / lbm.c:346-435.  World box [-4,4]x[-2,2]x[-2,2]; q = 0.5 on
 * every fluid->solid link. */
void LBM_SetSolidAABB(LBMGrid *grid, float minX, float minY, float minZ,
                      float maxX, float maxY, float maxZ);

/* lbm.h:74 / lbm.c:670-721.  f = f_new = feq(1,u), velocity = (u,1).
 * Returns 1 on success, 0 on failure. */
int LBM_InitializeFlow(LBMGrid *grid, float ux, float uy, float uz);

/* lbm.h:77 / lbm.c:723-821.  One collide + stream step (asynchronous). */
void LBM_Step(LBMGrid *grid, float inletVelX, float inletVelY,
              float inletVelZ);

/* lbm.h:80 / lbm.c:823-825.  The reference returns the GL SSBO holding
 * vec4(ux,uy,uz,rho) per cell; this returns the CUDA device pointer to the
 * same float4 array (x-fastest, 16 bytes per cell), valid until the next
 * LBM_Step / LBM_Free.  The stream is synchronised before returning. */
const void *LBM_GetVelocityBuffer(LBMGrid *grid);

/* lbm.h:83-86 / lbm.c:827-833 */
void LBM_ComputeDragForce(LBMGrid *grid, float *forceX, float *forceY,
                          float *forceZ);

/* lbm.h:90-96 / lbm.c:835-918.  Mei-Luo-Shyy momentum exchange with the
 * reference's per-cell x1e4 integer quantisation; pressure pointers may be
 * NULL. */
void LBM_ComputeDragForceDecomposed(LBMGrid *grid, float *forceX,
                                    float *forceY, float *forceZ,
                                    float *pressureX, float *pressureY,
                                    float *pressureZ);

/* lbm.h:99-101 / lbm.c:920-940: |Fx| / (0.5 U^2 A) */
float LBM_ComputeDragCoefficient(LBMGrid *grid, float inletVelocity,
                                 float refArea);

/* lbm.h:104-106 / lbm.c:942-962: |Fy| / (0.5 U^2 A) */
float LBM_ComputeLiftCoefficient(LBMGrid *grid, float inletVelocity,
                                 float refArea);

/* lbm.h:109-110 / lbm.c:437-535.  Analytic ray-sphere Bouzidi q. */
void LBM_SetSolidSphere(LBMGrid *grid, float cx, float cy, float cz,
                        float radius);

/* lbm.h:114 / lbm.c:537-614.  Ground cells get solid = 2. */
void LBM_AddGroundPlane(LBMGrid *grid, float worldZ);

/* lbm.h:118 / lbm.c:616-668.  Count of (.,.) columns holding a solid==1
 * cell along `axis` (0 = x, 1 = y, 2 = z). */
float LBM_ComputeProjectedArea(LBMGrid *grid, int axis);

/* lbm.h:121-129 / lbm.c:964-1223.  `triangles` holds 12 floats per
 * triangle {v0,pad,v1,pad,v2,pad} (GPUTriangle, model_bounds.h:14-18);
 * +x ray-parity fill inside the given box, Moller-Trumbore q per link. */
void LBM_SetSolidMesh(LBMGrid *grid, float *triangles, int numTriangles,
                      float minX, float minY, float minZ, float maxX,
                      float maxY, float maxZ);

/* simulation/lib/vti_export.h (vti_export.c:10-116): writes
 * <path>/field_<step %06d>.vti with velocity, rho and solid. */
void writeVTI(LBMGrid *grid, const char *path, int step);

/* ---------------------------------------------------------------------
 * Replacements for the reference's direct GL buffer access
 * (main.c:1029, vti_export.c:30-34, test_lbm.c:258,503 read
 * grid->solidBuffer / grid->velocityBuffer with glGetBufferSubData).
 * All return 1 on success, 0 on failure, and synchronise the stream.
 * ------------------------------------------------------------------- */

/* float4 (ux,uy,uz,rho) per cell -> host[4*totalCells] */
int LBM_CopyVelocity(LBMGrid *grid, float *host);
/* int32 solid mask (0 fluid, 1 body, 2 ground) -> host[totalCells] */
int LBM_CopySolid(LBMGrid *grid, int32_t *host);
/* post-stream populations f in the reference's AoS order
 * host[i + 19*cell]; FP64 grids convert to float */
int LBM_CopyPopulations(LBMGrid *grid, float *host);
/* post-collision populations f_new (the reference's fNewBuffer) */
int LBM_CopyPostCollision(LBMGrid *grid, float *host);
/* FP64 grids: both population arrays in double */
int LBM_CopyPopulationsF64(LBMGrid *grid, double *host);
int LBM_CopyPostCollisionF64(LBMGrid *grid, double *host);
/* dense Bouzidi table q[i + 19*cell], -1 where there is no link (the
 * reference's qBuffer) */
int LBM_CopyQ(LBMGrid *grid, float *host);
/* number of boundary links (entries with q >= 0) */
long long LBM_GetBoundaryLinkCount(LBMGrid *grid);
/* compacted boundary-link list sorted by (cell, direction); any of the
 * three output pointers may be NULL */
int LBM_CopyBoundaryLinks(LBMGrid *grid, int32_t *cell, int32_t *dir,
                          float *q);
/* device pointer of the grid's cudaStream_t */
void *LBM_GetStream(LBMGrid *grid);

/* ---------------------------------------------------------------------
 * Extensions
 * ------------------------------------------------------------------- */

/* LBM_Create with a population storage format (LBM_STORAGE_*). */
LBMGrid *LBM_CreateEx(int sizeX, int sizeY, int sizeZ, float viscosity,
                      int storage);

/* LBM_SetSolidSphere with q = 0.5 on every link (half-way bounce-back). */
void LBM_SetSolidSphereHalfway(LBMGrid *grid, float cx, float cy, float cz,
                               float radius);

/* Run `nSteps` steps with a constant inlet velocity; launches are
 * captured into a CUDA graph and replayed. */
void LBM_StepN(LBMGrid *grid, int nSteps, float inletVelX, float inletVelY,
               float inletVelZ);

/* Force with FP64 accumulation (no quantisation): out[6] = fx,fy,fz,px,py,pz.
 * Also returns the reference's int-quantised sums in raw7 (may be NULL):
 * x,y,z,count,px,py,pz in units of 1e-4. */
int LBM_ComputeDragForceF64(LBMGrid *grid, double *out6, long long *raw7);

/* Global sums in FP64 over all cells of the post-stream state:
 * out[0] = mass (sum of rho), out[1..3] = momentum.  Returns 1 on success,
 * 0 on failure (as LBM_InitializeFlow). */
int LBM_ComputeMassMomentum(LBMGrid *grid, double *out4);

/* No counterpart in the reference.  FP64 mass and momentum (out4[0] =
 * sum of rho, out4[1..3] = momentum) of a caller-owned FP32 population field
 * in this library's SoA layout, populations[i * numCells + cell], computed
 * on `stream` (a cudaStream_t; NULL is the legacy default stream).  The call
 * synchronises that stream and writes the four sums to host memory out4
 * before it returns.  It allocates nothing, for callers that cannot call
 * cudaMalloc: real-time loops that must not stall on an allocation, and
 * applications whose device memory belongs to another allocator.  The
 * scratch is a fixed 128 KiB __device__ array held per GPU for the life of
 * the process, which limits numCells to 268,435,456.  The first call on each
 * device looks up that array's device address (cudaGetSymbolAddress), so
 * make it before any stream capture.  All calls share the array: calls that
 * overlap on the GPU race.
 * Return convention: LBM_OK (0) on success -- the opposite of
 * LBM_ComputeMassMomentum, which returns 1 on success.  Errors:
 * LBM_ERR_INVALID_ARGUMENT for a NULL pointer, numCells <= 0 or above the
 * maximum (nothing is launched); LBM_ERR_CUDA when the address lookup, a
 * launch or the copy fails, or when the stream synchronisation reports an
 * error (which may come from earlier work on the same stream). */
int LBM_MassMomentumNoAlloc(const float *populations, long long numCells,
                            double *out4, void *stream);

/* Cells reset by the stability guard since LBM_InitializeFlow. */
long long LBM_GetGuardResetCount(LBMGrid *grid);

/* Load post-stream populations (reference AoS order, float) as the new
 * state; velocity is recomputed on demand.  Checkpoint restore. */
int LBM_LoadPopulations(LBMGrid *grid, const float *host);

/* Initialise from a macroscopic field: f = f_new = feq(rho, u) per cell,
 * host arrays rho[totalCells], u[3*totalCells] (x-fastest). */
int LBM_InitializeFromField(LBMGrid *grid, const float *rho, const float *u);

/* Last error code of the grid (LBM_ERR_*), and a readable name. */
int LBM_GetLastError(LBMGrid *grid);
const char *LBM_GetErrorString(int code);

/* Bytes of population traffic one lattice update moves (19 loads + 19
 * stores of the storage type): 152 FP32, 76 FP16/BF16, 304 FP64. */
int LBM_BytesPerUpdate(LBMGrid *grid);

/* Fused steps of 32 x 8 launch tiles can stage their pull neighbourhood in
 * shared memory with TMA bulk tensor copies (FP32 / FP16 / BF16 storage,
 * sizeX * element size a multiple of 16 bytes); results are identical to
 * the direct kernel's, throughput is lower on B200 (0.75-0.91x).  enable =
 * 0 turns it off, 1 on where possible; the return value is whether it is
 * on.  Off by default; LBM_TMA=1 in the environment when the grid is
 * created turns it on. */
int LBM_SetTMAStaging(LBMGrid *grid, int enable);

/* ---------------------------------------------------------------------
 * Particles (particle_lbm.comp:46-89 trilinear sampler, :207-293 Euler
 * step with collisionMode 0).  Particles live in device memory.
 * ------------------------------------------------------------------- */
typedef struct LBMParticles LBMParticles;

/* n particles seeded uniformly on the inlet plane x = -4 (y, z uniform in
 * [-2, 2)) by a counter hash of (seed, index); velocity 0, life 1. */
LBMParticles *LBM_ParticlesCreate(int n, unsigned int seed);
void LBM_ParticlesFree(LBMParticles *p);
/* One Euler step of dt through the grid's current velocity field; runs on
 * the grid's stream. */
int LBM_ParticlesStep(LBMParticles *p, LBMGrid *grid, float dt);
int LBM_ParticlesCopy(LBMParticles *p, LBMParticle *host);
int LBM_ParticlesLoad(LBMParticles *p, const LBMParticle *host);
/* device pointer to the LBMParticle array */
void *LBM_ParticlesDevice(LBMParticles *p);

/* ---------------------------------------------------------------------
 * Batched sweeps: many independent grids advanced together, replayed from
 * a CUDA graph of 32 steps (one graph launch per 32 steps of the batch), each grid with its own size, tau, operator,
 * Smagorinsky constant, geometry, periodic flag and inlet velocity.  The
 * reference runs one grid per process (main.c); a parameter sweep there is
 * many processes.  Every grid's populations are bit-identical to stepping
 * it alone with LBM_Step.
 * ------------------------------------------------------------------- */
typedef struct LBMBatch LBMBatch;

/* Group `count` grids (caller-owned, all with the same storage format,
 * LBM_ARITH_EXACT, already initialised).  The grids stay usable through the
 * rest of the API between runs.  Returns NULL on invalid input. */
LBMBatch *LBM_BatchCreate(LBMGrid **grids, int count);
void LBM_BatchFree(LBMBatch *batch);

/* Advance every grid by nSteps steps; inlet holds 3 floats per grid (the
 * LBM_Step inlet velocity).  Asynchronous with respect to the host; later
 * calls on any member grid are ordered after it.  Returns LBM_OK or an
 * LBM_ERR_* code. */
int LBM_BatchRun(LBMBatch *batch, int nSteps, const float *inlet);

/* Choose each grid's tile width (32, 64, 128 or 256 cells along x; 256 /
 * width rows) for each schedule by timing `trialLaunches` launches of each
 * candidate on that grid alone, then the schedule (below) by timing a whole
 * step of each.  The timed launches write only the buffer the grids' next
 * step overwrites, after materialising the velocity field, so the grids'
 * state is untouched.  Returns LBM_OK or an LBM_ERR_* code. */
int LBM_BatchAutotune(LBMBatch *batch, int trialLaunches);

/* Tile shape of grid `index` (tileX cells along x by tileY rows). */
int LBM_BatchGetTile(LBMBatch *batch, int index, int *tileX, int *tileY);
int LBM_BatchSetTile(LBMBatch *batch, int index, int tileX);

/* Schedule of a step: LBM_BATCH_FUSED (one kernel launch per step for up to
 * 64 grids of one collision operator) or LBM_BATCH_GRAPH (each grid's own
 * step kernel, grids spread over 4 concurrent streams); both replayed from a
 * CUDA graph of 32 steps.  LBM_BatchAutotune picks the faster one. */
#define LBM_BATCH_FUSED 0
#define LBM_BATCH_GRAPH 1
int LBM_BatchGetSchedule(LBMBatch *batch);
int LBM_BatchSetSchedule(LBMBatch *batch, int schedule);

/* 256-cell tiles of one batched step over all grids, and the CUDA stream of
 * the batch. */
long long LBM_BatchTilesPerStep(LBMBatch *batch);
void *LBM_BatchGetStream(LBMBatch *batch);

/* ---------------------------------------------------------------------
 * Warm-start network kernels (no counterpart in the reference, whose
 * learned components are CPU MLPs).  3x3x3 convolutions with zero padding
 * over channels-last BF16 activations on the tensor cores (tcgen05, FP32
 * accumulation).  All pointers are device pointers; channel counts,
 * strides and offsets are multiples of 8.  Weights are BF16
 * [coutPad][LBM_NNKPad(cin)] with k = tap * cin + c, tap = (dz+1)*9 +
 * (dy+1)*3 + (dx+1), zero-padded.  coutPad is 16, 32, 48, 64, 96, 128 or
 * 192 (forward) and 16, 32, 64 or 128 (weight gradient).  Calls are
 * asynchronous on `stream` (a cudaStream_t).
 * ------------------------------------------------------------------- */

/* 27 * cin rounded up to a multiple of 128. */
int LBM_NNKPad(int cin);

/* y = act(conv(x, w) + bias) for the first coutStore output channels;
 * act 0 = linear, 1 = leaky ReLU (slope 0.1).  Output to BF16 `y` and/or
 * FP32 `y32` (both with stride yStride and offset yOff; `accumulate` adds
 * into y32).  The input gradient of a convolution is this call on the
 * weights from LBM_NNWeightTranspose with act = 0. */
int LBM_NNConvForward(const void *x, int xStride, int xOff, int cin, const void *w,
                      const float *bias, int coutPad, int act, void *y, float *y32, int yStride,
                      int yOff, int coutStore, int accumulate, int nb, int nz, int ny, int nx,
                      void *stream);

/* wt[ci][(26 - tap) * cout + co] = w[co][tap * cin + ci]: the weights of
 * the input-gradient convolution, [wtRows][LBM_NNKPad(cout)], rows >= cin
 * zero. */
int LBM_NNWeightTranspose(const void *w, int cout, int cin, void *wt, int wtRows, void *stream);

/* dw[co][k] (+)= sum over voxels of g[v][co] * x[neighbour(v, tap)][c],
 * k = tap * cin + c < 27 * cin, co < cout; FP32 result.  The reduction
 * runs over chunksPerSplit * 64 voxels per CTA with FP32 partial tiles in
 * `workspace` (LBM_NNWgradWorkspaceBytes) summed in a fixed order. */
long long LBM_NNWgradWorkspaceBytes(int cin, int coutPad, int nb, int nz, int ny, int nx,
                                    int chunksPerSplit);
int LBM_NNConvWeightGrad(const void *x, int xStride, int xOff, int cin, const void *g,
                         int gStride, int cout, int coutPad, float *dw, int accumulate,
                         float *workspace, long long workspaceBytes, int chunksPerSplit, int nb,
                         int nz, int ny, int nx, void *stream);

/* Synchronises the device; LBM_ERR_TIMEOUT if a convolution kernel gave up
 * waiting for its tensor-core work since the last call, else LBM_OK. */
int LBM_NNTakeError(void);

/* Which convolution kernels LBM_NNConvForward, LBM_NNConvWeightGrad and
 * the network use: 0 (default) the halo-tiled forward kernel wherever the
 * shape allows it (input channels a multiple of 16, NX a multiple of 8, NY
 * a multiple of 16, coutPad 16 / 32 / 48 / 64 / 96) and the cp.async-
 * pipelined im2col kernels elsewhere (and for every weight gradient); 1 the
 * original synchronous im2col kernels for every shape; 2 the pipelined
 * im2col kernels for every shape; 3 as 0 with the z-folded forward (three
 * z taps per MMA, coutPad 16 / 32 / 48) wherever the shape allows it, also where
 * 0 would not choose it for lack of parallelism.  Process-wide; not
 * thread-safe against concurrent launches.  LBM_OK or
 * LBM_ERR_INVALID_ARGUMENT. */
int LBM_NNSetConvPath(int path);

/* The warm-start network: a 4-level 3D conv encoder-decoder (8->16->32->64
 * ->128 channels and back, skip connections, ~1.9 M parameters, leaky ReLU)
 * mapping per-voxel (solid fraction, U, Re) at 1/4 of the grid's resolution
 * to ((rho - 1) / U^2, u / U).  BF16 activations and weights, FP32 master
 * weights, Adam; forward and backward run on the kernels above.  nx, ny, nz
 * are the network's resolution (multiples of 8); features are float
 * [batch][voxel][3] = (solid fraction, U, Re), targets and predictions
 * float [batch][voxel][4].  Parameters are packed layer by layer as
 * (w [cout][27 cin], b [cout]).  The *Device variants take device
 * pointers; the others host pointers.  All synchronise the network's
 * stream and return LBM_OK or an LBM_ERR_* code. */
typedef struct LBMWarmNet LBMWarmNet;
long long LBM_WarmNetParamCount(void);
LBMWarmNet *LBM_WarmNetCreate(int nx, int ny, int nz, int maxBatch, unsigned seed);
void LBM_WarmNetFree(LBMWarmNet *net);
int LBM_WarmNetGetParams(LBMWarmNet *net, float *host);
int LBM_WarmNetSetParams(LBMWarmNet *net, const float *host);
int LBM_WarmNetForward(LBMWarmNet *net, const float *features, int batch, float *pred);
int LBM_WarmNetForwardDevice(LBMWarmNet *net, const float *features, int batch, float *pred);
/* mean squared error and (gradHost != NULL) its gradient, packed like the
 * parameters */
int LBM_WarmNetLossGrad(LBMWarmNet *net, const float *features, const float *target, int batch,
                        double *loss, float *gradHost);
int LBM_WarmNetLossGradDevice(LBMWarmNet *net, const float *features, const float *target,
                              int batch, double *loss, float *gradHost);
/* one Adam step (beta 0.9 / 0.999) at learning rate lr; *loss before it */
int LBM_WarmNetTrainStep(LBMWarmNet *net, const float *features, const float *target, int batch,
                         float lr, double *loss);
int LBM_WarmNetTrainStepDevice(LBMWarmNet *net, const float *features, const float *target,
                               int batch, float lr, double *loss);
void *LBM_WarmNetGetStream(LBMWarmNet *net);
/* Predictions (LBM_WarmNetForward*, LBM_InitializeFromWarmNet) are
 * shift + scale * network output per channel; training targets are given
 * in the network's normalised units, (target - shift) / scale.  Default
 * scale 1, shift 0. */
int LBM_WarmNetSetOutputScaling(LBMWarmNet *net, const float *scale4, const float *shift4);
/* Scale each training step's gradient by min(1, maxNorm / ||g||) (global
 * L2 norm over all parameters); 0 turns clipping off (the default). */
int LBM_WarmNetSetGradClip(LBMWarmNet *net, float maxNorm);
/* Features / targets of a grid at 1/factor resolution into device arrays:
 * solid fraction of each factor^3 block with U and Re; block means of
 * ((rho - 1) / U^2, u / U) over fluid cells (solid cells count as rho = 1,
 * u = 0) of the grid's current velocity field. */
int LBM_WarmNetGridFeatures(LBMGrid *grid, int factor, float U, float Re, float *featDev);
int LBM_WarmNetGridTargets(LBMGrid *grid, int factor, float U, float *targetDev);
/* Warm start: run the network on the grid's mask (grid = factor x network
 * resolution on every axis), interpolate its prediction trilinearly to the
 * grid, and initialise f = f_new = feq(rho, u) (solid cells rho = 1, u = 0)
 * -- LBM_InitializeFlow with a predicted field instead of a uniform one.
 * flags: LBM_WARM_UNIFORM_DENSITY keeps rho = 1 and takes only the
 * predicted velocity; LBM_WARM_FLUX_CORRECT then shifts u_x in every
 * x-plane so that it carries the inlet mass flux U * NY * NZ and shifts rho
 * so that the outlet plane's mean is 1 (continuity of the initial field,
 * which otherwise launches a tunnel-length pressure wave). */
#define LBM_WARM_UNIFORM_DENSITY 1
#define LBM_WARM_FLUX_CORRECT 2
int LBM_InitializeFromWarmNet(LBMGrid *grid, LBMWarmNet *net, float U, float Re, int flags);

/* ---------------------------------------------------------------------
 * Host side of the driver: OBJ ingestion, model placement, Re -> tau,
 * Strouhal number.  Plain C on the host, no device work.
 * ------------------------------------------------------------------- */

/* Same layout as the reference's Model (obj-file-loader/lib/model_loader.h:
 * 4-18): vertices x,y,z per vertex, faces three 1-based indices per face. */
typedef struct {
    float *vertices;
    int *faces;
    int vertexCount;
    int faceCount;
} LBMModel;

/* Replaces loadOBJ (obj-file-loader/lib/model_loader.c:54-151): "v x y z"
 * lines, "f a b c" lines in any of v, v/vt, v/vt/vn, v//vn; only the first
 * three references of a face are kept.  Returns 1, or 0 when the file
 * cannot be opened. */
int LBM_LoadOBJ(const char *path, LBMModel *model);
/* Replaces freeModel (model_loader.c:153-160). */
void LBM_FreeModel(LBMModel *model);

/* Replaces computeModelBounds (src/model_bounds.c:146-209): bounds9 =
 * {minX,minY,minZ, maxX,maxY,maxZ, centerX,centerY,centerZ} of the
 * vertices scaled, offset and rotated by rotationY degrees about y. */
int LBM_ModelBounds(const LBMModel *model, float scale, float offsetX, float offsetY,
                    float offsetZ, float rotationY, float *bounds9);

/* Replaces createTriangleBuffer (src/model_bounds.c:211-287): 12 floats per
 * valid face (three xyz+pad vertices, the layout LBM_SetSolidMesh takes);
 * faces with an index out of range are skipped.  Free with
 * LBM_FreeTriangles. */
float *LBM_CreateTriangleBuffer(const LBMModel *model, float scale, float offsetX,
                                float offsetY, float offsetZ, float rotationY,
                                int *outCount);
void LBM_FreeTriangles(float *triangles);

/* The placement main.c applies after loading (src/main.c:250-349): scale
 * 2.4 / largest raw extent unless scaleOrZero > 0, centre at the origin,
 * rotate 90 degrees about y when z is longer than x, centre at x = -2. */
int LBM_PlaceModel(const LBMModel *model, float scaleOrZero, float *scale, float *offset3,
                   float *rotationY);

/* src/main.c:447-460: nu = U L / Re, tau = 3 nu + 0.5, clamped at 0.52
 * (then Re = U L / nu).  Returns 1, 2 when clamped, 0 on bad arguments. */
int LBM_ReynoldsToTau(float latticeVelocity, float charLength, float reynolds, float *tau,
                      float *viscosity, float *effectiveReynolds);

/* Replaces compute_strouhal (src/drag_metrics.c:8-68) with the sample
 * interval as an argument (CD_SAMPLE_INTERVAL = 20 in the reference) and
 * the result returned instead of printed: St = f_peak L / U from a
 * Hann-windowed DFT of the last 65 % of the Cl series. */
float LBM_Strouhal(const float *clSeries, int clCount, int lbmSubsteps, int sampleInterval,
                   float charLength, float latticeVelocity, float *peakFrequency);

/* ---------------------------------------------------------------------
 * Headless wind-tunnel driver: the solver loop of the reference's main()
 * without rendering (src/main.c:438-553, 893-1391).  Its stdout lines keep
 * the reference's formats, so scripts that scrape the reference's binary
 * (modal_worker.py:474-560, test/benchmark.sh:57-79) read it unchanged.
 * ------------------------------------------------------------------- */
#define LBM_CD_SAMPLE_INTERVAL 20 /* frames between Cd samples (drag_metrics.h:5) */
#define LBM_CD_HISTORY_SIZE 100   /* samples in the convergence window (drag_metrics.h:4) */
#define LBM_RAMP_FRAMES 300       /* inlet ramp length in frames (main.c:944) */

/* Cd convergence monitor (main.c:1309-1391): EMA of the corrected Cd
 * (alpha 0.1, seeded while no sample has been accepted), ring of the last
 * 100 accepted Cd values (0 < Cd < 1000), converged once their relative
 * standard deviation drops below 1 %. */
typedef struct {
    float history[LBM_CD_HISTORY_SIZE];
    int historyCount;
    int converged;
    float ema;
    float convergedMean;
    float convergedRelStd;
} LBMCdMonitor;

void LBM_CdMonitorInit(LBMCdMonitor *m);
/* Add one sample; returns 1 when this sample made the series converge. */
int LBM_CdMonitorAdd(LBMCdMonitor *m, float cd, float cdCorr);

/* Coefficients of one sample (main.c:1256-1270): dynamic pressure
 * 0.5 rho0 U^2 with rho0 = 1, Cd = |Fx| / (q A), Cl = Fy / (q A) (signed),
 * Cd_pressure = |Px| / (q A), Cd_friction = max(Cd - Cd_pressure, 0),
 * Cd_corr = Cd * blockageFactor. */
typedef struct {
    float cd, cdCorr, cl, cdPressure, cdFriction;
} LBMCoefficients;
void LBM_TunnelCoefficients(float fx, float fy, float px, float latticeVelocity, float refArea,
                            float blockageFactor, LBMCoefficients *out);

/* First frame that samples Cd (main.c:968-981): 300 ramp frames plus three
 * flow-throughs, pulled back to 2/3 of a short run's frame budget. */
int LBM_TunnelCdStartFrame(int sizeX, float latticeVelocity, int substeps, int maxFrames);

/* Inlet ramp factor of a frame (main.c:944-947): frame / 300, then 1. */
float LBM_TunnelRampFactor(int frame);

typedef struct {
    const char *modelPath;   /* OBJ file; NULL or "" = no mesh (AABB fallback box) */
    float windSpeed;         /* 0-5; Re = 200 * wind (at least 50) when reynolds <= 0 */
    int renderDuration;      /* seconds of output at 60 frames/s (> 0) */
    float reynolds;          /* <= 0: derived from windSpeed */
    float scale;             /* <= 0: auto scale 2.4 / largest extent */
    int gridX, gridY, gridZ; /* 128 x 64 x 64 in the reference */
    float smagorinskyCs;     /* 0.1 in the reference */
    int substeps;            /* lattice steps per frame, 10 in the reference */
    float latticeVelocity;   /* 0.05 in the reference */
    const char *vtkOutputPath; /* NULL or "": no VTI dumps */
    int vtkInterval;         /* frames between VTI dumps */
    const char *logPath;     /* NULL or "": stdout; else the lines go to this file */
    int storage;             /* LBM_STORAGE_* of the populations */
} LBMTunnelOptions;

/* The reference's defaults (cli.c:12-39, main.c:59,434). */
void LBM_TunnelDefaults(LBMTunnelOptions *o);

typedef struct {
    int frames;              /* frames run */
    long long latticeSteps;  /* frames * substeps */
    int cdSamples;           /* Cd lines printed */
    int cdStartFrame;
    float tau, viscosity, reynolds, charLength;
    float refArea, blockage, blockageFactor;
    float lastCd, lastCdCorr, lastCl, cdEma;
    int converged;
    float convergedMean;
    float strouhal, sheddingFrequency;
    double seconds;          /* wall time of the frame loop */
    double mlups;            /* lattice updates / s / 1e6 over the frame loop */
    int solidCells;
    int triangles;
} LBMTunnelResult;

/* Run the headless loop: load and place the model, set the mesh, Re -> tau,
 * MRT + Smagorinsky + periodic y/z, ramped inlet, Cd every 20 frames after
 * the start frame, EMA and convergence (which shortens the run to 120 more
 * frames), Strouhal at the end.  Returns LBM_OK or an LBM_ERR_* code. */
int LBM_TunnelRun(const LBMTunnelOptions *options, LBMTunnelResult *result);

/* ---------------------------------------------------------------------
 * Super-resolution upscaling of the velocity field: the reference's
 * SR_* API (simulation/lib/superres.h, simulation/src/superres.c:178-285,
 * simulation/shaders/superres_upscale.comp).  Per coarse cell, the 3x3x3
 * neighbourhood of (ux, uy, uz, rho) -- clamped at the grid faces,
 * normalised by the channel mean and std -- feeds an MLP 108 -> 128 -> 128
 * -> 128 -> 32 (ReLU between layers) whose output corrects a trilinear
 * estimate of the 2x2x2 fine cells; the sum is denormalised and written to
 * the fine field (2x the coarse size in each direction).  The MLP runs on
 * the tensor cores with BF16 operands and FP32 accumulation.
 * ------------------------------------------------------------------- */
typedef struct LBMSuperRes LBMSuperRes;

/* SR_Create (superres.c:178-236): weights from an LTWS file (magic "LTWS",
 * version, parameter count, then per parameter its rank, shape and FP32
 * values: b0, W0, b1, W1, b2, W2, b3, W3 -- superres.c:43-101), the channel
 * mean[4] and std[4] from normPath (two FP32 vec4; a missing file means mean
 * 0 and std 1, as the reference does, superres.c:103-127).  NULL when the
 * weights cannot be read or do not have the 51,104 values of this network,
 * or when an allocation fails. */
LBMSuperRes *LBM_SuperResCreate(int coarseX, int coarseY, int coarseZ, const char *weightsPath,
                                const char *normPath);
/* The same from host arrays: `weights` holds the 51,104 values in the file's
 * order, mean and std 4 values each. */
LBMSuperRes *LBM_SuperResCreateFromArrays(int coarseX, int coarseY, int coarseZ,
                                          const float *weights, long long count,
                                          const float *mean, const float *std);
/* SR_Free (superres.c:238-244); accepts NULL. */
void LBM_SuperResFree(LBMSuperRes *sr);
/* SR_Upscale (superres.c:246-274): `coarseVelocity` is a device array of
 * coarseX*coarseY*coarseZ vec4 (ux, uy, uz, rho) -- LBM_GetVelocityBuffer of a
 * grid of that size -- and the fine field is written on `stream` (a
 * cudaStream_t, NULL for the legacy default stream), asynchronously.
 * Returns LBM_OK, LBM_ERR_INVALID_ARGUMENT or LBM_ERR_CUDA. */
int LBM_SuperResUpscale(LBMSuperRes *sr, const float *coarseVelocity, void *stream);
/* SR_GetFineVelocityBuffer (superres.c:276-278): the device fine field,
 * fineX*fineY*fineZ vec4, cell = x + fineX*(y + fineY*z). */
const float *LBM_SuperResGetFineVelocity(LBMSuperRes *sr);
/* SR_GetFineSize (superres.c:280-285). */
void LBM_SuperResGetFineSize(LBMSuperRes *sr, int *fineX, int *fineY, int *fineZ);
/* Copy the fine field to host memory (4 floats per fine cell) after the
 * device is done with it; also reports a tensor-core wait that gave up
 * (LBM_ERR_TIMEOUT).  Returns LBM_OK or an LBM_ERR_* code. */
int LBM_SuperResCopyFine(LBMSuperRes *sr, float *host);

#ifdef __cplusplus
}
#endif
#endif
