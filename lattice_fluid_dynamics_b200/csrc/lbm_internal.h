// Internal device state of an LBMGrid and the launchers shared by the
// translation units of the library.  Not part of the public ABI.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/lattice_lbm.h"

namespace lbm {

// collision operators (lbm_collide.comp:488-625)
enum { OP_BGK = 0, OP_REG = 1, OP_MRT = 2 };

// Compacted boundary-link structure.  A boundary cell is a cell owning at
// least one link with q >= 0 (the reference's dense q table entry for
// (cell, dir)).  Links are stored sorted by (cell, dir); a boundary cell b
// owns links [first[b], first[b+1]) and `mask[b]` has bit d set for each
// linked direction d, so the link of direction d is
// first[b] + popc(mask[b] & ((1 << d) - 1)).
struct LinkList {
    int nb = 0;              // boundary cells
    long long nl = 0;        // links
    int32_t *bcell = nullptr;   // [nb]
    uint32_t *bmask = nullptr;  // [nb]
    int32_t *bfirst = nullptr;  // [nb + 1]
    float *lq = nullptr;        // [nl]
    int32_t *lcell = nullptr;   // [nl]
    int32_t *ldir = nullptr;    // [nl]
};

// What the population buffers hold.
//   - `g` (index gbuf) always holds post-collision populations f_new.
//   - When fbuf >= 0, buffer fbuf holds explicit post-stream f; otherwise
//     f is implicit: f = Stream(g) with the links and periodic flag of the
//     step that produced g.
//   - The velocity field of the last step is derived from that step's
//     input (buffer `vin`, kind `vin_kind`) until it is materialised in
//     `vel` (vel_valid).
enum InputKind { IN_EXPLICIT_F = 0, IN_POST_COLLISION = 1 };

struct GridImpl {
    int nx = 0, ny = 0, nz = 0;
    long long n = 0;
    int storage = LBM_STORAGE_FP32;
    size_t elem = 4;          // bytes per stored population
    cudaStream_t stream = nullptr;

    void *pop[2] = {nullptr, nullptr};  // SoA planes pop[i * n + cell]
    float4 *vel = nullptr;
    double4 *vel64 = nullptr;           // FP64 grids: full-precision copy of vel
    int32_t *solid = nullptr;
    uint8_t *flags = nullptr;
    int32_t *slot = nullptr;            // boundary-cell index or -1
    LinkList links;

    long long *force_i64 = nullptr;     // [7] of a 16-slot block
    double *force_f64 = nullptr;        // [6], slots 8.. of the same block
    unsigned *force_ticket = nullptr;   // slot 15 of the same block
    long long *force_part = nullptr;    // 16 slots per k_force block
    int force_part_blocks = 0;
    double *sums_f64 = nullptr;         // [4]
    unsigned long long *guard = nullptr;  // cumulative guard resets
    int *err_flag = nullptr;            // device-side error word
    long long *host_pinned = nullptr;   // small pinned readback area (64 B)

    bool initialized = false;
    int gbuf = 1;
    int fbuf = 0;             // -1 when f is implicit
    int stream_periodic = 0;  // periodic flag of the stream that turns g into f
    bool vel_valid = true;
    int vin = 0;
    int vin_kind = IN_EXPLICIT_F;
    int vin_periodic = 0;     // periodic flag of the stream feeding vin (post-collision kind)
    float vin_inlet[3] = {0, 0, 0};

    // launch configuration of the step kernel: block shape and cells per
    // thread along x (cpt = 2: the paired kernel, with pbx threads along x
    // and 128 / pbx rows per block)
    int bx = 128, by = 1, cpt = 1, minb = 1;
    int pbx = 32;

    // CUDA graphs for LBM_StepN, one per starting buffer parity (gbuf)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int graph_key[2][8] = {{0}, {0}};

    // TMA descriptors of the two population buffers as rank-4 tensors
    // (x, y, z, direction); `tma` is set when they could be made (FP32 /
    // FP16 / BF16 storage, rows a multiple of 16 bytes)
    alignas(64) CUtensorMap tmap[2];
    bool tma = false;
};

// The fused step with the pull neighbourhood staged in shared memory by TMA
// (k_step_tma): tiles of 32 x TMA_BOX_Y cells, TMA_ZSEG z-planes per block.
// The box of one direction spans the tile's 32 x plus tma_xpad() elements on
// either side, so that its first x is a 16-byte multiple.
constexpr int TMA_BOX_Y = 8, TMA_ZSEG = 8;
__host__ __device__ constexpr int tma_xpad(size_t elem) { return (int)(16 / elem); }
__host__ __device__ constexpr int tma_box_x(size_t elem) { return 32 + 2 * tma_xpad(elem); }
__host__ __device__ constexpr int tma_stage_bytes(size_t elem) {
    return 19 * tma_box_x(elem) * TMA_BOX_Y * (int)elem;
}
// dynamic shared memory of one block: barriers, alignment slack, 2 stages
__host__ __device__ constexpr int tma_smem_bytes(size_t elem) {
    return 256 + 2 * tma_stage_bytes(elem);
}

struct StepArgs {
    const void *src;   // populations read (post-collision g or explicit f)
    void *dst;         // populations written (post-collision)
    const uint8_t *flags;
    const int32_t *slot;
    const uint32_t *bmask;
    const int32_t *bfirst;
    const float *lq;
    int nx, ny, nz;
    long long n;
    int periodic;      // periodic flag of the stream part
    float tau, omega, smag18;   // omega = 1/tau, smag18 = 18*Cs*Cs (FP32 arithmetic)
    double omega_d, smag18_d;   // the same in FP64 arithmetic (FP64 storage)
    float inX, inY, inZ;
    unsigned long long *guard;
    int *err;          // device error word (bit 0: a TMA wait gave up)
};

// Per-launch element offsets of the fused step, computed on the host so
// that every address is a per-thread base plus a kernel-parameter constant:
// pull[i] = i*n - e_ix - e_iy*NX - e_iz*NX*NY (the pulled neighbour of an
// interior cell in plane i), dir[i] = i*n (plane i of the cell itself).
struct StepOffsets {
    long long pull[19];
    long long dir[19];
};

// Kernel parameter of the paired (two cells per thread) step: per-direction
// base pointers so that every access is a 32-bit cell index added to a
// parameter.
struct PairTable {
    const void *pull[19];  // src + i*n - (e_x + e_y NX + e_z NX NY): pulled value of an interior cell
    const void *own[19];   // src + i*n: the cell's own value in plane i
    void *dst[19];         // dst + i*n
    float2 nz;             // (-0, -0): addend of the paired products
};

// One grid of a batched paired step launch (k_step_batch_pair), kept in
// device memory (one table per buffer parity) and copied into shared memory
// by each block that works on the grid.  The kernel computes the
// per-direction pointers from a.src / a.dst and the extents.
struct alignas(16) BatchGridDev {
    StepArgs a;
    float2 nz;    // (-0, -0): addend of the paired products
    int combo;    // op * 2 + smagorinsky
    int lbx;      // 1 << lbx threads along x (two cells each), 128 >> lbx rows
    int tiles_x;
    int tiles_y;
};

// One grid of a batched step launch (k_step_batch): its step arguments,
// operator, and tile shape -- 1 << lbx cells along x (32..256) by
// 256 >> lbx rows, tiles_x * tiles_y tiles per z plane.
struct BatchEntry {
    StepArgs a;
    int combo;    // op * 2 + smagorinsky
    int lbx;
    int tiles_x;
    int tiles_y;
};

// Operator sets a batched kernel is compiled for: each single (op, smag)
// combination, BGK + regularized, and all six.
enum {
    BATCH_SET_BGK = 0, BATCH_SET_BGK_SMAG, BATCH_SET_REG, BATCH_SET_REG_SMAG, BATCH_SET_MRT,
    BATCH_SET_MRT_SMAG, BATCH_SET_BGK_REG, BATCH_SET_ALL
};
__host__ __device__ constexpr unsigned batch_set_mask(int set) {
    return set < 6 ? (1u << set) : set == BATCH_SET_BGK_REG ? 0x5u : 0x3fu;
}

// lbm_capi.cu: the grid state machine, for the batched driver
StepArgs grid_step_args(LBMGrid *grid, float inX, float inY, float inZ);
int grid_op(LBMGrid *grid);
bool grid_enqueue_step(LBMGrid *grid, float inX, float inY, float inZ);
// the state transition of k fused steps run outside the grid's own launcher
void grid_note_fused_steps(LBMGrid *grid, int k, float inX, float inY, float inZ);
bool grid_ok(LBMGrid *grid, cudaError_t e);
// materialise the velocity of the last step (after which the buffer that step
// read is free until the next step)
bool grid_ensure_velocity(LBMGrid *grid);
// f = f_new = feq(rho, u) from device fields rho[n], u[3n]; returns 1 or 0
int grid_init_from_device(LBMGrid *grid, const float *drho, const float *du);

// lbm_step.cu
// Arguments of one batched launch, passed by value as a kernel parameter
// (constant bank): up to BATCH_LAUNCH_MAX grids, work unit t (a column of
// BATCH_ZB z-planes of one tile) belonging to grid g with starts[g] <= t <
// starts[g + 1].
constexpr int BATCH_LAUNCH_MAX = 64;
constexpr int BATCH_ZB = 1;  // z-planes of one tile per thread block
struct BatchLaunchParams {
    BatchEntry e[BATCH_LAUNCH_MAX];
    unsigned starts[BATCH_LAUNCH_MAX + 1];
    int count;
};
cudaError_t launch_step_batch(int storage, const BatchLaunchParams &p, int set, cudaStream_t s);

// Arguments of one batched paired launch: the grids' entries in device
// memory, and work unit t (one tile of one z-plane) belonging to grid g with
// starts[g] <= t < starts[g + 1].
struct BatchPairParams {
    const BatchGridDev *grids;
    unsigned starts[BATCH_LAUNCH_MAX + 1];
    int count;
};
cudaError_t launch_step_batch_pair(int storage, const BatchPairParams &p, int set,
                                   cudaStream_t s);

// The launchers of one storage format and arithmetic flavour.  Each step
// translation unit (lbm_step_{f32,f16,bf16,f64}.cu, lbm_step_fast_*.cu)
// instantiates the kernels of its format and exports one table; the
// dispatcher (lbm_dispatch.cu) sees only these tables, so no kernel is
// compiled twice.
struct StepOps {
    cudaError_t (*step)(const GridImpl &, const StepArgs &, bool fused, int op, bool smag,
                        cudaStream_t);
    cudaError_t (*batch)(const BatchLaunchParams &, int set, cudaStream_t);
    cudaError_t (*batch_pair)(const BatchPairParams &, int set, cudaStream_t);
    cudaError_t (*tma_prepare)();
    cudaError_t (*stream_only)(const GridImpl &, const StepArgs &, cudaStream_t);
    cudaError_t (*velocity)(const GridImpl &, const StepArgs &, int kind, float4 *, double4 *,
                            cudaStream_t);
    cudaError_t (*init_uniform)(const GridImpl &, void *, void *, float, float, float,
                                cudaStream_t);
    cudaError_t (*init_field)(const GridImpl &, void *, void *, const float *, const float *,
                              cudaStream_t);
    cudaError_t (*export_aos)(const GridImpl &, const void *, void *, bool, cudaStream_t);
    cudaError_t (*import_aos)(const GridImpl &, const float *, void *, cudaStream_t);
    cudaError_t (*mass_momentum)(const GridImpl &, const void *, double *, cudaStream_t);
};
extern const StepOps step_ops_f32, step_ops_f16, step_ops_bf16, step_ops_f64;
extern const StepOps step_ops_fast_f32, step_ops_fast_f16, step_ops_fast_bf16;
cudaError_t launch_step(const GridImpl &g, const StepArgs &a, bool fused, int op, bool smag,
                        bool fast_arith, cudaStream_t s);
// Encode the grid's TMA descriptors and allow k_step_tma's shared memory;
// sets g.tma (false for FP64 storage or rows that are not a multiple of 16
// bytes, and, unless `force`, unless LBM_TMA=1 is set in the environment).
void setup_tma(GridImpl &g, bool force);
cudaError_t launch_stream_only(const GridImpl &g, const void *src, void *dst, int periodic,
                               cudaStream_t s);
cudaError_t launch_velocity(const GridImpl &g, const void *src, int kind, int periodic,
                            float inX, float inY, float inZ, float4 *vel, double4 *vel64,
                            cudaStream_t s);
cudaError_t launch_init_uniform(const GridImpl &g, void *a, void *b, float ux, float uy,
                                float uz, cudaStream_t s);
cudaError_t launch_init_field(const GridImpl &g, void *a, void *b, const float *rho,
                              const float *u, cudaStream_t s);
cudaError_t launch_export_aos(const GridImpl &g, const void *src, void *dst, bool as_double,
                              cudaStream_t s);
cudaError_t launch_import_aos(const GridImpl &g, const float *src, void *dst, cudaStream_t s);
cudaError_t launch_mass_momentum(const GridImpl &g, const void *f_explicit, double *out4,
                                 cudaStream_t s);

// lbm_geometry.cu
cudaError_t geo_fill_q(float *qd, long long n19, cudaStream_t s);
cudaError_t geo_links_to_dense(const GridImpl &g, float *qd, cudaStream_t s);
cudaError_t geo_aabb(GridImpl &g, float *qd, float minX, float minY, float minZ, float maxX,
                     float maxY, float maxZ, cudaStream_t s);
cudaError_t geo_sphere(GridImpl &g, float *qd, float cx, float cy, float cz, float r,
                       bool halfway, cudaStream_t s);
cudaError_t geo_ground(GridImpl &g, float *qd, float worldZ, cudaStream_t s);
cudaError_t geo_mesh(GridImpl &g, float *qd, const float *tris_dev, int ntris,
                     const float bbox[6], cudaStream_t s);
cudaError_t geo_compact(GridImpl &g, const float *qd, cudaStream_t s);
cudaError_t geo_projected_area(const GridImpl &g, int axis, int *count_dev, cudaStream_t s);
void geo_free_links(LinkList &l);

// lbm_force.cu
cudaError_t launch_force(const GridImpl &g, const void *gsrc, const void *f_explicit,
                         int periodic, const float4 *vel_or_null, const double4 *vel64_or_null,
                         const void *vin_src,
                         int vin_kind, int vin_periodic, const float vin_inlet[3],
                         long long *i64, double *f64, long long *part, unsigned *ticket,
                         cudaStream_t s);
// blocks of one k_force launch over nb boundary cells (16 partial slots each)
int force_blocks(int nb);

// lbm_particles.cu
cudaError_t launch_particles(LBMParticle *p, int n, const float4 *vel, int nx, int ny, int nz,
                             float dt, uint32_t seed, cudaStream_t s);
void particles_seed_host(LBMParticle *p, int n, uint32_t seed);

}  // namespace lbm
