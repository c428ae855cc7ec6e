/*
 * CPU oracle for the D3Q19 wind-tunnel hot path of Lattice
 * (MarcosAsh/Lattice_Fluid_Dynamics).
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the
 * reference's OpenGL compute shaders and of the host geometry code in
 * simulation/src/lbm.c.  It is the parity checker for the CUDA library
 * and the timed CPU baseline; nothing in the product links it.  Only the
 * test-suite, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load it.
 *
 * Layout follows the reference exactly: populations are AoS
 * f[i + 19*cell], cell = x + NX*(y + NY*z); velocity is vec4 (ux,uy,uz,rho)
 * per cell; solid is int32 per cell (0 fluid, 1 body, 2 ground); q is the
 * dense Bouzidi table q[i + 19*cell] with -1 meaning "no link".
 *
 * Two arithmetic precisions share one source (oracle_core.inc): FP32
 * (bit-for-bit the shader arithmetic written as IEEE single operations,
 * compiled with -ffp-contract=off) and FP64 (the same operation order in
 * double, the "FP64 oracle" for the reduced-precision storage variants).
 *
 * Parity pins: the known-answer tests of simulation/test/test_lbm.c:191-366
 * (weights, equilibrium moments, MRT transforms) run against this code in
 * tests/test_oracle_kat.py; feq and the two MRT transforms are required to
 * equal, bit for bit, the reference's own CPU mirrors of them
 * (test_lbm.c:43-187, compiled by `make -C oracle ref`) in
 * tests/test_ref_math_cpu.py, against the fixture tests/golden/
 * ref_math.json that tests/golden/make_ref_math.py made from them.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OrGrid {
    int nx, ny, nz;
    int64_t n;                /* total cells */
    float tau;
    int useRegularized;
    int useMRT;
    int useSmagorinsky;
    float smagorinskyCs;
    int periodicYZ;
    int prec;                 /* 4 = FP32 storage/compute, 8 = FP64 */
    void *f;                  /* [19*n] REAL, post-stream populations      */
    void *f_new;              /* [19*n] REAL, post-collision populations   */
    void *vel;                /* [4*n]  REAL, (ux,uy,uz,rho) pre-collision */
    int32_t *solid;           /* [n] */
    float *q;                 /* [19*n] */
    int64_t force_raw[7];     /* last force pass: x,y,z,count,px,py,pz (x1e4 ints) */
    double force_f64[6];      /* last force pass summed in FP64: fx,fy,fz,px,py,pz */
    int64_t guard_resets;     /* cells reset by the stability guard (cumulative) */
} OrGrid;

/* lbm.c:46-318 (tau clamp [0.52, 2.0]; buffers zeroed; q = -1) */
OrGrid *or_create(int nx, int ny, int nz, float viscosity, int prec);
void or_free(OrGrid *g);
void or_set_threads(int n);

/* lbm.c:346-435 */
void or_set_solid_aabb(OrGrid *g, float minX, float minY, float minZ,
                       float maxX, float maxY, float maxZ);
/* lbm.c:437-535; halfway != 0 writes q = 0.5 on every link instead of the
 * analytic ray-sphere distance (half-way bounce-back) */
void or_set_solid_sphere(OrGrid *g, float cx, float cy, float cz, float r,
                         int halfway);
/* lbm.c:537-614 */
void or_add_ground_plane(OrGrid *g, float worldZ);
/* lbm.c:964-1223; tris are 12 floats each (GPUTriangle, model_bounds.h:14-18) */
void or_set_solid_mesh(OrGrid *g, const float *tris, int ntris, float minX,
                       float minY, float minZ, float maxX, float maxY,
                       float maxZ);
/* lbm.c:616-668 */
float or_projected_area(OrGrid *g, int axis);
/* lbm.c:670-721 */
int or_initialize_flow(OrGrid *g, float ux, float uy, float uz);

/* lbm.c:723-821 -> lbm_collide.comp:313-626 then lbm_stream.comp:76-129 */
void or_step(OrGrid *g, float inX, float inY, float inZ);
/* the two halves of a step, for staged comparisons */
void or_collide(OrGrid *g, float inX, float inY, float inZ);
void or_stream(OrGrid *g);

/* lbm.c:835-918 -> lbm_force.comp:94-151.  out6 = fx,fy,fz,px,py,pz as the
 * reference returns them (int sum / 10000.0f). */
void or_drag_force_decomposed(OrGrid *g, float *out6);
/* lbm.c:920-962 (note: lift uses |Fy| exactly like lbm.c:949) */
float or_drag_coefficient(OrGrid *g, float U, float A);
float or_lift_coefficient(OrGrid *g, float U, float A);

/* ---- scalar building blocks, exported for the known-answer tests ---- */
float or_feq_f32(int i, float rho, float ux, float uy, float uz);
double or_feq_f64(int i, double rho, double ux, double uy, double uz);
void or_mrt_forward_f32(const float *fi, float *m);
void or_mrt_inverse_f32(const float *m, float *fi);
void or_mrt_meq_f32(float rho, float ux, float uy, float uz, float *meq);
float or_weight_f32(int i);
/* batched over n states (state = rho, ux, uy, uz; 19 values per state out) */
void or_feq_batch_f32(int64_t n, const float *state, float *out);
void or_mrt_forward_batch_f32(int64_t n, const float *fi, float *m);
void or_mrt_inverse_batch_f32(int64_t n, const float *m, float *fi);

/* ---- particles (particle_lbm.comp:46-89 sampler, :207-293 Euler step,
 * collisionMode 0).  Particle = 8 floats {x,y,z,pad,vx,vy,vz,life}.  The
 * respawn position uses the counter hash below instead of the shader's
 * fract(sin()) so CPU and GPU agree bit for bit. ---- */
uint32_t or_hash3(uint32_t seed, uint32_t idx, uint32_t k);
float or_uniform01(uint32_t seed, uint32_t idx, uint32_t k);
void or_particles_seed_inlet(float *p, int n, uint32_t seed);
void or_particles_step(const float *vel4, int nx, int ny, int nz, float *p,
                       int n, float dt, uint32_t seed);

/* ---- VTK ImageData writer (vti_export.c:10-116) from host arrays ---- */
int or_write_vti(const char *filename, int nx, int ny, int nz,
                 const float *vel4, const int32_t *solid);

#ifdef __cplusplus
}
#endif
#endif
