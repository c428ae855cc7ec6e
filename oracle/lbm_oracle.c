/*
 * CPU oracle for the Lattice D3Q19 hot path (TEST INFRASTRUCTURE ONLY;
 * see lbm_oracle.h).  Build: oracle/Makefile (-O2 -ffp-contract=off).
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* D3Q19 velocity set and opposites (lbm_collide.comp:33-77, lbm.c:30-35) */
static const int EX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
static const int EY[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
static const int EZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
static const int OPP[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};

/* FP32 instantiation */
#define REAL float
#define SFX(name) name##_f32
#define SQRT sqrtf
#define RINT rintf
#include "oracle_core.inc"
#undef REAL
#undef SFX
#undef SQRT
#undef RINT

/* FP64 instantiation */
#define REAL double
#define SFX(name) name##_f64
#define SQRT sqrt
#define RINT rint
#include "oracle_core.inc"
#undef REAL
#undef SFX
#undef SQRT
#undef RINT

void or_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0)
        omp_set_num_threads(n);
#else
    (void)n;
#endif
}

OrGrid *or_create(int nx, int ny, int nz, float viscosity, int prec) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || (prec != 4 && prec != 8))
        return NULL;
    OrGrid *g = (OrGrid *)calloc(1, sizeof(OrGrid));
    if (!g)
        return NULL;
    g->nx = nx;
    g->ny = ny;
    g->nz = nz;
    g->n = (int64_t)nx * ny * nz;
    g->prec = prec;
    /* lbm.c:56-60 */
    g->tau = 0.5f + 3.0f * viscosity;
    if (g->tau < 0.52f)
        g->tau = 0.52f;
    if (g->tau > 2.0f)
        g->tau = 2.0f;
    /* lbm.c:272-276 */
    g->useRegularized = 0;
    g->useMRT = 0;
    g->useSmagorinsky = 0;
    g->smagorinskyCs = 0.1f;
    g->periodicYZ = 0;
    size_t n = (size_t)g->n;
    g->f = calloc(19 * n, (size_t)prec);
    g->f_new = calloc(19 * n, (size_t)prec);
    g->vel = calloc(4 * n, (size_t)prec);
    g->solid = (int32_t *)calloc(n, sizeof(int32_t));
    g->q = (float *)malloc(19 * n * sizeof(float));
    if (!g->f || !g->f_new || !g->vel || !g->solid || !g->q) {
        or_free(g);
        return NULL;
    }
    for (size_t i = 0; i < 19 * n; i++)
        g->q[i] = -1.0f;
    return g;
}

void or_free(OrGrid *g) {
    if (!g)
        return;
    free(g->f);
    free(g->f_new);
    free(g->vel);
    free(g->solid);
    free(g->q);
    free(g);
}

static inline int64_t cidx(const OrGrid *g, int x, int y, int z) {
    return (int64_t)x + (int64_t)y * g->nx + (int64_t)z * g->nx * g->ny;
}

static void reset_q(OrGrid *g) {
    for (int64_t i = 0; i < 19 * g->n; i++)
        g->q[i] = -1.0f;
}

/* lbm.c:346-435 */
void or_set_solid_aabb(OrGrid *g, float minX, float minY, float minZ,
                       float maxX, float maxY, float maxZ) {
    float scaleX = g->nx / 8.0f;
    float scaleY = g->ny / 4.0f;
    float scaleZ = g->nz / 4.0f;
    int gMinX = (int)((minX + 4.0f) * scaleX);
    int gMaxX = (int)((maxX + 4.0f) * scaleX);
    int gMinY = (int)((minY + 2.0f) * scaleY);
    int gMaxY = (int)((maxY + 2.0f) * scaleY);
    int gMinZ = (int)((minZ + 2.0f) * scaleZ);
    int gMaxZ = (int)((maxZ + 2.0f) * scaleZ);
    if (gMinX < 0) gMinX = 0;
    if (gMaxX >= g->nx) gMaxX = g->nx - 1;
    if (gMinY < 0) gMinY = 0;
    if (gMaxY >= g->ny) gMaxY = g->ny - 1;
    if (gMinZ < 0) gMinZ = 0;
    if (gMaxZ >= g->nz) gMaxZ = g->nz - 1;

    memset(g->solid, 0, (size_t)g->n * sizeof(int32_t));
    for (int z = gMinZ; z <= gMaxZ; z++)
        for (int y = gMinY; y <= gMaxY; y++)
            for (int x = gMinX; x <= gMaxX; x++)
                g->solid[cidx(g, x, y, z)] = 1;

    reset_q(g);
    for (int gz = 0; gz < g->nz; gz++)
        for (int gy = 0; gy < g->ny; gy++)
            for (int gx = 0; gx < g->nx; gx++) {
                int64_t ci = cidx(g, gx, gy, gz);
                if (g->solid[ci] == 1)
                    continue;
                for (int i = 1; i < 19; i++) {
                    int nx = gx + EX[i], ny = gy + EY[i], nz = gz + EZ[i];
                    if (nx < 0 || nx >= g->nx || ny < 0 || ny >= g->ny ||
                        nz < 0 || nz >= g->nz)
                        continue;
                    if (g->solid[cidx(g, nx, ny, nz)] == 1)
                        g->q[ci * 19 + i] = 0.5f;
                }
            }
}

/* lbm.c:437-535 */
void or_set_solid_sphere(OrGrid *g, float cx, float cy, float cz, float radius,
                         int halfway) {
    float scaleX = g->nx / 8.0f;
    float scaleY = g->ny / 4.0f;
    float scaleZ = g->nz / 4.0f;
    memset(g->solid, 0, (size_t)g->n * sizeof(int32_t));
    for (int gz = 0; gz < g->nz; gz++)
        for (int gy = 0; gy < g->ny; gy++)
            for (int gx = 0; gx < g->nx; gx++) {
                float wx = (gx + 0.5f) / scaleX - 4.0f;
                float wy = (gy + 0.5f) / scaleY - 2.0f;
                float wz = (gz + 0.5f) / scaleZ - 2.0f;
                float dx = wx - cx, dy = wy - cy, dz = wz - cz;
                if (dx * dx + dy * dy + dz * dz <= radius * radius)
                    g->solid[cidx(g, gx, gy, gz)] = 1;
            }

    reset_q(g);
    for (int gz = 0; gz < g->nz; gz++)
        for (int gy = 0; gy < g->ny; gy++)
            for (int gx = 0; gx < g->nx; gx++) {
                int64_t ci = cidx(g, gx, gy, gz);
                if (g->solid[ci] == 1)
                    continue;
                float wx = (gx + 0.5f) / scaleX - 4.0f;
                float wy = (gy + 0.5f) / scaleY - 2.0f;
                float wz = (gz + 0.5f) / scaleZ - 2.0f;
                for (int i = 1; i < 19; i++) {
                    int nx = gx + EX[i], ny = gy + EY[i], nz = gz + EZ[i];
                    if (nx < 0 || nx >= g->nx || ny < 0 || ny >= g->ny ||
                        nz < 0 || nz >= g->nz)
                        continue;
                    if (g->solid[cidx(g, nx, ny, nz)] != 1)
                        continue;
                    float q = 0.5f;
                    if (!halfway) {
                        float dx = (float)EX[i] / scaleX;
                        float dy = (float)EY[i] / scaleY;
                        float dz = (float)EZ[i] / scaleZ;
                        float ox = wx - cx, oy = wy - cy, oz = wz - cz;
                        float a = dx * dx + dy * dy + dz * dz;
                        float b = 2.0f * (ox * dx + oy * dy + oz * dz);
                        float c = ox * ox + oy * oy + oz * oz - radius * radius;
                        float disc = b * b - 4.0f * a * c;
                        if (disc >= 0.0f) {
                            float t = (-b - sqrtf(disc)) / (2.0f * a);
                            if (t > 0.0f && t <= 1.0f)
                                q = t;
                        }
                        if (q < 0.01f)
                            q = 0.01f;
                        if (q > 0.99f)
                            q = 0.99f;
                    }
                    g->q[ci * 19 + i] = q;
                }
            }
}

/* lbm.c:537-614 */
void or_add_ground_plane(OrGrid *g, float worldZ) {
    float scaleZ = g->nz / 4.0f;
    int gzGround = (int)((worldZ + 2.0f) * scaleZ);
    if (gzGround < 0)
        gzGround = 0;
    if (gzGround >= g->nz)
        gzGround = g->nz - 1;
    for (int gz = 0; gz <= gzGround; gz++)
        for (int gy = 0; gy < g->ny; gy++)
            for (int gx = 0; gx < g->nx; gx++) {
                int64_t idx = cidx(g, gx, gy, gz);
                if (g->solid[idx] == 0)
                    g->solid[idx] = 2;
            }
    int gzAbove = gzGround + 1;
    if (gzAbove < g->nz) {
        for (int gy = 0; gy < g->ny; gy++)
            for (int gx = 0; gx < g->nx; gx++) {
                int64_t ci = cidx(g, gx, gy, gzAbove);
                if (g->solid[ci] != 0)
                    continue;
                for (int i = 1; i < 19; i++) {
                    if (EZ[i] != -1)
                        continue;
                    int nz = gzAbove + EZ[i];
                    int ny = gy + EY[i], nx = gx + EX[i];
                    if (nx < 0 || nx >= g->nx || ny < 0 || ny >= g->ny || nz < 0)
                        continue;
                    int64_t ni = cidx(g, nx, ny, nz);
                    if (g->solid[ni] != 0 && g->q[ci * 19 + i] < 0.0f)
                        g->q[ci * 19 + i] = 0.5f;
                }
            }
    }
}

/* lbm.c:616-668 */
float or_projected_area(OrGrid *g, int axis) {
    int count = 0;
    if (axis == 0) {
        for (int gz = 0; gz < g->nz; gz++)
            for (int gy = 0; gy < g->ny; gy++) {
                int found = 0;
                for (int gx = 0; gx < g->nx && !found; gx++)
                    if (g->solid[cidx(g, gx, gy, gz)] == 1)
                        found = 1;
                count += found;
            }
    } else if (axis == 1) {
        for (int gz = 0; gz < g->nz; gz++)
            for (int gx = 0; gx < g->nx; gx++) {
                int found = 0;
                for (int gy = 0; gy < g->ny && !found; gy++)
                    if (g->solid[cidx(g, gx, gy, gz)] == 1)
                        found = 1;
                count += found;
            }
    } else {
        for (int gy = 0; gy < g->ny; gy++)
            for (int gx = 0; gx < g->nx; gx++) {
                int found = 0;
                for (int gz = 0; gz < g->nz && !found; gz++)
                    if (g->solid[cidx(g, gx, gy, gz)] == 1)
                        found = 1;
                count += found;
            }
    }
    return (float)count;
}

/* lbm.c:964-1223 */
void or_set_solid_mesh(OrGrid *g, const float *triangles, int numTriangles,
                       float minX, float minY, float minZ, float maxX,
                       float maxY, float maxZ) {
    typedef struct {
        float minY, maxY, minZ, maxZ, maxX;
    } TriBounds;
    TriBounds *tb = (TriBounds *)malloc((size_t)(numTriangles > 0 ? numTriangles : 1) *
                                        sizeof(TriBounds));
    if (!tb)
        return;
    for (int t = 0; t < numTriangles; t++) {
        const float *tri = &triangles[(size_t)t * 12];
        float v0y = tri[1], v0z = tri[2], v0x = tri[0];
        float v1y = tri[5], v1z = tri[6], v1x = tri[4];
        float v2y = tri[9], v2z = tri[10], v2x = tri[8];
        tb[t].minY = fminf(v0y, fminf(v1y, v2y));
        tb[t].maxY = fmaxf(v0y, fmaxf(v1y, v2y));
        tb[t].minZ = fminf(v0z, fminf(v1z, v2z));
        tb[t].maxZ = fmaxf(v0z, fmaxf(v1z, v2z));
        tb[t].maxX = fmaxf(v0x, fmaxf(v1x, v2x));
    }
    float scaleX = g->nx / 8.0f;
    float scaleY = g->ny / 4.0f;
    float scaleZ = g->nz / 4.0f;

    memset(g->solid, 0, (size_t)g->n * sizeof(int32_t));
    const int NX = g->nx, NY = g->ny, NZ = g->nz;
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int gz = 0; gz < NZ; gz++)
        for (int gy = 0; gy < NY; gy++)
            for (int gx = 0; gx < NX; gx++) {
                float wx = (gx + 0.5f) / scaleX - 4.0f;
                float wy = (gy + 0.5f) / scaleY - 2.0f;
                float wz = (gz + 0.5f) / scaleZ - 2.0f;
                if (wx < minX || wx > maxX || wy < minY || wy > maxY ||
                    wz < minZ || wz > maxZ)
                    continue;
                int intersections = 0;
                for (int t = 0; t < numTriangles; t++) {
                    if (wy < tb[t].minY || wy > tb[t].maxY || wz < tb[t].minZ ||
                        wz > tb[t].maxZ || wx > tb[t].maxX)
                        continue;
                    const float *tri = &triangles[(size_t)t * 12];
                    float v0x = tri[0], v0y = tri[1], v0z = tri[2];
                    float v1x = tri[4], v1y = tri[5], v1z = tri[6];
                    float v2x = tri[8], v2y = tri[9], v2z = tri[10];
                    float e1x = v1x - v0x, e1y = v1y - v0y, e1z = v1z - v0z;
                    float e2x = v2x - v0x, e2y = v2y - v0y, e2z = v2z - v0z;
                    float hx = 0, hy = -e2z, hz = e2y;
                    float a = e1x * hx + e1y * hy + e1z * hz;
                    if (a > -0.00001f && a < 0.00001f)
                        continue;
                    float f = 1.0f / a;
                    float sx = wx - v0x, sy = wy - v0y, sz = wz - v0z;
                    float u = f * (sx * hx + sy * hy + sz * hz);
                    if (u < 0.0f || u > 1.0f)
                        continue;
                    float qx = sy * e1z - sz * e1y;
                    float qy = sz * e1x - sx * e1z;
                    float qz = sx * e1y - sy * e1x;
                    float v = f * qx;
                    if (v < 0.0f || u + v > 1.0f)
                        continue;
                    float dist = f * (e2x * qx + e2y * qy + e2z * qz);
                    if (dist > 0.00001f)
                        intersections++;
                }
                if (intersections % 2 == 1)
                    g->solid[cidx(g, gx, gy, gz)] = 1;
            }

    reset_q(g);
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int gz = 0; gz < NZ; gz++)
        for (int gy = 0; gy < NY; gy++)
            for (int gx = 0; gx < NX; gx++) {
                int64_t cellIdx = cidx(g, gx, gy, gz);
                if (g->solid[cellIdx] == 1)
                    continue;
                float wx = (gx + 0.5f) / scaleX - 4.0f;
                float wy = (gy + 0.5f) / scaleY - 2.0f;
                float wz = (gz + 0.5f) / scaleZ - 2.0f;
                for (int i = 1; i < 19; i++) {
                    int nx = gx + EX[i], ny = gy + EY[i], nz = gz + EZ[i];
                    if (nx >= 0 && nx < g->nx && ny >= 0 && ny < g->ny &&
                        nz >= 0 && nz < g->nz) {
                        if (g->solid[cidx(g, nx, ny, nz)] == 0)
                            continue;
                    } else {
                        continue;
                    }
                    float dx = (float)EX[i] / scaleX;
                    float dy = (float)EY[i] / scaleY;
                    float dz = (float)EZ[i] / scaleZ;
                    float bestT = 2.0f;
                    for (int t = 0; t < numTriangles; t++) {
                        if (wy < tb[t].minY || wy > tb[t].maxY ||
                            wz < tb[t].minZ || wz > tb[t].maxZ ||
                            wx > tb[t].maxX)
                            continue;
                        const float *tri = &triangles[(size_t)t * 12];
                        float v0x = tri[0], v0y = tri[1], v0z = tri[2];
                        float v1x = tri[4], v1y = tri[5], v1z = tri[6];
                        float v2x = tri[8], v2y = tri[9], v2z = tri[10];
                        float e1x = v1x - v0x, e1y = v1y - v0y, e1z = v1z - v0z;
                        float e2x = v2x - v0x, e2y = v2y - v0y, e2z = v2z - v0z;
                        float hx = dy * e2z - dz * e2y;
                        float hy = dz * e2x - dx * e2z;
                        float hz = dx * e2y - dy * e2x;
                        float a = e1x * hx + e1y * hy + e1z * hz;
                        if (a > -1e-6f && a < 1e-6f)
                            continue;
                        float f = 1.0f / a;
                        float sx = wx - v0x, sy = wy - v0y, sz = wz - v0z;
                        float u = f * (sx * hx + sy * hy + sz * hz);
                        if (u < 0.0f || u > 1.0f)
                            continue;
                        float qx = sy * e1z - sz * e1y;
                        float qy = sz * e1x - sx * e1z;
                        float qz = sx * e1y - sy * e1x;
                        float v = f * (dx * qx + dy * qy + dz * qz);
                        if (v < 0.0f || u + v > 1.0f)
                            continue;
                        float tHit = f * (e2x * qx + e2y * qy + e2z * qz);
                        if (tHit > 0.0f && tHit < bestT)
                            bestT = tHit;
                    }
                    float q = (bestT <= 1.0f) ? bestT : 0.5f;
                    if (q < 0.01f)
                        q = 0.01f;
                    if (q > 0.99f)
                        q = 0.99f;
                    g->q[cellIdx * 19 + i] = q;
                }
            }
    free(tb);
}

int or_initialize_flow(OrGrid *g, float ux, float uy, float uz) {
    if (g->prec == 4)
        init_flow_f32(g, ux, uy, uz);
    else
        init_flow_f64(g, ux, uy, uz);
    return 1;
}

void or_collide(OrGrid *g, float inX, float inY, float inZ) {
    if (g->prec == 4)
        collide_all_f32(g, inX, inY, inZ);
    else
        collide_all_f64(g, inX, inY, inZ);
}

void or_stream(OrGrid *g) {
    if (g->prec == 4)
        stream_all_f32(g);
    else
        stream_all_f64(g);
}

void or_step(OrGrid *g, float inX, float inY, float inZ) {
    or_collide(g, inX, inY, inZ);
    or_stream(g);
}

/* lbm.c:835-918 */
void or_drag_force_decomposed(OrGrid *g, float *out6) {
    if (g->prec == 4)
        force_all_f32(g);
    else
        force_all_f64(g);
    /* lbm.c:909-917: int results / 10000.0f (int32 in the reference; the
     * sums here are int64 and equal whenever the int32 sum did not wrap) */
    out6[0] = (float)(int32_t)g->force_raw[0] / 10000.0f;
    out6[1] = (float)(int32_t)g->force_raw[1] / 10000.0f;
    out6[2] = (float)(int32_t)g->force_raw[2] / 10000.0f;
    out6[3] = (float)(int32_t)g->force_raw[4] / 10000.0f;
    out6[4] = (float)(int32_t)g->force_raw[5] / 10000.0f;
    out6[5] = (float)(int32_t)g->force_raw[6] / 10000.0f;
}

/* lbm.c:920-940 */
float or_drag_coefficient(OrGrid *g, float U, float A) {
    float o[6];
    or_drag_force_decomposed(g, o);
    float dragForce = fabsf(o[0]);
    float rho = 1.0f;
    float dynamicPressure = 0.5f * rho * U * U;
    if (dynamicPressure * A < 1e-10f)
        return 0.0f;
    return dragForce / (dynamicPressure * A);
}

/* lbm.c:942-962 */
float or_lift_coefficient(OrGrid *g, float U, float A) {
    float o[6];
    or_drag_force_decomposed(g, o);
    float liftForce = fabsf(o[1]);
    float rho = 1.0f;
    float dynamicPressure = 0.5f * rho * U * U;
    if (dynamicPressure * A < 1e-10f)
        return 0.0f;
    return liftForce / (dynamicPressure * A);
}

/* ---- scalar exports for the known-answer tests ---- */
float or_feq_f32(int i, float rho, float ux, float uy, float uz) {
    return feq_f32(i, rho, ux, uy, uz);
}
double or_feq_f64(int i, double rho, double ux, double uy, double uz) {
    return feq_f64(i, rho, ux, uy, uz);
}
void or_mrt_forward_f32(const float *fi, float *m) { mrt_fwd_f32(fi, m); }
void or_mrt_inverse_f32(const float *m, float *fi) { mrt_inv_f32(m, fi); }
void or_mrt_meq_f32(float rho, float ux, float uy, float uz, float *meq) {
    mrt_meq_f32(rho, ux, uy, uz, meq);
}
float or_weight_f32(int i) { return wgt_f32(i); }

/* Batched forms of the above for the comparisons against the reference's own
 * C mirrors (simulation/test/test_lbm.c:71-187) on millions of states:
 * out[19 k + i] = feq(i, state[4 k .. 4 k + 3]) with state = (rho, ux, uy, uz). */
void or_feq_batch_f32(int64_t n, const float *state, float *out) {
    for (int64_t k = 0; k < n; k++) {
        const float *s = state + 4 * k;
        for (int i = 0; i < 19; i++) out[19 * k + i] = feq_f32(i, s[0], s[1], s[2], s[3]);
    }
}
void or_mrt_forward_batch_f32(int64_t n, const float *fi, float *m) {
    for (int64_t k = 0; k < n; k++) mrt_fwd_f32(fi + 19 * k, m + 19 * k);
}
void or_mrt_inverse_batch_f32(int64_t n, const float *m, float *fi) {
    for (int64_t k = 0; k < n; k++) mrt_inv_f32(m + 19 * k, fi + 19 * k);
}

/* ---- particles ---- */

/* 32-bit counter hash (three rounds of the "lowbias32" integer mixer of
 * C. Wellons' hash-prospector) over (seed, idx, k).  Identical in
 * lattice_fluid_dynamics_b200/csrc/lbm_particles.cu. */
static inline uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}
uint32_t or_hash3(uint32_t seed, uint32_t idx, uint32_t k) {
    return mix32(mix32(mix32(seed ^ 0x9e3779b9U) + idx) + k * 0x85ebca6bU);
}
float or_uniform01(uint32_t seed, uint32_t idx, uint32_t k) {
    return (float)(or_hash3(seed, idx, k) >> 8) * (1.0f / 16777216.0f);
}

void or_particles_seed_inlet(float *p, int n, uint32_t seed) {
    for (int i = 0; i < n; i++) {
        float *q = p + 8 * (size_t)i;
        q[0] = -4.0f;
        q[1] = or_uniform01(seed, (uint32_t)i, 0u) * 4.0f - 2.0f;
        q[2] = or_uniform01(seed, (uint32_t)i, 1u) * 4.0f - 2.0f;
        q[3] = 0.0f;
        q[4] = 0.0f;
        q[5] = 0.0f;
        q[6] = 0.0f;
        q[7] = 1.0f;
    }
}

static inline float mixf(float a, float b, float t) {
    /* GLSL mix: x * (1 - a) + y * a */
    return a * (1.0f - t) + b * t;
}
static inline float clampf(float v, float lo, float hi) {
    return fminf(fmaxf(v, lo), hi);
}

/* particle_lbm.comp:46-89 */
static void sample_velocity(const float *vel, int nx, int ny, int nz,
                            const float *pos, float *out) {
    float gp[3];
    gp[0] = (pos[0] + 4.0f) / 8.0f * (float)nx;
    gp[1] = (pos[1] + 2.0f) / 4.0f * (float)ny;
    gp[2] = (pos[2] + 2.0f) / 4.0f * (float)nz;
    gp[0] = clampf(gp[0], 0.0f, (float)nx - 1.0f);
    gp[1] = clampf(gp[1], 0.0f, (float)ny - 1.0f);
    gp[2] = clampf(gp[2], 0.0f, (float)nz - 1.0f);
    int i0[3], i1[3], dims[3] = {nx, ny, nz};
    float fr[3];
    for (int a = 0; a < 3; a++) {
        float fl = floorf(gp[a]);
        i0[a] = (int)fl;
        i1[a] = i0[a] + 1 < dims[a] - 1 ? i0[a] + 1 : dims[a] - 1;
        fr[a] = gp[a] - fl;
    }
#define VIDX(x, y, z) (4 * ((int64_t)(x) + (int64_t)(y) * nx + (int64_t)(z) * nx * ny))
    for (int c = 0; c < 3; c++) {
        float v000 = vel[VIDX(i0[0], i0[1], i0[2]) + c];
        float v100 = vel[VIDX(i1[0], i0[1], i0[2]) + c];
        float v010 = vel[VIDX(i0[0], i1[1], i0[2]) + c];
        float v110 = vel[VIDX(i1[0], i1[1], i0[2]) + c];
        float v001 = vel[VIDX(i0[0], i0[1], i1[2]) + c];
        float v101 = vel[VIDX(i1[0], i0[1], i1[2]) + c];
        float v011 = vel[VIDX(i0[0], i1[1], i1[2]) + c];
        float v111 = vel[VIDX(i1[0], i1[1], i1[2]) + c];
        float v00 = mixf(v000, v100, fr[0]);
        float v10 = mixf(v010, v110, fr[0]);
        float v01 = mixf(v001, v101, fr[0]);
        float v11 = mixf(v011, v111, fr[0]);
        float v0 = mixf(v00, v10, fr[1]);
        float v1 = mixf(v01, v11, fr[1]);
        out[c] = mixf(v0, v1, fr[2]);
    }
#undef VIDX
}

/* particle_lbm.comp:207-293 with useLBM = 1, collisionMode = 0 */
void or_particles_step(const float *vel4, int nx, int ny, int nz, float *p,
                       int n, float dt, uint32_t seed) {
#pragma omp parallel for schedule(static)
    for (int idx = 0; idx < n; idx++) {
        float *q = p + 8 * (size_t)idx;
        float flow[3];
        sample_velocity(vel4, nx, ny, nz, q, flow);
        flow[0] *= 2.0f;
        flow[1] *= 2.0f;
        flow[2] *= 2.0f;
        float relaxation = 5.0f * dt;
        q[4] = mixf(q[4], flow[0], relaxation);
        q[5] = mixf(q[5], flow[1], relaxation);
        q[6] = mixf(q[6], flow[2], relaxation);
        q[0] += q[4] * dt;
        q[1] += q[5] * dt;
        q[2] += q[6] * dt;
        q[7] -= 0.01f * dt;
        if (q[7] <= 0.0f || q[0] > 4.0f || fabsf(q[1]) > 2.0f ||
            fabsf(q[2]) > 2.0f) {
            q[0] = -4.0f;
            q[1] = (or_uniform01(seed, (uint32_t)idx, 2u) - 0.5f) * 3.0f;
            q[2] = (or_uniform01(seed, (uint32_t)idx, 3u) - 0.5f) * 3.0f;
            q[4] = 0.5f + or_uniform01(seed, (uint32_t)idx, 4u) * 0.2f;
            q[5] = 0.0f;
            q[6] = 0.0f;
            q[7] = 1.0f;
        }
    }
}

/* vti_export.c:10-116 from host arrays */
int or_write_vti(const char *filename, int nx, int ny, int nz,
                 const float *vel, const int32_t *solid) {
    size_t total = (size_t)nx * ny * nz;
    FILE *f = fopen(filename, "wb");
    if (!f)
        return 0;
    size_t rhoOffset = sizeof(uint64_t) + total * 3 * sizeof(float);
    size_t solidOffset = rhoOffset + sizeof(uint64_t) + total * sizeof(float);
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
            nx, ny, nz, nx, ny, nz, (unsigned long)rhoOffset,
            (unsigned long)solidOffset);
    int ok = 1;
    uint64_t sz = (uint64_t)total * 3 * sizeof(float);
    ok = ok && fwrite(&sz, sizeof(uint64_t), 1, f) == 1;
    for (size_t i = 0; i < total && ok; i++)
        ok = fwrite(&vel[i * 4], sizeof(float), 3, f) == 3;
    sz = (uint64_t)total * sizeof(float);
    ok = ok && fwrite(&sz, sizeof(uint64_t), 1, f) == 1;
    for (size_t i = 0; i < total && ok; i++)
        ok = fwrite(&vel[i * 4 + 3], sizeof(float), 1, f) == 1;
    sz = (uint64_t)total * sizeof(int32_t);
    ok = ok && fwrite(&sz, sizeof(uint64_t), 1, f) == 1;
    ok = ok && fwrite(solid, sizeof(int32_t), total, f) == total;
    if (!ok) {
        fclose(f);
        return 0;
    }
    fprintf(f, "\n  </AppendedData>\n</VTKFile>\n");
    fclose(f);
    return 1;
}
