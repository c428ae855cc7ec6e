/*
 * CPU oracle of the warm-start network (TEST INFRASTRUCTURE ONLY).
 *
 * The network has no counterpart in the reference: it is the learned
 * warm start of the B200 solver (a 4-level 3D conv encoder-decoder mapping
 * voxel mask + inflow + Re at quarter resolution to (rho, u)).  This file
 * restates its forward and backward passes in plain C with double
 * accumulation, so that the GPU kernels (tensor-core convolutions and the
 * element-wise kernels) can be checked against it, and it checks itself by
 * finite differences in the tests.  With `bf16` set it rounds to bfloat16
 * (round to nearest even) exactly where the GPU stores bfloat16: weights,
 * activations, pooled and upsampled values, the prediction and every
 * pre-activation gradient fed to a convolution.
 *
 * Layout: channels-last, voxel v = ((b * NZ + z) * NY + y) * NX + x.
 * Convolution weights w[co][tap * cin + ci], tap = (dz+1)*9 + (dy+1)*3 +
 * (dx+1), zero padding at the borders.  Parameters are packed layer by layer
 * as (w [cout][27 cin], bias [cout]) in the order of NN_LAYERS.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "nn_oracle.h"

/* {cin, cout, act} of the 16 convolutions (see nn_oracle.h) */
const int NN_LAYERS[NN_NUM_LAYERS][3] = {
    {8, 16, 1},   {16, 16, 1},  {16, 32, 1},  {32, 32, 1},  {32, 64, 1},  {64, 64, 1},
    {64, 128, 1}, {128, 128, 1}, {128, 128, 1}, {192, 64, 1}, {64, 64, 1},  {96, 32, 1},
    {32, 32, 1},  {48, 16, 1},  {16, 16, 1},  {16, 4, 0}};

float nno_bf16(float v) {
    uint32_t u;
    memcpy(&u, &v, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return v; /* inf / nan unchanged */
    u = (u + 0x7fffu + ((u >> 16) & 1u)) & 0xffff0000u;
    memcpy(&v, &u, 4);
    return v;
}

static float rnd(float v, int bf16) { return bf16 ? nno_bf16(v) : v; }

static float leaky(float v) { return v > 0.f ? v : 0.1f * v; }

long long nno_param_count(void) {
    long long n = 0;
    for (int l = 0; l < NN_NUM_LAYERS; l++)
        n += (long long)NN_LAYERS[l][1] * 27 * NN_LAYERS[l][0] + NN_LAYERS[l][1];
    return n;
}

static long long neighbour(int nb, int nz, int ny, int nx, long long v, int tap) {
    const int x = (int)(v % nx);
    long long t = v / nx;
    const int y = (int)(t % ny);
    t /= ny;
    const int z = (int)(t % nz);
    const int b = (int)(t / nz);
    const int zz = z + tap / 9 - 1, yy = y + (tap / 3) % 3 - 1, xx = x + tap % 3 - 1;
    if (zz < 0 || zz >= nz || yy < 0 || yy >= ny || xx < 0 || xx >= nx) return -1;
    (void)nb;
    return (((long long)b * nz + zz) * ny + yy) * nx + xx;
}

/* y[v][co] = sum x[nbr][ci] w[co][tap cin + ci] + bias[co]  (no activation) */
void nno_conv_fwd(const float *x, int xs, int xo, int cin, const float *w, const float *bias,
                  int cout, float *y, int ys, int yo, int nb, int nz, int ny, int nx) {
    const long long m = (long long)nb * nz * ny * nx;
#pragma omp parallel for schedule(static)
    for (long long v = 0; v < m; v++) {
        for (int co = 0; co < cout; co++) {
            double s = bias ? bias[co] : 0.0;
            for (int tap = 0; tap < 27; tap++) {
                const long long q = neighbour(nb, nz, ny, nx, v, tap);
                if (q < 0) continue;
                const float *xp = x + q * xs + xo;
                const float *wp = w + (long long)co * 27 * cin + tap * cin;
                for (int ci = 0; ci < cin; ci++) s += (double)xp[ci] * wp[ci];
            }
            y[v * ys + yo + co] = (float)s;
        }
    }
}

/* dx[v][ci] = sum over taps and co of g[nbr'][co] w[co][(26 - tap) ...]:
 * the adjoint of nno_conv_fwd */
void nno_conv_dgrad(const float *g, int gs, int cout, const float *w, int cin, float *dx,
                    int dxs, int dxo, int nb, int nz, int ny, int nx) {
    const long long m = (long long)nb * nz * ny * nx;
#pragma omp parallel for schedule(static)
    for (long long v = 0; v < m; v++) {
        for (int ci = 0; ci < cin; ci++) {
            double s = 0.0;
            for (int tap = 0; tap < 27; tap++) {
                /* output voxel u with neighbour(u, tap) == v is neighbour(v, 26 - tap) */
                const long long u = neighbour(nb, nz, ny, nx, v, 26 - tap);
                if (u < 0) continue;
                for (int co = 0; co < cout; co++)
                    s += (double)g[u * gs + co] * w[(long long)co * 27 * cin + tap * cin + ci];
            }
            dx[v * dxs + dxo + ci] = (float)s;
        }
    }
}

/* dw[co][tap cin + ci] = sum_v g[v][co] x[nbr(v, tap)][ci]; db[co] = sum_v g */
void nno_conv_wgrad(const float *x, int xs, int xo, int cin, const float *g, int gs, int cout,
                    float *dw, float *db, int nb, int nz, int ny, int nx) {
    const long long m = (long long)nb * nz * ny * nx;
#pragma omp parallel for schedule(static)
    for (int co = 0; co < cout; co++) {
        for (int tap = 0; tap < 27; tap++) {
            for (int ci = 0; ci < cin; ci++) {
                double s = 0.0;
                for (long long v = 0; v < m; v++) {
                    const long long q = neighbour(nb, nz, ny, nx, v, tap);
                    if (q < 0) continue;
                    s += (double)g[v * gs + co] * x[q * xs + xo + ci];
                }
                dw[(long long)co * 27 * cin + tap * cin + ci] = (float)s;
            }
        }
        if (db) {
            double s = 0.0;
            for (long long v = 0; v < m; v++) s += g[v * gs + co];
            db[co] = (float)s;
        }
    }
}

/* ---- the network ---------------------------------------------------- */

typedef struct {
    int nz, ny, nx;
    long long m; /* voxels at this level, whole batch */
} Level;

static float *zalloc(long long n) { return (float *)calloc((size_t)(n > 0 ? n : 1), sizeof(float)); }

/* average of the 2x2x2 children */
static void pool(const float *s, int ss, int so, int c, const Level *fine, float *out,
                 const Level *coarse, int nb, int bf16) {
    for (int b = 0; b < nb; b++)
        for (int z = 0; z < coarse->nz; z++)
            for (int y = 0; y < coarse->ny; y++)
                for (int x = 0; x < coarse->nx; x++) {
                    const long long o = (((long long)b * coarse->nz + z) * coarse->ny + y) * coarse->nx + x;
                    for (int ch = 0; ch < c; ch++) {
                        float acc = 0.f;
                        for (int k = 0; k < 8; k++) {
                            const long long f = (((long long)b * fine->nz + 2 * z + (k >> 2)) * fine->ny +
                                                 2 * y + ((k >> 1) & 1)) * fine->nx + 2 * x + (k & 1);
                            acc += s[f * ss + so + ch];
                        }
                        out[o * c + ch] = rnd(acc * 0.125f, bf16);
                    }
                }
}

static void pool_bwd(const float *dout, int c, const Level *coarse, float *ds, int dss, int dso,
                     const Level *fine, int nb) {
    for (int b = 0; b < nb; b++)
        for (int z = 0; z < fine->nz; z++)
            for (int y = 0; y < fine->ny; y++)
                for (int x = 0; x < fine->nx; x++) {
                    const long long f = (((long long)b * fine->nz + z) * fine->ny + y) * fine->nx + x;
                    const long long o = (((long long)b * coarse->nz + z / 2) * coarse->ny + y / 2) * coarse->nx + x / 2;
                    for (int ch = 0; ch < c; ch++) ds[f * dss + dso + ch] += dout[o * c + ch] * 0.125f;
                }
}

static void upsample(const float *d, int c, const Level *coarse, float *out, int os, int oo,
                     const Level *fine, int nb) {
    for (int b = 0; b < nb; b++)
        for (int z = 0; z < fine->nz; z++)
            for (int y = 0; y < fine->ny; y++)
                for (int x = 0; x < fine->nx; x++) {
                    const long long f = (((long long)b * fine->nz + z) * fine->ny + y) * fine->nx + x;
                    const long long o = (((long long)b * coarse->nz + z / 2) * coarse->ny + y / 2) * coarse->nx + x / 2;
                    for (int ch = 0; ch < c; ch++) out[f * os + oo + ch] = d[o * c + ch];
                }
}

static void upsample_bwd(const float *dout, int os, int oo, int c, const Level *fine, float *dd,
                         const Level *coarse, int nb) {
    memset(dd, 0, sizeof(float) * (size_t)(coarse->m * c));
    for (int b = 0; b < nb; b++)
        for (int z = 0; z < fine->nz; z++)
            for (int y = 0; y < fine->ny; y++)
                for (int x = 0; x < fine->nx; x++) {
                    const long long f = (((long long)b * fine->nz + z) * fine->ny + y) * fine->nx + x;
                    const long long o = (((long long)b * coarse->nz + z / 2) * coarse->ny + y / 2) * coarse->nx + x / 2;
                    for (int ch = 0; ch < c; ch++) dd[o * c + ch] += dout[f * os + oo + ch];
                }
}

/* one convolution layer with the GPU's roundings: weights rounded, output
 * activated and rounded */
static void layer_fwd(const float *x, int xs, int xo, int l, const float *const *wr,
                      const float *const *bias, float *y, int ys, int yo, const Level *L, int nb,
                      int bf16) {
    const int cin = NN_LAYERS[l][0], cout = NN_LAYERS[l][1], act = NN_LAYERS[l][2];
    nno_conv_fwd(x, xs, xo, cin, wr[l], bias[l], cout, y, ys, yo, nb, L->nz, L->ny, L->nx);
    for (long long v = 0; v < L->m; v++)
        for (int c = 0; c < cout; c++) {
            float *p = y + v * ys + yo + c;
            *p = rnd(act ? leaky(*p) : *p, bf16);
        }
}

/* dPre = round(dOut * act'(out)) */
static void act_bwd(const float *dout, int ds, int dof, const float *out, int os, int oo, int c,
                    int act, long long m, float *dpre, int bf16) {
    for (long long v = 0; v < m; v++)
        for (int ch = 0; ch < c; ch++) {
            float g = dout[v * ds + dof + ch];
            if (act && !(out[v * os + oo + ch] > 0.f)) g *= 0.1f;
            dpre[v * c + ch] = rnd(g, bf16);
        }
}

double nno_net(const float *params, int nb, int nz, int ny, int nx, const float *features,
               const float *target, int bf16, float *pred_out, float *grad_out) {
    Level L[4];
    for (int i = 0; i < 4; i++) {
        L[i].nz = nz >> i;
        L[i].ny = ny >> i;
        L[i].nx = nx >> i;
        L[i].m = (long long)nb * L[i].nz * L[i].ny * L[i].nx;
    }
    /* weights (rounded copies) and biases */
    const float *wv[NN_NUM_LAYERS], *bv[NN_NUM_LAYERS];
    float *wr[NN_NUM_LAYERS];
    long long off = 0;
    for (int l = 0; l < NN_NUM_LAYERS; l++) {
        const long long nw = (long long)NN_LAYERS[l][1] * 27 * NN_LAYERS[l][0];
        wv[l] = params + off;
        wr[l] = zalloc(nw);
        for (long long i = 0; i < nw; i++) wr[l][i] = rnd(wv[l][i], bf16);
        bv[l] = params + off + nw;
        off += nw + NN_LAYERS[l][1];
    }
    const long long m1 = L[0].m, m2 = L[1].m, m3 = L[2].m, m4 = L[3].m;
    /* input: 8 channels (mask, U / 0.1, log(Re / 100) / log(20), zeros) */
    float *in0 = zalloc(m1 * 8);
    for (long long v = 0; v < m1; v++) {
        in0[v * 8 + 0] = rnd(features[v * 3 + 0], bf16);
        in0[v * 8 + 1] = rnd(features[v * 3 + 1] / 0.1f, bf16);
        in0[v * 8 + 2] = rnd((float)(log(features[v * 3 + 2] / 100.0) / log(20.0)), bf16);
    }
    float *a1 = zalloc(m1 * 16), *cat1 = zalloc(m1 * 48), *in2 = zalloc(m2 * 16);
    float *a2 = zalloc(m2 * 32), *cat2 = zalloc(m2 * 96), *in3 = zalloc(m3 * 32);
    float *a3 = zalloc(m3 * 64), *cat3 = zalloc(m3 * 192), *in4 = zalloc(m4 * 64);
    float *a4 = zalloc(m4 * 128), *b4 = zalloc(m4 * 128), *s4 = zalloc(m4 * 128);
    float *c3 = zalloc(m3 * 64), *d3 = zalloc(m3 * 64), *c2 = zalloc(m2 * 32), *d2 = zalloc(m2 * 32);
    float *c1 = zalloc(m1 * 16), *d1 = zalloc(m1 * 16), *pr = zalloc(m1 * 4);

    layer_fwd(in0, 8, 0, 0, (const float *const *)wr, bv, a1, 16, 0, &L[0], nb, bf16);
    layer_fwd(a1, 16, 0, 1, (const float *const *)wr, bv, cat1, 48, 0, &L[0], nb, bf16);
    pool(cat1, 48, 0, 16, &L[0], in2, &L[1], nb, bf16);
    layer_fwd(in2, 16, 0, 2, (const float *const *)wr, bv, a2, 32, 0, &L[1], nb, bf16);
    layer_fwd(a2, 32, 0, 3, (const float *const *)wr, bv, cat2, 96, 0, &L[1], nb, bf16);
    pool(cat2, 96, 0, 32, &L[1], in3, &L[2], nb, bf16);
    layer_fwd(in3, 32, 0, 4, (const float *const *)wr, bv, a3, 64, 0, &L[2], nb, bf16);
    layer_fwd(a3, 64, 0, 5, (const float *const *)wr, bv, cat3, 192, 0, &L[2], nb, bf16);
    pool(cat3, 192, 0, 64, &L[2], in4, &L[3], nb, bf16);
    layer_fwd(in4, 64, 0, 6, (const float *const *)wr, bv, a4, 128, 0, &L[3], nb, bf16);
    layer_fwd(a4, 128, 0, 7, (const float *const *)wr, bv, b4, 128, 0, &L[3], nb, bf16);
    layer_fwd(b4, 128, 0, 8, (const float *const *)wr, bv, s4, 128, 0, &L[3], nb, bf16);
    upsample(s4, 128, &L[3], cat3, 192, 64, &L[2], nb);
    layer_fwd(cat3, 192, 0, 9, (const float *const *)wr, bv, c3, 64, 0, &L[2], nb, bf16);
    layer_fwd(c3, 64, 0, 10, (const float *const *)wr, bv, d3, 64, 0, &L[2], nb, bf16);
    upsample(d3, 64, &L[2], cat2, 96, 32, &L[1], nb);
    layer_fwd(cat2, 96, 0, 11, (const float *const *)wr, bv, c2, 32, 0, &L[1], nb, bf16);
    layer_fwd(c2, 32, 0, 12, (const float *const *)wr, bv, d2, 32, 0, &L[1], nb, bf16);
    upsample(d2, 32, &L[1], cat1, 48, 16, &L[0], nb);
    layer_fwd(cat1, 48, 0, 13, (const float *const *)wr, bv, c1, 16, 0, &L[0], nb, bf16);
    layer_fwd(c1, 16, 0, 14, (const float *const *)wr, bv, d1, 16, 0, &L[0], nb, bf16);
    layer_fwd(d1, 16, 0, 15, (const float *const *)wr, bv, pr, 4, 0, &L[0], nb, bf16);
    if (pred_out) memcpy(pred_out, pr, sizeof(float) * (size_t)(m1 * 4));

    double loss = 0.0;
    if (target) {
        for (long long i = 0; i < m1 * 4; i++) {
            const double d = (double)pr[i] - target[i];
            loss += d * d;
        }
        loss /= (double)(m1 * 4);
    }
    if (grad_out && target) {
        float *gw[NN_NUM_LAYERS], *gb[NN_NUM_LAYERS];
        off = 0;
        for (int l = 0; l < NN_NUM_LAYERS; l++) {
            const long long nw = (long long)NN_LAYERS[l][1] * 27 * NN_LAYERS[l][0];
            gw[l] = grad_out + off;
            gb[l] = grad_out + off + nw;
            off += nw + NN_LAYERS[l][1];
        }
        const float scale = 2.0f / (float)(m1 * 4);
        float *g = zalloc(m1 * 192); /* pre-activation gradient scratch, largest layer */
        float *dd1 = zalloc(m1 * 16), *dc1 = zalloc(m1 * 16), *dcat1 = zalloc(m1 * 48);
        float *dd2 = zalloc(m2 * 32), *dc2 = zalloc(m2 * 32), *dcat2 = zalloc(m2 * 96);
        float *dd3 = zalloc(m3 * 64), *dc3 = zalloc(m3 * 64), *dcat3 = zalloc(m3 * 192);
        float *ds4 = zalloc(m4 * 128), *db4 = zalloc(m4 * 128), *da4 = zalloc(m4 * 128);
        float *din4 = zalloc(m4 * 64), *da3 = zalloc(m3 * 64), *din3 = zalloc(m3 * 32);
        float *da2 = zalloc(m2 * 32), *din2 = zalloc(m2 * 16), *da1 = zalloc(m1 * 16);
        /* output layer */
        for (long long i = 0; i < m1 * 4; i++) g[i] = rnd(scale * (pr[i] - target[i]), bf16);
#define BACK(l, X, XS, XO, M_, LV, DX, DXS, DXO)                                                 \
    nno_conv_wgrad(X, XS, XO, NN_LAYERS[l][0], g, NN_LAYERS[l][1], NN_LAYERS[l][1], gw[l], gb[l], \
                   nb, (LV)->nz, (LV)->ny, (LV)->nx);                                            \
    if (DX)                                                                                      \
        nno_conv_dgrad(g, NN_LAYERS[l][1], NN_LAYERS[l][1], wr[l], NN_LAYERS[l][0], DX, DXS,      \
                       DXO, nb, (LV)->nz, (LV)->ny, (LV)->nx);
        BACK(15, d1, 16, 0, m1, &L[0], dd1, 16, 0);
        act_bwd(dd1, 16, 0, d1, 16, 0, 16, 1, m1, g, bf16);
        BACK(14, c1, 16, 0, m1, &L[0], dc1, 16, 0);
        act_bwd(dc1, 16, 0, c1, 16, 0, 16, 1, m1, g, bf16);
        BACK(13, cat1, 48, 0, m1, &L[0], dcat1, 48, 0);
        upsample_bwd(dcat1, 48, 16, 32, &L[0], dd2, &L[1], nb);
        act_bwd(dd2, 32, 0, d2, 32, 0, 32, 1, m2, g, bf16);
        BACK(12, c2, 32, 0, m2, &L[1], dc2, 32, 0);
        act_bwd(dc2, 32, 0, c2, 32, 0, 32, 1, m2, g, bf16);
        BACK(11, cat2, 96, 0, m2, &L[1], dcat2, 96, 0);
        upsample_bwd(dcat2, 96, 32, 64, &L[1], dd3, &L[2], nb);
        act_bwd(dd3, 64, 0, d3, 64, 0, 64, 1, m3, g, bf16);
        BACK(10, c3, 64, 0, m3, &L[2], dc3, 64, 0);
        act_bwd(dc3, 64, 0, c3, 64, 0, 64, 1, m3, g, bf16);
        BACK(9, cat3, 192, 0, m3, &L[2], dcat3, 192, 0);
        upsample_bwd(dcat3, 192, 64, 128, &L[2], ds4, &L[3], nb);
        act_bwd(ds4, 128, 0, s4, 128, 0, 128, 1, m4, g, bf16);
        BACK(8, b4, 128, 0, m4, &L[3], db4, 128, 0);
        act_bwd(db4, 128, 0, b4, 128, 0, 128, 1, m4, g, bf16);
        BACK(7, a4, 128, 0, m4, &L[3], da4, 128, 0);
        act_bwd(da4, 128, 0, a4, 128, 0, 128, 1, m4, g, bf16);
        BACK(6, in4, 64, 0, m4, &L[3], din4, 64, 0);
        pool_bwd(din4, 64, &L[3], dcat3, 192, 0, &L[2], nb);
        act_bwd(dcat3, 192, 0, cat3, 192, 0, 64, 1, m3, g, bf16);
        BACK(5, a3, 64, 0, m3, &L[2], da3, 64, 0);
        act_bwd(da3, 64, 0, a3, 64, 0, 64, 1, m3, g, bf16);
        BACK(4, in3, 32, 0, m3, &L[2], din3, 32, 0);
        pool_bwd(din3, 32, &L[2], dcat2, 96, 0, &L[1], nb);
        act_bwd(dcat2, 96, 0, cat2, 96, 0, 32, 1, m2, g, bf16);
        BACK(3, a2, 32, 0, m2, &L[1], da2, 32, 0);
        act_bwd(da2, 32, 0, a2, 32, 0, 32, 1, m2, g, bf16);
        BACK(2, in2, 16, 0, m2, &L[1], din2, 16, 0);
        pool_bwd(din2, 16, &L[1], dcat1, 48, 0, &L[0], nb);
        act_bwd(dcat1, 48, 0, cat1, 48, 0, 16, 1, m1, g, bf16);
        BACK(1, a1, 16, 0, m1, &L[0], da1, 16, 0);
        act_bwd(da1, 16, 0, a1, 16, 0, 16, 1, m1, g, bf16);
        BACK(0, in0, 8, 0, m1, &L[0], (float *)0, 0, 0);
#undef BACK
        free(g);
        free(dd1); free(dc1); free(dcat1); free(dd2); free(dc2); free(dcat2);
        free(dd3); free(dc3); free(dcat3); free(ds4); free(db4); free(da4);
        free(din4); free(da3); free(din3); free(da2); free(din2); free(da1);
    }
    free(in0); free(a1); free(cat1); free(in2); free(a2); free(cat2); free(in3); free(a3);
    free(cat3); free(in4); free(a4); free(b4); free(s4); free(c3); free(d3); free(c2); free(d2);
    free(c1); free(d1); free(pr);
    for (int l = 0; l < NN_NUM_LAYERS; l++) free(wr[l]);
    return loss;
}
