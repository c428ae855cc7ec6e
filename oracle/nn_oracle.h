/*
 * CPU oracle of the warm-start network (TEST INFRASTRUCTURE ONLY; see
 * nn_oracle.c).
 *
 * Architecture (quarter-resolution input NX x NY x NZ, all divisible by 8):
 *   level 1 (full):   conv 8->16, conv 16->16 = s1
 *   level 2 (1/2):    pool(s1), conv 16->32, conv 32->32 = s2
 *   level 3 (1/4):    pool(s2), conv 32->64, conv 64->64 = s3
 *   level 4 (1/8):    pool(s3), conv 64->128, 128->128, 128->128 = s4
 *   decoder 3:        [s3, up(s4)] 192 -> 64 -> 64 = d3
 *   decoder 2:        [s2, up(d3)] 96 -> 32 -> 32 = d2
 *   decoder 1:        [s1, up(d2)] 48 -> 16 -> 16 = d1
 *   output:           conv 16 -> 4, linear
 * 3x3x3 convolutions, zero padding, leaky ReLU (slope 0.1) except the
 * output; pool = 2x2x2 average, up = nearest-neighbour x2.  Input channels:
 * mask, U / 0.1, log(Re / 100) / log(20), five zeros.  Loss: mean squared
 * error over all voxels and the 4 output channels.
 */
#ifndef NN_ORACLE_H
#define NN_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define NN_NUM_LAYERS 16
extern const int NN_LAYERS[NN_NUM_LAYERS][3]; /* cin, cout, leaky */

float nno_bf16(float v);
long long nno_param_count(void);
void nno_conv_fwd(const float *x, int xs, int xo, int cin, const float *w, const float *bias,
                  int cout, float *y, int ys, int yo, int nb, int nz, int ny, int nx);
void nno_conv_dgrad(const float *g, int gs, int cout, const float *w, int cin, float *dx,
                    int dxs, int dxo, int nb, int nz, int ny, int nx);
void nno_conv_wgrad(const float *x, int xs, int xo, int cin, const float *g, int gs, int cout,
                    float *dw, float *db, int nb, int nz, int ny, int nx);
/* forward (pred [m][4]) and, with a target, the mean squared error and the
 * gradient of every parameter (packed like params) */
double nno_net(const float *params, int nb, int nz, int ny, int nx, const float *features,
               const float *target, int bf16, float *pred_out, float *grad_out);

#ifdef __cplusplus
}
#endif
#endif
