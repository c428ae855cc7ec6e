/*
 * TEST INFRASTRUCTURE ONLY: a checker, never linked into the product.
 *
 * Exports the reference's own plain-C mirrors of the collision shader's
 * arithmetic -- the D3Q19 weights and velocity set, feq, cpu_forwardMRT and
 * cpu_inverseMRT of simulation/test/test_lbm.c:43-187 -- so that the tests
 * can run them beside the oracle (oracle_core.inc) and the CUDA kernels.
 * The block is cut out of the reference's test file, where it lies, by the
 * `ref` target of oracle/Makefile into oracle/_ref/test_lbm_math.inc and
 * compiled here with -ffp-contract=off (IEEE single precision, no fused
 * multiply-add), the rounding the GLSL source specifies.  Nothing of the
 * reference is copied into this repository.
 */
#include <stdint.h>

#include "test_lbm_math.inc"

float ref_weight(int i) { return w[i]; }

/* out[19 k + i] = feq(i, rho_k, ux_k, uy_k, uz_k); state = (rho, ux, uy, uz) per k */
void ref_feq_batch(int64_t n, const float *state, float *out) {
    for (int64_t k = 0; k < n; k++) {
        const float *s = state + 4 * k;
        for (int i = 0; i < 19; i++) out[19 * k + i] = feq(i, s[0], s[1], s[2], s[3]);
    }
}

void ref_forward_mrt_batch(int64_t n, const float *fi, float *m) {
    for (int64_t k = 0; k < n; k++) cpu_forwardMRT(fi + 19 * k, m + 19 * k);
}

void ref_inverse_mrt_batch(int64_t n, const float *m, float *fi) {
    for (int64_t k = 0; k < n; k++) cpu_inverseMRT(m + 19 * k, fi + 19 * k);
}
