/*
 * Exhaustive check that division by a constant y computed as
 *     q1 = RN(x * zh);  r = fma(-q1, y, x);  q = fma(r, zh, q1)
 * with zh = RN(1/y) (P. Markstein, "Computation of elementary functions on
 * the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990;
 * the division theorem restated in Brisebarre, Muller and Raina, IEEE
 * Trans. Computers 53(8), 2004) returns the IEEE quotient RN(x / y) for
 * every finite single-precision x.  The solver uses this sequence for
 * its divisions by compile-time constants.
 *
 * usage: cdiv_check <stride> <y>...   (stride 1 = all 2^32 bit patterns)
 * Mismatches are reported overall and inside |x| in [2^-100, 2^100]; the
 * exit status is nonzero only for mismatches inside that range (outside it
 * the intermediate product underflows or overflows, which the solver's
 * operands never reach: they are bounded populations and moments).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static float bits2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

int main(int argc, char **argv) {
    if (argc < 3) return 2;
    uint64_t stride = strtoull(argv[1], NULL, 10);
    int bad_total = 0;
    for (int a = 2; a < argc; a++) {
        float y = strtof(argv[a], NULL);
        float zh = 1.0f / y;
        uint64_t checked = 0, bad = 0;
        float worst = INFINITY, worst_hi = 0.0f;
        uint64_t bad_mid = 0;
        for (uint64_t u = 0; u < (1ull << 32); u += stride) {
            float x = bits2f((uint32_t)u);
            if (!isfinite(x)) continue;
            float ref = x / y;
            float q1 = x * zh;
            float r = fmaf(-q1, y, x);
            float q = fmaf(r, zh, q1);
            checked++;
            if (memcmp(&q, &ref, 4) != 0 && !(q == 0.0f && ref == 0.0f)) {
                bad++;
                if (fabsf(x) < worst) worst = fabsf(x);
                if (fabsf(x) > worst_hi) worst_hi = fabsf(x);
                if (fabsf(x) >= 0x1p-100f && fabsf(x) <= 0x1p100f) bad_mid++;
            }
        }
        printf("%.9g checked=%llu mismatches=%llu in[2^-100,2^100]=%llu min|x|=%.9g max|x|=%.9g\n",
               (double)y, (unsigned long long)checked, (unsigned long long)bad,
               (unsigned long long)bad_mid, (double)worst, (double)worst_hi);
        if (bad_mid) bad_total = 1;
    }
    return bad_total;
}
