// D3Q19 lattice constants, population storage formats and the per-cell
// collision of the Lattice wind-tunnel solver, for sm_100a.
//
// The collision follows simulation/shaders/lbm_collide.comp:313-626 of the
// reference (solid swap, Zou-He velocity inlet / pressure outlet, moments,
// stability guard, Smagorinsky tau_eff, then regularized / MRT / BGK).
// Every expression keeps the shader's operand order; the library is built
// with --fmad=false and IEEE division/sqrt so that the FP32 path performs
// the same sequence of single-precision roundings as the C oracle, which
// is what makes the populations comparable bit for bit.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "lbm_internal.h"

// Arithmetic flavour of the device code compiled in this translation unit:
// `exact` (the default, --fmad=false and IEEE division/sqrt: the oracle's
// rounding sequence) or `fast` (LBM_FAST_ARITH: contracted FMAs and
// hardware-approximate division/sqrt).  Each flavour lives in its own
// namespace so both can be linked into one library.
#ifdef LBM_FAST_ARITH
#define LBM_ARITH_NS fast
#else
#define LBM_ARITH_NS exact
#endif

namespace lbm {
namespace LBM_ARITH_NS {

// velocity set (lbm_collide.comp:33-52) and opposites (:76-77)
__host__ __device__ constexpr int cx(int i) {
    return (i == 1 || i == 7 || i == 9 || i == 11 || i == 13) ? 1
           : (i == 2 || i == 8 || i == 10 || i == 12 || i == 14) ? -1
                                                                 : 0;
}
__host__ __device__ constexpr int cy(int i) {
    return (i == 3 || i == 7 || i == 8 || i == 15 || i == 17) ? 1
           : (i == 4 || i == 9 || i == 10 || i == 16 || i == 18) ? -1
                                                                 : 0;
}
__host__ __device__ constexpr int cz(int i) {
    return (i == 5 || i == 11 || i == 12 || i == 15 || i == 16) ? 1
           : (i == 6 || i == 13 || i == 14 || i == 17 || i == 18) ? -1
                                                                  : 0;
}
__host__ __device__ constexpr int opp(int i) {
    return i == 0 ? 0 : i == 1 ? 2 : i == 2 ? 1 : i == 3 ? 4 : i == 4 ? 3
         : i == 5 ? 6 : i == 6 ? 5 : i == 7 ? 10 : i == 8 ? 9 : i == 9 ? 8
         : i == 10 ? 7 : i == 11 ? 14 : i == 12 ? 13 : i == 13 ? 12
         : i == 14 ? 11 : i == 15 ? 18 : i == 16 ? 17 : i == 17 ? 16 : 15;
}

// weights 1/3, 1/18, 1/36 evaluated in the arithmetic type (:55-73)
template <typename R>
__host__ __device__ __forceinline__ constexpr R wgt(int i) {
    return i == 0 ? R(1) / R(3) : (i <= 6 ? R(1) / R(18) : R(1) / R(36));
}

// flag byte per cell
enum : uint8_t {
    FLAG_SOLID_MASK = 0x3,  // 0 fluid, 1 body, 2 ground (reference solid[])
    FLAG_BOUNDARY = 0x4     // cell owns at least one boundary link
};

// ---------------------------------------------------------------------
// Population storage formats.  R is the collision arithmetic type.
// FP16/BF16 keep the deviation f_i - w_i (w_i in FP32).
// ---------------------------------------------------------------------
// load2/store2 move the populations of two neighbouring cells (p must be
// aligned to two elements).  `load` reads global memory through the
// read-only path; `lds` reads a population staged in shared memory.
struct StoreF32 {
    using T = float;
    using R = float;
    static __device__ __forceinline__ R load(const T *p, int) { return __ldg(p); }
    static __device__ __forceinline__ R lds(const T *p, int) { return *p; }
    static __device__ __forceinline__ void store(T *p, R v, int) { *p = v; }
    static __device__ __forceinline__ void load2(const T *p, int, R &a, R &b) {
        const float2 v = __ldg(reinterpret_cast<const float2 *>(p));
        a = v.x;
        b = v.y;
    }
    static __device__ __forceinline__ void store2(T *p, R a, R b, int) {
        *reinterpret_cast<float2 *>(p) = make_float2(a, b);
    }
};
struct StoreF64 {
    using T = double;
    using R = double;
    static __device__ __forceinline__ R load(const T *p, int) { return __ldg(p); }
    static __device__ __forceinline__ R lds(const T *p, int) { return *p; }
    static __device__ __forceinline__ void store(T *p, R v, int) { *p = v; }
    static __device__ __forceinline__ void load2(const T *p, int, R &a, R &b) {
        const double2 v = __ldg(reinterpret_cast<const double2 *>(p));
        a = v.x;
        b = v.y;
    }
    static __device__ __forceinline__ void store2(T *p, R a, R b, int) {
        *reinterpret_cast<double2 *>(p) = make_double2(a, b);
    }
};
// paired IEEE add / subtract (defined below)
__device__ __forceinline__ float2 padd(float2 a, float2 b);
__device__ __forceinline__ float2 psub(float2 a, float2 b);

// The 16-bit formats store f_i - w_i.  load2 / store2 move two neighbouring
// cells with one packed conversion and one paired add / subtract: the same
// roundings as two scalar loads / stores.
struct StoreF16 {
    using T = __half;
    using R = float;
    static __device__ __forceinline__ R load(const T *p, int i) {
        return __half2float(__ldg(p)) + wgt<float>(i);
    }
    static __device__ __forceinline__ R lds(const T *p, int i) {
        return __half2float(*p) + wgt<float>(i);
    }
    static __device__ __forceinline__ void store(T *p, R v, int i) {
        *p = __float2half_rn(v - wgt<float>(i));
    }
    static __device__ __forceinline__ void load2(const T *p, int i, R &a, R &b) {
        const __half2 v = __ldg(reinterpret_cast<const __half2 *>(p));
        const float2 r = padd(__half22float2(v), make_float2(wgt<float>(i), wgt<float>(i)));
        a = r.x;
        b = r.y;
    }
    static __device__ __forceinline__ void store2(T *p, R a, R b, int i) {
        const float2 d = psub(make_float2(a, b), make_float2(wgt<float>(i), wgt<float>(i)));
        *reinterpret_cast<__half2 *>(p) = __floats2half2_rn(d.x, d.y);
    }
};
struct StoreBF16 {
    using T = __nv_bfloat16;
    using R = float;
    static __device__ __forceinline__ R load(const T *p, int i) {
        return __bfloat162float(__ldg(p)) + wgt<float>(i);
    }
    static __device__ __forceinline__ R lds(const T *p, int i) {
        return __bfloat162float(*p) + wgt<float>(i);
    }
    static __device__ __forceinline__ void store(T *p, R v, int i) {
        *p = __float2bfloat16_rn(v - wgt<float>(i));
    }
    static __device__ __forceinline__ void load2(const T *p, int i, R &a, R &b) {
        const __nv_bfloat162 v = __ldg(reinterpret_cast<const __nv_bfloat162 *>(p));
        const float2 r = padd(__bfloat1622float2(v), make_float2(wgt<float>(i), wgt<float>(i)));
        a = r.x;
        b = r.y;
    }
    static __device__ __forceinline__ void store2(T *p, R a, R b, int i) {
        const float2 d = psub(make_float2(a, b), make_float2(wgt<float>(i), wgt<float>(i)));
        *reinterpret_cast<__nv_bfloat162 *>(p) = __floats2bfloat162_rn(d.x, d.y);
    }
};

template <typename R> __device__ __forceinline__ R dsqrt(R v);
#ifdef LBM_FAST_ARITH
template <> __device__ __forceinline__ float dsqrt<float>(float v) { return sqrtf(v); }
#else
template <> __device__ __forceinline__ float dsqrt<float>(float v) { return __fsqrt_rn(v); }
#endif
template <> __device__ __forceinline__ double dsqrt<double>(double v) { return __dsqrt_rn(v); }

template <typename R> __device__ __forceinline__ R ddiv(R a, R b);
#ifdef LBM_FAST_ARITH
template <> __device__ __forceinline__ float ddiv<float>(float a, float b) { return __fdividef(a, b); }
#else
template <> __device__ __forceinline__ float ddiv<float>(float a, float b) { return __fdiv_rn(a, b); }
#endif
template <> __device__ __forceinline__ double ddiv<double>(double a, double b) { return __ddiv_rn(a, b); }

// Correctly rounded division by a constant y, given zh = RN(1/y):
//   q1 = RN(x*zh); r = fma(-q1, y, x) (exact); q = fma(r, zh, q1)
// (P. Markstein, IBM J. Res. Dev. 34(1), 1990).  For every divisor it is
// used with, the sequence was checked against IEEE x / y on all 2^32
// single-precision inputs (tests/native/cdiv_check.c): it agrees whenever
// x == 0 or 2^-100 <= |x| <= 2^100.  Outside that range its result still
// has magnitude below 2^-93 for |x| < 2^-100 (q1, r and q are all bounded
// by a few |x|); the callers below only use it where such a value is
// absorbed exactly as the IEEE quotient would be.  Double precision always
// divides with the IEEE operation.
template <typename R> __device__ __forceinline__ R cdiv(R x, R y, R zh);
template <>
__device__ __forceinline__ float cdiv<float>(float x, float y, float zh) {
#ifdef LBM_FAST_ARITH
    (void)y;
    return x * zh;
#else
    const float q1 = __fmul_rn(x, zh);
    const float r = __fmaf_rn(-q1, y, x);
    return __fmaf_rn(r, zh, q1);
#endif
}
template <>
__device__ __forceinline__ double cdiv<double>(double x, double y, double) {
    return __ddiv_rn(x, y);
}

// Equilibrium (lbm_collide.comp:94-101, lbm_force.comp:87-92):
// feq_i(rho, u) = w_i rho (1 + eu/cs2 + eu^2/(2 cs2^2) - u^2/(2 cs2))
// evaluated in the reference's order (lbm.c:37-44).  The three quotients
// are by the constants cs2, 2 cs2^2 and 2 cs2 and use cdiv, which equals
// the IEEE quotient here: a numerator below 2^-100 gives a quotient that
// 1 + ... absorbs either way.
template <typename R>
__device__ __forceinline__ R feq(int i, R rho, R ux, R uy, R uz) {
    R eu = R(cx(i)) * ux + R(cy(i)) * uy + R(cz(i)) * uz;
    R u2 = ux * ux + uy * uy + uz * uz;
    constexpr R cs2 = R(1) / R(3);
    constexpr R c2 = R(2) * cs2 * cs2;
    constexpr R c1 = R(2) * cs2;
    return wgt<R>(i) * rho *
           (((R(1) + cdiv<R>(eu, cs2, R(1) / cs2)) + cdiv<R>(eu * eu, c2, R(1) / c2)) -
            cdiv<R>(u2, c1, R(1) / c1));
}

// a*b + c with one rounding.  Used only where a is +-2, +-4 or +-8, so the
// product is exact and the result equals the separately rounded a*b + c.
template <typename R> __device__ __forceinline__ R fmx(R a, R b, R c);
template <> __device__ __forceinline__ float fmx<float>(float a, float b, float c) {
    return __fmaf_rn(a, b, c);
}
template <> __device__ __forceinline__ double fmx<double>(double a, double b, double c) {
    return __fma_rn(a, b, c);
}

// Paired single precision (sm_100 f32x2 add / sub / mul / fma): two
// independent IEEE round-to-nearest operations per instruction, so every
// lane is bit-identical to the scalar operation it replaces.  They are
// issued as PTX with an explicit .rn modifier, which forbids the compiler
// from contracting a paired multiply and add into one fused operation.
__device__ __forceinline__ unsigned long long pbits(float2 a) {
    return (unsigned long long)__float_as_uint(a.x) |
           ((unsigned long long)__float_as_uint(a.y) << 32);
}
__device__ __forceinline__ float2 pfloat(unsigned long long d) {
    return make_float2(__uint_as_float((unsigned)d), __uint_as_float((unsigned)(d >> 32)));
}
__device__ __forceinline__ float2 p2(float a, float b) { return make_float2(a, b); }
// Operands pass through .b64 registers inside the asm block, so a constant
// operand is moved as a bit pattern (an immediate on the arithmetic
// instruction itself would be read as a number).
__device__ __forceinline__ float2 padd(float2 a, float2 b) {
    unsigned long long d;
    asm("{\n\t.reg .b64 ra, rb;\n\tmov.b64 ra, %1;\n\tmov.b64 rb, %2;\n\t"
        "add.rn.f32x2 %0, ra, rb;\n\t}"
        : "=l"(d) : "l"(pbits(a)), "l"(pbits(b)));
    return pfloat(d);
}
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
    unsigned long long d;
    asm("{\n\t.reg .b64 ra, rb;\n\tmov.b64 ra, %1;\n\tmov.b64 rb, %2;\n\t"
        "sub.rn.f32x2 %0, ra, rb;\n\t}"
        : "=l"(d) : "l"(pbits(a)), "l"(pbits(b)));
    return pfloat(d);
}
__device__ __forceinline__ float2 pmul(float2 a, float2 b) {
    unsigned long long d;
    asm("{\n\t.reg .b64 ra, rb;\n\tmov.b64 ra, %1;\n\tmov.b64 rb, %2;\n\t"
        "mul.rn.f32x2 %0, ra, rb;\n\t}"
        : "=l"(d) : "l"(pbits(a)), "l"(pbits(b)));
    return pfloat(d);
}
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) {
    unsigned long long d;
    asm("{\n\t.reg .b64 ra, rb, rc;\n\tmov.b64 ra, %1;\n\tmov.b64 rb, %2;\n\tmov.b64 rc, %3;\n\t"
        "fma.rn.f32x2 %0, ra, rb, rc;\n\t}"
        : "=l"(d) : "l"(pbits(a)), "l"(pbits(b)), "l"(pbits(c)));
    return pfloat(d);
}
__device__ __forceinline__ float2 pneg(float2 a) { return make_float2(-a.x, -a.y); }
// Measured on sm_100: a paired multiply whose result feeds a paired add or
// subtract is contracted into one fused operation even with explicit .rn,
// and so are pairs of scalar multiplies the compiler merges.  Paired
// arithmetic is therefore used only where no product feeds a paired sum:
// sums, and fused operations whose products are exact or intended.

// Zou-He boundaries (lbm_collide.comp:336-408); rewrite f in place.
template <typename R>
__device__ __forceinline__ void zou_he_inlet(R (&f)[19], R ux, R uy, R uz) {
    R f0 = f[0], f2 = f[2], f3 = f[3], f4 = f[4], f5 = f[5], f6 = f[6];
    R f8 = f[8], f10 = f[10], f12 = f[12], f14 = f[14];
    R f15 = f[15], f16 = f[16], f17 = f[17], f18 = f[18];
    R knowns_0 = f0 + f3 + f4 + f5 + f6 + f15 + f16 + f17 + f18;
    R knowns_neg = f2 + f8 + f10 + f12 + f14;
    R rho_in = ddiv<R>(knowns_0 + R(2) * knowns_neg, R(1) - ux);
    f[1] = f2 + (R(1) / R(3)) * rho_in * ux;
    f[7] = f10 + (R(1) / R(6)) * rho_in * (ux + uy);
    f[9] = f8 + (R(1) / R(6)) * rho_in * (ux - uy);
    f[11] = f14 + (R(1) / R(6)) * rho_in * (ux + uz);
    f[13] = f12 + (R(1) / R(6)) * rho_in * (ux - uz);
}

template <typename R>
__device__ __forceinline__ void zou_he_outlet(R (&f)[19]) {
    R f0 = f[0], f1 = f[1], f3 = f[3], f4 = f[4], f5 = f[5], f6 = f[6];
    R f7 = f[7], f9 = f[9], f11 = f[11], f13 = f[13];
    R f15 = f[15], f16 = f[16], f17 = f[17], f18 = f[18];
    R knowns_0 = f0 + f3 + f4 + f5 + f6 + f15 + f16 + f17 + f18;
    R knowns_pos = f1 + f7 + f9 + f11 + f13;
    const R rho_out = R(1);
    R ux = R(-1) + (knowns_0 + R(2) * knowns_pos) / rho_out;
    f[2] = f1 - (R(1) / R(3)) * rho_out * ux;
    f[10] = f7 - (R(1) / R(6)) * rho_out * ux;
    f[8] = f9 - (R(1) / R(6)) * rho_out * ux;
    f[14] = f11 - (R(1) / R(6)) * rho_out * ux;
    f[12] = f13 - (R(1) / R(6)) * rho_out * ux;
}

// length(u) > 0.40 of the guard.  sqrt is correctly rounded and monotone,
// so in single precision RN(sqrt(u2)) > 0.4f exactly when u2 > 0x3e23d70b
// (0.16000001f), the largest float whose rounded square root is 0.4f
// (checked over every float in tests/test_const_division.py).
__device__ __forceinline__ bool speed_exceeds(float u2) {
    return u2 > __uint_as_float(0x3e23d70bu);
}
__device__ __forceinline__ bool speed_exceeds(double u2) { return __dsqrt_rn(u2) > 0.40; }

// Macroscopic moments (:411-424) and the stability guard test (:429-430).
// Returns true when the cell must be reset to feq(1, 0).
template <typename R>
__device__ __forceinline__ bool moments(const R (&f)[19], R &rho, R &ux, R &uy, R &uz) {
    // The shader accumulates rho += f_i and u += e_i f_i over i = 0..18.  The
    // e-components are 0 or +-1, so u is the signed sum of the f_i with a
    // nonzero component, in index order (a 0 * f_i term only adds a signed
    // zero and cannot change a value).
    rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8] + f[9] + f[10] + f[11] +
          f[12] + f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
    ux = f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[11] - f[12] + f[13] - f[14];
    uy = f[3] - f[4] + f[7] + f[8] - f[9] - f[10] + f[15] - f[16] + f[17] - f[18];
    uz = f[5] - f[6] + f[11] + f[12] - f[13] - f[14] + f[15] + f[16] - f[17] - f[18];
    if (rho > R(0.0001)) {
        ux = ddiv<R>(ux, rho);
        uy = ddiv<R>(uy, rho);
        uz = ddiv<R>(uz, rho);
    }
    return rho < R(0.3) || rho > R(2.0) || speed_exceeds(ux * ux + uy * uy + uz * uz) ||
           isinf(rho) || isnan(rho);
}

// Boundary/solid preprocessing shared by the step and the velocity
// recomputation: applies the solid rule, Zou-He and the guard.  Returns
//   0  -> fluid cell, f holds the (possibly Zou-He rewritten) populations
//         and rho/u the moments;
//   1  -> solid body cell (velocity (0,0,0,1));
//   2  -> guard reset (velocity (0,0,0,1), populations feq(1,0)).
template <typename R>
__device__ __forceinline__ int prepare_cell(R (&f)[19], int solid, int x, int nx,
                                            R inX, R inY, R inZ, R &rho, R &ux,
                                            R &uy, R &uz) {
    if (solid == 1) {
        rho = R(1);
        ux = uy = uz = R(0);
        return 1;
    }
    if (x == 0) zou_he_inlet<R>(f, inX, inY, inZ);
    if (x == nx - 1) zou_he_outlet<R>(f);
    if (moments<R>(f, rho, ux, uy, uz)) {
        rho = R(1);
        ux = uy = uz = R(0);
        return 2;
    }
    return 0;
}

// MRT transforms (lbm_collide.comp:110-181, :185-311)
template <typename R>
__device__ __forceinline__ void mrt_forward(const R (&fi)[19], R (&m)[19]) {
    // Terms of the form (2^k) * s + t use one fused operation: the product
    // by a power of two is exact, so the single rounding equals the
    // shader's two.
    R sf = fi[1] + fi[2] + fi[3] + fi[4] + fi[5] + fi[6];
    R se = fi[7] + fi[8] + fi[9] + fi[10] + fi[11] + fi[12] + fi[13] + fi[14] + fi[15] + fi[16] +
           fi[17] + fi[18];
    m[0] = fi[0] + sf + se;
    m[1] = fmx<R>(R(8), se, R(-30) * fi[0] - R(11) * sf);
    m[2] = fmx<R>(R(-4), sf, R(12) * fi[0]) + se;
    const R d12 = fi[1] - fi[2], d34 = fi[3] - fi[4], d56 = fi[5] - fi[6];
    m[3] = d12 + fi[7] - fi[8] + fi[9] - fi[10] + fi[11] - fi[12] + fi[13] - fi[14];
    m[4] = fmx<R>(R(-4), d12, fi[7]) - fi[8] + fi[9] - fi[10] + fi[11] - fi[12] + fi[13] - fi[14];
    m[5] = d34 + fi[7] + fi[8] - fi[9] - fi[10] + fi[15] - fi[16] + fi[17] - fi[18];
    m[6] = fmx<R>(R(-4), d34, fi[7]) + fi[8] - fi[9] - fi[10] + fi[15] - fi[16] + fi[17] - fi[18];
    m[7] = d56 + fi[11] + fi[12] - fi[13] - fi[14] + fi[15] + fi[16] - fi[17] - fi[18];
    m[8] = fmx<R>(R(-4), d56, fi[11]) + fi[12] - fi[13] - fi[14] + fi[15] + fi[16] - fi[17] -
           fi[18];
    const R sXY = fi[7] + fi[8] + fi[9] + fi[10];
    const R sXZ = fi[11] + fi[12] + fi[13] + fi[14];
    const R sYZ = fi[15] + fi[16] + fi[17] + fi[18];
    const R s12 = fi[1] + fi[2], s34 = fi[3] + fi[4], s56 = fi[5] + fi[6];
    m[9] = fmx<R>(R(-2), sYZ, fmx<R>(R(2), s12, -s34) - s56 + sXY + sXZ);
    m[10] = fmx<R>(R(-2), sYZ, fmx<R>(R(2), s56, fmx<R>(R(2), s34, R(-4) * s12)) + sXY + sXZ);
    m[11] = s34 - s56 + sXY - sXZ;
    m[12] = fmx<R>(R(2), s56, R(-2) * s34) + sXY - sXZ;
    m[13] = fi[7] - fi[8] - fi[9] + fi[10];
    m[14] = fi[15] - fi[16] - fi[17] + fi[18];
    m[15] = fi[11] - fi[12] - fi[13] + fi[14];
    m[16] = fi[7] - fi[8] + fi[9] - fi[10] - fi[11] + fi[12] - fi[13] + fi[14];
    m[17] = -fi[7] - fi[8] + fi[9] + fi[10] + fi[15] - fi[16] + fi[17] - fi[18];
    m[18] = fi[11] + fi[12] - fi[13] - fi[14] - fi[15] - fi[16] + fi[17] + fi[18];
}

template <typename R>
__device__ __forceinline__ void mrt_inverse(const R (&m)[19], R (&fi)[19]) {
    // m_k / |M_k|^2 (lbm_collide.comp:187-205).  The divisors are constants
    // checked with cdiv on all 2^32 inputs; a quotient that cdiv could get
    // wrong has magnitude below 2^-93 and every population below sums it
    // into terms led by m_0 / 19 = rho / 19, which absorb it either way.
    auto q = [](R x, R y) { return cdiv<R>(x, y, R(1) / y); };
    R ms[19];
    ms[0] = q(m[0], R(19));
    ms[1] = q(m[1], R(2394));
    ms[2] = q(m[2], R(252));
    ms[3] = q(m[3], R(10));
    ms[4] = q(m[4], R(40));
    ms[5] = q(m[5], R(10));
    ms[6] = q(m[6], R(40));
    ms[7] = q(m[7], R(10));
    ms[8] = q(m[8], R(40));
    ms[9] = q(m[9], R(36));
    ms[10] = q(m[10], R(72));
    ms[11] = q(m[11], R(12));
    ms[12] = q(m[12], R(24));
    ms[13] = m[13] * R(0.25);  // division by a power of two is exact
    ms[14] = m[14] * R(0.25);
    ms[15] = m[15] * R(0.25);
    ms[16] = m[16] * R(0.125);
    ms[17] = m[17] * R(0.125);
    ms[18] = m[18] * R(0.125);

    // lbm_collide.comp:210-310, left to right; products by 2, 4, 8 fused
#if !defined(LBM_FAST_ARITH) && !defined(LBM_NO_PAIRED)
    if constexpr (sizeof(R) == 4) {
        // Populations in pairs (i, j) whose sums take the same operands in
        // the same order with per-lane signs: each step is one paired
        // fma with a sign pair in {+-1, +-2, +-4} (exact products), i.e.
        // the scalar add or subtract of the shader on both lanes.
        float2 B[19];
#pragma unroll
        for (int k = 0; k < 19; k++) B[k] = p2(ms[k], ms[k]);
        auto S = [](float a, float b) { return p2(a, b); };
        fi[0] = (ms[0] - R(30) * ms[1]) + R(12) * ms[2];
        const float a0 = fmx<R>(R(-4), ms[2], ms[0] - R(11) * ms[1]);
        const float b0 = fmx<R>(R(8), ms[1], ms[0]) + ms[2];
        const float2 A0 = p2(a0, a0), B0 = p2(b0, b0);
        float2 P;
        P = pfma(S(1, -1), B[3], A0);
        P = pfma(S(-4, 4), B[4], P);
        P = pfma(S(2, 2), B[9], P);
        P = pfma(S(-4, -4), B[10], P);
        fi[1] = P.x, fi[2] = P.y;
        P = pfma(S(1, -1), B[5], A0);
        P = pfma(S(-4, 4), B[6], P);
        P = psub(P, B[9]);
        P = pfma(S(2, 2), B[10], P);
        P = padd(P, B[11]);
        P = pfma(S(-2, -2), B[12], P);
        fi[3] = P.x, fi[4] = P.y;
        P = pfma(S(1, -1), B[7], A0);
        P = pfma(S(-4, 4), B[8], P);
        P = psub(P, B[9]);
        P = pfma(S(2, 2), B[10], P);
        P = psub(P, B[11]);
        P = pfma(S(2, 2), B[12], P);
        fi[5] = P.x, fi[6] = P.y;
        P = pfma(S(1, -1), B[3], B0);  // 7, 8
        P = pfma(S(1, -1), B[4], P);
        P = padd(P, B[5]);
        P = padd(P, B[6]);
        P = padd(P, B[9]);
        P = padd(P, B[10]);
        P = padd(P, B[11]);
        P = padd(P, B[12]);
        P = pfma(S(1, -1), B[13], P);
        P = pfma(S(1, -1), B[16], P);
        P = psub(P, B[17]);
        fi[7] = P.x, fi[8] = P.y;
        P = pfma(S(1, -1), B[3], B0);  // 9, 10
        P = pfma(S(1, -1), B[4], P);
        P = psub(P, B[5]);
        P = psub(P, B[6]);
        P = padd(P, B[9]);
        P = padd(P, B[10]);
        P = padd(P, B[11]);
        P = padd(P, B[12]);
        P = pfma(S(-1, 1), B[13], P);
        P = pfma(S(1, -1), B[16], P);
        P = padd(P, B[17]);
        fi[9] = P.x, fi[10] = P.y;
        P = pfma(S(1, -1), B[3], B0);  // 11, 12
        P = pfma(S(1, -1), B[4], P);
        P = padd(P, B[7]);
        P = padd(P, B[8]);
        P = padd(P, B[9]);
        P = padd(P, B[10]);
        P = psub(P, B[11]);
        P = psub(P, B[12]);
        P = pfma(S(1, -1), B[15], P);
        P = pfma(S(-1, 1), B[16], P);
        P = padd(P, B[18]);
        fi[11] = P.x, fi[12] = P.y;
        P = pfma(S(1, -1), B[3], B0);  // 13, 14
        P = pfma(S(1, -1), B[4], P);
        P = psub(P, B[7]);
        P = psub(P, B[8]);
        P = padd(P, B[9]);
        P = padd(P, B[10]);
        P = psub(P, B[11]);
        P = psub(P, B[12]);
        P = pfma(S(-1, 1), B[15], P);
        P = pfma(S(-1, 1), B[16], P);
        P = psub(P, B[18]);
        fi[13] = P.x, fi[14] = P.y;
        P = pfma(S(1, -1), B[5], B0);  // 15, 16
        P = pfma(S(1, -1), B[6], P);
        P = padd(P, B[7]);
        P = padd(P, B[8]);
        P = pfma(S(-2, -2), B[9], P);
        P = pfma(S(-2, -2), B[10], P);
        P = pfma(S(1, -1), B[14], P);
        P = pfma(S(1, -1), B[17], P);
        P = psub(P, B[18]);
        fi[15] = P.x, fi[16] = P.y;
        P = pfma(S(1, -1), B[5], B0);  // 17, 18
        P = pfma(S(1, -1), B[6], P);
        P = psub(P, B[7]);
        P = psub(P, B[8]);
        P = pfma(S(-2, -2), B[9], P);
        P = pfma(S(-2, -2), B[10], P);
        P = pfma(S(-1, 1), B[14], P);
        P = pfma(S(1, -1), B[17], P);
        P = padd(P, B[18]);
        fi[17] = P.x, fi[18] = P.y;
        return;
    }
#endif
    fi[0] = (ms[0] - R(30) * ms[1]) + R(12) * ms[2];
    const R a0 = fmx<R>(R(-4), ms[2], ms[0] - R(11) * ms[1]);  // ms0 - 11ms1 - 4ms2
    fi[1] = fmx<R>(R(-4), ms[10], fmx<R>(R(2), ms[9], fmx<R>(R(-4), ms[4], a0 + ms[3])));
    fi[2] = fmx<R>(R(-4), ms[10], fmx<R>(R(2), ms[9], fmx<R>(R(4), ms[4], a0 - ms[3])));
    fi[3] = fmx<R>(R(-2), ms[12],
                   fmx<R>(R(2), ms[10], fmx<R>(R(-4), ms[6], a0 + ms[5]) - ms[9]) + ms[11]);
    fi[4] = fmx<R>(R(-2), ms[12],
                   fmx<R>(R(2), ms[10], fmx<R>(R(4), ms[6], a0 - ms[5]) - ms[9]) + ms[11]);
    fi[5] = fmx<R>(R(2), ms[12],
                   fmx<R>(R(2), ms[10], fmx<R>(R(-4), ms[8], a0 + ms[7]) - ms[9]) - ms[11]);
    fi[6] = fmx<R>(R(2), ms[12],
                   fmx<R>(R(2), ms[10], fmx<R>(R(4), ms[8], a0 - ms[7]) - ms[9]) - ms[11]);
    const R b0 = fmx<R>(R(8), ms[1], ms[0]) + ms[2];  // ms0 + 8ms1 + ms2
    fi[7] = b0 + ms[3] + ms[4] + ms[5] + ms[6] + ms[9] + ms[10] + ms[11] + ms[12] + ms[13] + ms[16] -
            ms[17];
    fi[8] = b0 - ms[3] - ms[4] + ms[5] + ms[6] + ms[9] + ms[10] + ms[11] + ms[12] - ms[13] - ms[16] -
            ms[17];
    fi[9] = b0 + ms[3] + ms[4] - ms[5] - ms[6] + ms[9] + ms[10] + ms[11] + ms[12] - ms[13] + ms[16] +
            ms[17];
    fi[10] = b0 - ms[3] - ms[4] - ms[5] - ms[6] + ms[9] + ms[10] + ms[11] + ms[12] + ms[13] -
             ms[16] + ms[17];
    fi[11] = b0 + ms[3] + ms[4] + ms[7] + ms[8] + ms[9] + ms[10] - ms[11] - ms[12] + ms[15] -
             ms[16] + ms[18];
    fi[12] = b0 - ms[3] - ms[4] + ms[7] + ms[8] + ms[9] + ms[10] - ms[11] - ms[12] - ms[15] +
             ms[16] + ms[18];
    fi[13] = b0 + ms[3] + ms[4] - ms[7] - ms[8] + ms[9] + ms[10] - ms[11] - ms[12] - ms[15] -
             ms[16] - ms[18];
    fi[14] = b0 - ms[3] - ms[4] - ms[7] - ms[8] + ms[9] + ms[10] - ms[11] - ms[12] + ms[15] +
             ms[16] - ms[18];
    fi[15] = fmx<R>(R(-2), ms[10], fmx<R>(R(-2), ms[9], b0 + ms[5] + ms[6] + ms[7] + ms[8])) +
             ms[14] + ms[17] - ms[18];
    fi[16] = fmx<R>(R(-2), ms[10], fmx<R>(R(-2), ms[9], b0 - ms[5] - ms[6] + ms[7] + ms[8])) -
             ms[14] - ms[17] - ms[18];
    fi[17] = fmx<R>(R(-2), ms[10], fmx<R>(R(-2), ms[9], b0 + ms[5] + ms[6] - ms[7] - ms[8])) -
             ms[14] + ms[17] + ms[18];
    fi[18] = fmx<R>(R(-2), ms[10], fmx<R>(R(-2), ms[9], b0 - ms[5] - ms[6] - ms[7] - ms[8])) +
             ms[14] - ms[17] + ms[18];
}

// Equilibria of the 19 directions (lbm_collide.comp:94-101):
//   feq_i = (w_i rho) * (((1 + eu_i/cs2) + eu_i^2/(2 cs2^2)) - u^2/(2 cs2))
// with eu_i evaluated exactly as the shader's (e_x ux + e_y uy) + e_z uz.
// Opposite directions have eu_j = -eu_i, and rounding is sign-symmetric,
// so each pair shares its two quotients.  The quotients by the constants
// use cdiv: when |eu| >= 2^-50 (and u^2 >= 2^-100) every operand is in the
// verified range; when |eu| < 2^-50, eu/cs2 and eu^2/(2cs2^2) are below
// 2^-90 under either division, and 1 + a, (1 + a) + b and s - cu round to
// the same floats, so the result is the IEEE one in every case.
template <typename R>
__device__ __forceinline__ void equilibria(R rho, R ux, R uy, R uz, R (&fe)[19]) {
    constexpr R cs2 = R(1) / R(3);
    constexpr R c1 = R(2) * cs2;
    constexpr R c2 = R(2) * cs2 * cs2;
    const R u2 = ux * ux + uy * uy + uz * uz;
    const R cu = cdiv<R>(u2, c1, R(1) / c1);
    const R wr0 = wgt<R>(0) * rho, wr1 = wgt<R>(1) * rho, wr2 = wgt<R>(7) * rho;
    fe[0] = wr0 * (R(1) - cu);
    auto pair = [&](R e, R wr, R &fi, R &fj) {
        const R a = cdiv<R>(e, cs2, R(1) / cs2);
        const R b = cdiv<R>(e * e, c2, R(1) / c2);
        fi = wr * (((R(1) + a) + b) - cu);
        fj = wr * (((R(1) - a) + b) - cu);
    };
#if !defined(LBM_FAST_ARITH) && !defined(LBM_NO_PAIRED)
    if constexpr (sizeof(R) == 4) {
        // two direction pairs per paired instruction; lane k evaluates the
        // scalar sequence of `pair` above.  Only sums and fused operations
        // of the Markstein quotient are paired: a paired product that feeds
        // a paired sum is contracted by the compiler (measured on sm_100).
        const float2 ONE = p2(1.0f, 1.0f), CU = p2(cu, cu);
        const float2 Y1 = p2(cs2, cs2), Z1 = p2(1.0f / cs2, 1.0f / cs2);
        const float2 Y2 = p2(c2, c2), Z2 = p2(1.0f / c2, 1.0f / c2);
        auto lanes = [&](float e0, float e1, float w0, float w1, float &fi0, float &fj0,
                         float &fi1, float &fj1) {
            const float2 E = p2(e0, e1);
            const float2 E2 = pmul(E, E);
            // Markstein: q1 = RN(x zh); r = fma(-q1, y, x); q = fma(r, zh, q1)
            const float2 q1a = pmul(E, Z1);
            const float2 ra = pfma(pneg(q1a), Y1, E);
            const float2 a = pfma(ra, Z1, q1a);
            const float2 q1b = pmul(E2, Z2);
            const float2 rb = pfma(pneg(q1b), Y2, E2);
            const float2 b = pfma(rb, Z2, q1b);
            const float2 Si = psub(padd(padd(ONE, a), b), CU);
            const float2 Sj = psub(padd(psub(ONE, a), b), CU);
            // the products by w rho stay scalar: they feed subtractions
            fi0 = __fmul_rn(w0, Si.x);
            fi1 = __fmul_rn(w1, Si.y);
            fj0 = __fmul_rn(w0, Sj.x);
            fj1 = __fmul_rn(w1, Sj.y);
        };
        lanes(ux, uy, wr1, wr1, fe[1], fe[2], fe[3], fe[4]);
        lanes(uz, ux + uy, wr1, wr2, fe[5], fe[6], fe[7], fe[10]);
        lanes(uy - ux, ux + uz, wr2, wr2, fe[8], fe[9], fe[11], fe[14]);
        lanes(uz - ux, uy + uz, wr2, wr2, fe[12], fe[13], fe[15], fe[18]);
        pair(uz - uy, wr2, fe[16], fe[17]);
        return;
    }
#endif
    pair(ux, wr1, fe[1], fe[2]);
    pair(uy, wr1, fe[3], fe[4]);
    pair(uz, wr1, fe[5], fe[6]);
    pair(ux + uy, wr2, fe[7], fe[10]);
    pair(uy - ux, wr2, fe[8], fe[9]);
    pair(ux + uz, wr2, fe[11], fe[14]);
    pair(uz - ux, wr2, fe[12], fe[13]);
    pair(uy + uz, wr2, fe[15], fe[18]);
    pair(uz - uy, wr2, fe[16], fe[17]);
}

// Non-equilibrium stress Pi_ab = sum_i e_ia e_ib (f_i - feq_i)
// (lbm_collide.comp:455-470, identical to :500-515), nonzero terms in
// index order.
template <typename R>
__device__ __forceinline__ void stress(const R (&f)[19], const R (&fe)[19], R &Pxx, R &Pyy,
                                       R &Pzz, R &Pxy, R &Pxz, R &Pyz) {
    R n[19];
#pragma unroll
    for (int i = 0; i < 19; i++) n[i] = f[i] - fe[i];
    Pxx = n[1] + n[2] + n[7] + n[8] + n[9] + n[10] + n[11] + n[12] + n[13] + n[14];
    Pyy = n[3] + n[4] + n[7] + n[8] + n[9] + n[10] + n[15] + n[16] + n[17] + n[18];
    Pzz = n[5] + n[6] + n[11] + n[12] + n[13] + n[14] + n[15] + n[16] + n[17] + n[18];
    Pxy = n[7] - n[8] - n[9] + n[10];
    Pxz = n[11] - n[12] - n[13] + n[14];
    Pyz = n[15] - n[16] - n[17] + n[18];
}

// Collision (lbm_collide.comp:445-625).  OP: 0 BGK, 1 regularized, 2 MRT.
// `omega_tau` is 1/tau computed on the host (the same IEEE quotient) and
// used when SMAG is off; `smag18` is 18*Cs*Cs.
template <typename R, int OP, bool SMAG>
__device__ __forceinline__ void collide(const R (&f)[19], R (&fn)[19], R rho, R ux, R uy, R uz,
                                        R tau, R omega_tau, R smag18) {
    R fe[19];
    if (SMAG || OP != OP_MRT) equilibria<R>(rho, ux, uy, uz, fe);
    R omega = omega_tau;
    R Pxx, Pyy, Pzz, Pxy, Pxz, Pyz;
    if (SMAG || OP == OP_REG) stress<R>(f, fe, Pxx, Pyy, Pzz, Pxy, Pxz, Pyz);
    if (SMAG) {
        // :472-484
        const R Pi_norm = dsqrt<R>(
            fmx<R>(R(2), Pxy * Pxy + Pxz * Pxz + Pyz * Pyz, Pxx * Pxx + Pyy * Pyy + Pzz * Pzz));
        const R tau_eff =
            R(0.5) * (tau + dsqrt<R>(tau * tau + ddiv<R>(smag18 * Pi_norm, rho + R(1e-10))));
        omega = ddiv<R>(R(1), tau_eff);
    }
    if (OP == OP_REG) {
        // :517-543: f_i = feq_i + (1 - omega) (w_i 4.5) Q_i:Pi, Q_i:Pi summed
        // in the shader's order with the zero products dropped
        constexpr R cs2 = R(1) / R(3);
        constexpr R k1 = R(1) - cs2;  // e_a^2 - cs2 for e_a = +-1
        constexpr R k0 = R(0) - cs2;  // e_a^2 - cs2 for e_a = 0
        const R om = R(1) - omega;
        const R Q0 = (k0 * Pxx + k0 * Pyy) + k0 * Pzz;
        const R Qx = (k1 * Pxx + k0 * Pyy) + k0 * Pzz;
        const R Qy = (k0 * Pxx + k1 * Pyy) + k0 * Pzz;
        const R Qz = (k0 * Pxx + k0 * Pyy) + k1 * Pzz;
        const R Txy = (k1 * Pxx + k1 * Pyy) + k0 * Pzz;
        const R Txz = (k1 * Pxx + k0 * Pyy) + k1 * Pzz;
        const R Tyz = (k0 * Pxx + k1 * Pyy) + k1 * Pzz;
        R Q[19];
        Q[0] = Q0;
        Q[1] = Q[2] = Qx;
        Q[3] = Q[4] = Qy;
        Q[5] = Q[6] = Qz;
        Q[7] = Q[10] = fmx<R>(R(2), Pxy, Txy);
        Q[8] = Q[9] = fmx<R>(R(-2), Pxy, Txy);
        Q[11] = Q[14] = fmx<R>(R(2), Pxz, Txz);
        Q[12] = Q[13] = fmx<R>(R(-2), Pxz, Txz);
        Q[15] = Q[18] = fmx<R>(R(2), Pyz, Tyz);
        Q[16] = Q[17] = fmx<R>(R(-2), Pyz, Tyz);
        {
#pragma unroll
            for (int i = 0; i < 19; i++) fn[i] = fe[i] + om * ((wgt<R>(i) * R(4.5)) * Q[i]);
        }
    } else if (OP == OP_MRT) {
        // :550-616
        R m[19], meq[19];
        mrt_forward<R>(f, m);
        const R uyy = uy * uy, uzz = uz * uz;
        const R u2 = ux * ux + uyy + uzz;
        const R pxx = R(2) * ux * ux - uyy - uzz;  // (2 ux) ux - uy^2 - uz^2
        const R pww = uyy - uzz;
        meq[1] = R(-11) * rho + R(19) * rho * u2;
        meq[2] = R(3) * rho - R(5.5) * rho * u2;
        meq[4] = R(-2) / R(3) * rho * ux;
        meq[6] = R(-2) / R(3) * rho * uy;
        meq[8] = R(-2) / R(3) * rho * uz;
        meq[9] = rho * pxx;
        meq[10] = R(-0.5) * rho * pxx;
        meq[11] = rho * pww;
        meq[12] = R(-0.5) * rho * pww;
        meq[13] = rho * ux * uy;
        meq[14] = rho * uy * uz;
        meq[15] = rho * ux * uz;
        const R s_nu = omega;
        // relaxation m - s (m - meq); the conserved moments 0, 3, 5, 7 have
        // s = 0 and keep their value; meq of the ghost modes 16-18 is 0
        {
            m[1] = m[1] - R(1.19) * (m[1] - meq[1]);
            m[2] = m[2] - R(1.4) * (m[2] - meq[2]);
            m[4] = m[4] - R(1.2) * (m[4] - meq[4]);
            m[6] = m[6] - R(1.2) * (m[6] - meq[6]);
            m[8] = m[8] - R(1.2) * (m[8] - meq[8]);
            m[9] = m[9] - s_nu * (m[9] - meq[9]);
            m[10] = m[10] - R(1.4) * (m[10] - meq[10]);
            m[11] = m[11] - s_nu * (m[11] - meq[11]);
            m[12] = m[12] - R(1.4) * (m[12] - meq[12]);
            m[13] = m[13] - s_nu * (m[13] - meq[13]);
            m[14] = m[14] - s_nu * (m[14] - meq[14]);
            m[15] = m[15] - s_nu * (m[15] - meq[15]);
            m[16] = m[16] - R(1.98) * m[16];
            m[17] = m[17] - R(1.98) * m[17];
            m[18] = m[18] - R(1.98) * m[18];
        }
        mrt_inverse<R>(m, fn);
    } else {
        // :618-625
        {
#pragma unroll
            for (int i = 0; i < 19; i++) fn[i] = f[i] - omega * (f[i] - fe[i]);
        }
    }
}

}  // namespace LBM_ARITH_NS
}  // namespace lbm
