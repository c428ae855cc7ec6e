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

namespace lbm {

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
struct StoreF32 {
    using T = float;
    using R = float;
    static __device__ __forceinline__ R load(const T *p, int) { return __ldg(p); }
    static __device__ __forceinline__ void store(T *p, R v, int) { *p = v; }
};
struct StoreF64 {
    using T = double;
    using R = double;
    static __device__ __forceinline__ R load(const T *p, int) { return __ldg(p); }
    static __device__ __forceinline__ void store(T *p, R v, int) { *p = v; }
};
struct StoreF16 {
    using T = __half;
    using R = float;
    static __device__ __forceinline__ R load(const T *p, int i) {
        return __half2float(__ldg(p)) + wgt<float>(i);
    }
    static __device__ __forceinline__ void store(T *p, R v, int i) {
        *p = __float2half_rn(v - wgt<float>(i));
    }
};
struct StoreBF16 {
    using T = __nv_bfloat16;
    using R = float;
    static __device__ __forceinline__ R load(const T *p, int i) {
        return __bfloat162float(__ldg(p)) + wgt<float>(i);
    }
    static __device__ __forceinline__ void store(T *p, R v, int i) {
        *p = __float2bfloat16_rn(v - wgt<float>(i));
    }
};

// ---------------------------------------------------------------------
// Equilibrium (lbm_collide.comp:94-101, lbm_force.comp:216-221)
// ---------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ R feq(int i, R rho, R ux, R uy, R uz) {
    R eu = R(cx(i)) * ux + R(cy(i)) * uy + R(cz(i)) * uz;
    R u2 = ux * ux + uy * uy + uz * uz;
    const R cs2 = R(1) / R(3);
    return wgt<R>(i) * rho *
           (R(1) + eu / cs2 + (eu * eu) / (R(2) * cs2 * cs2) - u2 / (R(2) * cs2));
}

template <typename R> __device__ __forceinline__ R dsqrt(R v);
template <> __device__ __forceinline__ float dsqrt<float>(float v) { return __fsqrt_rn(v); }
template <> __device__ __forceinline__ double dsqrt<double>(double v) { return __dsqrt_rn(v); }

template <typename R> __device__ __forceinline__ R ddiv(R a, R b);
template <> __device__ __forceinline__ float ddiv<float>(float a, float b) { return __fdiv_rn(a, b); }
template <> __device__ __forceinline__ double ddiv<double>(double a, double b) { return __ddiv_rn(a, b); }

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

// Macroscopic moments (:411-424) and the stability guard test (:429-430).
// Returns true when the cell must be reset to feq(1, 0).
template <typename R>
__device__ __forceinline__ bool moments(const R (&f)[19], R &rho, R &ux, R &uy, R &uz) {
    rho = R(0);
    ux = R(0);
    uy = R(0);
    uz = R(0);
#pragma unroll
    for (int i = 0; i < 19; i++) {
        R fi = f[i];
        rho += fi;
        ux += R(cx(i)) * fi;
        uy += R(cy(i)) * fi;
        uz += R(cz(i)) * fi;
    }
    if (rho > R(0.0001)) {
        ux = ddiv<R>(ux, rho);
        uy = ddiv<R>(uy, rho);
        uz = ddiv<R>(uz, rho);
    }
    R u_mag = dsqrt<R>(ux * ux + uy * uy + uz * uz);
    return rho < R(0.3) || rho > R(2.0) || u_mag > R(0.40) || isinf(rho) || isnan(rho);
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
    R sf = fi[1] + fi[2] + fi[3] + fi[4] + fi[5] + fi[6];
    R se = fi[7] + fi[8] + fi[9] + fi[10] + fi[11] + fi[12] + fi[13] + fi[14] +
           fi[15] + fi[16] + fi[17] + fi[18];
    m[0] = fi[0] + sf + se;
    m[1] = R(-30) * fi[0] - R(11) * sf + R(8) * se;
    m[2] = R(12) * fi[0] - R(4) * sf + se;
    m[3] = fi[1] - fi[2] + fi[7] - fi[8] + fi[9] - fi[10] + fi[11] - fi[12] + fi[13] - fi[14];
    m[4] = R(-4) * (fi[1] - fi[2]) + fi[7] - fi[8] + fi[9] - fi[10] + fi[11] - fi[12] +
           fi[13] - fi[14];
    m[5] = fi[3] - fi[4] + fi[7] + fi[8] - fi[9] - fi[10] + fi[15] - fi[16] + fi[17] - fi[18];
    m[6] = R(-4) * (fi[3] - fi[4]) + fi[7] + fi[8] - fi[9] - fi[10] + fi[15] - fi[16] +
           fi[17] - fi[18];
    m[7] = fi[5] - fi[6] + fi[11] + fi[12] - fi[13] - fi[14] + fi[15] + fi[16] - fi[17] - fi[18];
    m[8] = R(-4) * (fi[5] - fi[6]) + fi[11] + fi[12] - fi[13] - fi[14] + fi[15] + fi[16] -
           fi[17] - fi[18];
    R sXY = fi[7] + fi[8] + fi[9] + fi[10];
    R sXZ = fi[11] + fi[12] + fi[13] + fi[14];
    R sYZ = fi[15] + fi[16] + fi[17] + fi[18];
    m[9] = R(2) * (fi[1] + fi[2]) - (fi[3] + fi[4]) - (fi[5] + fi[6]) + sXY + sXZ - R(2) * sYZ;
    m[10] = R(-4) * (fi[1] + fi[2]) + R(2) * (fi[3] + fi[4]) + R(2) * (fi[5] + fi[6]) + sXY +
            sXZ - R(2) * sYZ;
    m[11] = (fi[3] + fi[4]) - (fi[5] + fi[6]) + sXY - sXZ;
    m[12] = R(-2) * (fi[3] + fi[4]) + R(2) * (fi[5] + fi[6]) + sXY - sXZ;
    m[13] = fi[7] - fi[8] - fi[9] + fi[10];
    m[14] = fi[15] - fi[16] - fi[17] + fi[18];
    m[15] = fi[11] - fi[12] - fi[13] + fi[14];
    m[16] = fi[7] - fi[8] + fi[9] - fi[10] - fi[11] + fi[12] - fi[13] + fi[14];
    m[17] = -fi[7] - fi[8] + fi[9] + fi[10] + fi[15] - fi[16] + fi[17] - fi[18];
    m[18] = fi[11] + fi[12] - fi[13] - fi[14] - fi[15] - fi[16] + fi[17] + fi[18];
}

template <typename R>
__device__ __forceinline__ void mrt_inverse(const R (&m)[19], R (&fi)[19]) {
    R ms[19];
    ms[0] = ddiv<R>(m[0], R(19));
    ms[1] = ddiv<R>(m[1], R(2394));
    ms[2] = ddiv<R>(m[2], R(252));
    ms[3] = ddiv<R>(m[3], R(10));
    ms[4] = ddiv<R>(m[4], R(40));
    ms[5] = ddiv<R>(m[5], R(10));
    ms[6] = ddiv<R>(m[6], R(40));
    ms[7] = ddiv<R>(m[7], R(10));
    ms[8] = ddiv<R>(m[8], R(40));
    ms[9] = ddiv<R>(m[9], R(36));
    ms[10] = ddiv<R>(m[10], R(72));
    ms[11] = ddiv<R>(m[11], R(12));
    ms[12] = ddiv<R>(m[12], R(24));
    ms[13] = m[13] * R(0.25);   // division by a power of two is exact
    ms[14] = m[14] * R(0.25);
    ms[15] = m[15] * R(0.25);
    ms[16] = m[16] * R(0.125);
    ms[17] = m[17] * R(0.125);
    ms[18] = m[18] * R(0.125);

    fi[0] = ms[0] - R(30) * ms[1] + R(12) * ms[2];
    fi[1] = ms[0] - R(11) * ms[1] - R(4) * ms[2] + ms[3] - R(4) * ms[4] + R(2) * ms[9] -
            R(4) * ms[10];
    fi[2] = ms[0] - R(11) * ms[1] - R(4) * ms[2] - ms[3] + R(4) * ms[4] + R(2) * ms[9] -
            R(4) * ms[10];
    fi[3] = ms[0] - R(11) * ms[1] - R(4) * ms[2] + ms[5] - R(4) * ms[6] - ms[9] +
            R(2) * ms[10] + ms[11] - R(2) * ms[12];
    fi[4] = ms[0] - R(11) * ms[1] - R(4) * ms[2] - ms[5] + R(4) * ms[6] - ms[9] +
            R(2) * ms[10] + ms[11] - R(2) * ms[12];
    fi[5] = ms[0] - R(11) * ms[1] - R(4) * ms[2] + ms[7] - R(4) * ms[8] - ms[9] +
            R(2) * ms[10] - ms[11] + R(2) * ms[12];
    fi[6] = ms[0] - R(11) * ms[1] - R(4) * ms[2] - ms[7] + R(4) * ms[8] - ms[9] +
            R(2) * ms[10] - ms[11] + R(2) * ms[12];
    fi[7] = ms[0] + R(8) * ms[1] + ms[2] + ms[3] + ms[4] + ms[5] + ms[6] + ms[9] + ms[10] +
            ms[11] + ms[12] + ms[13] + ms[16] - ms[17];
    fi[8] = ms[0] + R(8) * ms[1] + ms[2] - ms[3] - ms[4] + ms[5] + ms[6] + ms[9] + ms[10] +
            ms[11] + ms[12] - ms[13] - ms[16] - ms[17];
    fi[9] = ms[0] + R(8) * ms[1] + ms[2] + ms[3] + ms[4] - ms[5] - ms[6] + ms[9] + ms[10] +
            ms[11] + ms[12] - ms[13] + ms[16] + ms[17];
    fi[10] = ms[0] + R(8) * ms[1] + ms[2] - ms[3] - ms[4] - ms[5] - ms[6] + ms[9] + ms[10] +
             ms[11] + ms[12] + ms[13] - ms[16] + ms[17];
    fi[11] = ms[0] + R(8) * ms[1] + ms[2] + ms[3] + ms[4] + ms[7] + ms[8] + ms[9] + ms[10] -
             ms[11] - ms[12] + ms[15] - ms[16] + ms[18];
    fi[12] = ms[0] + R(8) * ms[1] + ms[2] - ms[3] - ms[4] + ms[7] + ms[8] + ms[9] + ms[10] -
             ms[11] - ms[12] - ms[15] + ms[16] + ms[18];
    fi[13] = ms[0] + R(8) * ms[1] + ms[2] + ms[3] + ms[4] - ms[7] - ms[8] + ms[9] + ms[10] -
             ms[11] - ms[12] - ms[15] - ms[16] - ms[18];
    fi[14] = ms[0] + R(8) * ms[1] + ms[2] - ms[3] - ms[4] - ms[7] - ms[8] + ms[9] + ms[10] -
             ms[11] - ms[12] + ms[15] + ms[16] - ms[18];
    fi[15] = ms[0] + R(8) * ms[1] + ms[2] + ms[5] + ms[6] + ms[7] + ms[8] - R(2) * ms[9] -
             R(2) * ms[10] + ms[14] + ms[17] - ms[18];
    fi[16] = ms[0] + R(8) * ms[1] + ms[2] - ms[5] - ms[6] + ms[7] + ms[8] - R(2) * ms[9] -
             R(2) * ms[10] - ms[14] - ms[17] - ms[18];
    fi[17] = ms[0] + R(8) * ms[1] + ms[2] + ms[5] + ms[6] - ms[7] - ms[8] - R(2) * ms[9] -
             R(2) * ms[10] - ms[14] + ms[17] + ms[18];
    fi[18] = ms[0] + R(8) * ms[1] + ms[2] - ms[5] - ms[6] - ms[7] - ms[8] - R(2) * ms[9] -
             R(2) * ms[10] + ms[14] - ms[17] + ms[18];
}

// Collision operators.  OP: 0 BGK, 1 regularized, 2 MRT.  `omega_tau`
// is 1/tau precomputed on the host (the same IEEE quotient) and used when
// SMAG is off.

template <typename R, int OP, bool SMAG>
__device__ __forceinline__ void collide(const R (&f)[19], R (&fn)[19], R rho, R ux, R uy,
                                        R uz, R tau, R omega_tau, R smagCs) {
    R fe[19];
    if (SMAG || OP != OP_MRT) {
#pragma unroll
        for (int i = 0; i < 19; i++) fe[i] = feq<R>(i, rho, ux, uy, uz);
    }
    R omega = omega_tau;
    if (SMAG) {
        // :448-484
        R Sxx = R(0), Syy = R(0), Szz = R(0), Sxy = R(0), Sxz = R(0), Syz = R(0);
#pragma unroll
        for (int i = 0; i < 19; i++) {
            R f_neq = f[i] - fe[i];
            R ex = R(cx(i)), ey = R(cy(i)), ez = R(cz(i));
            Sxx += ex * ex * f_neq;
            Syy += ey * ey * f_neq;
            Szz += ez * ez * f_neq;
            Sxy += ex * ey * f_neq;
            Sxz += ex * ez * f_neq;
            Syz += ey * ez * f_neq;
        }
        R Pi_norm = dsqrt<R>(Sxx * Sxx + Syy * Syy + Szz * Szz +
                             R(2) * (Sxy * Sxy + Sxz * Sxz + Syz * Syz));
        R Cs2 = smagCs * smagCs;
        R tau_eff = R(0.5) * (tau + dsqrt<R>(tau * tau + ddiv<R>(R(18) * Cs2 * Pi_norm,
                                                                  rho + R(1e-10))));
        omega = ddiv<R>(R(1), tau_eff);
    }
    if (OP == OP_REG) {
        // :488-543
        R Pxx = R(0), Pyy = R(0), Pzz = R(0), Pxy = R(0), Pxz = R(0), Pyz = R(0);
#pragma unroll
        for (int i = 0; i < 19; i++) {
            R f_neq = f[i] - fe[i];
            R ex = R(cx(i)), ey = R(cy(i)), ez = R(cz(i));
            Pxx += ex * ex * f_neq;
            Pyy += ey * ey * f_neq;
            Pzz += ez * ez * f_neq;
            Pxy += ex * ey * f_neq;
            Pxz += ex * ez * f_neq;
            Pyz += ey * ez * f_neq;
        }
        const R inv_2cs4 = R(4.5);
        const R cs2 = R(1) / R(3);
#pragma unroll
        for (int i = 0; i < 19; i++) {
            R ex = R(cx(i)), ey = R(cy(i)), ez = R(cz(i));
            R QP = (ex * ex - cs2) * Pxx + (ey * ey - cs2) * Pyy + (ez * ez - cs2) * Pzz +
                   R(2) * ex * ey * Pxy + R(2) * ex * ez * Pxz + R(2) * ey * ez * Pyz;
            R f_neq_reg = wgt<R>(i) * inv_2cs4 * QP;
            fn[i] = fe[i] + (R(1) - omega) * f_neq_reg;
        }
    } else if (OP == OP_MRT) {
        // :544-617
        R m[19], meq[19];
        mrt_forward<R>(f, m);
        R u2 = ux * ux + uy * uy + uz * uz;
        meq[0] = rho;
        meq[1] = R(-11) * rho + R(19) * rho * u2;
        meq[2] = R(3) * rho - R(5.5) * rho * u2;
        meq[3] = rho * ux;
        meq[4] = R(-2) / R(3) * rho * ux;
        meq[5] = rho * uy;
        meq[6] = R(-2) / R(3) * rho * uy;
        meq[7] = rho * uz;
        meq[8] = R(-2) / R(3) * rho * uz;
        meq[9] = rho * (R(2) * ux * ux - uy * uy - uz * uz);
        meq[10] = R(-0.5) * rho * (R(2) * ux * ux - uy * uy - uz * uz);
        meq[11] = rho * (uy * uy - uz * uz);
        meq[12] = R(-0.5) * rho * (uy * uy - uz * uz);
        meq[13] = rho * ux * uy;
        meq[14] = rho * uy * uz;
        meq[15] = rho * ux * uz;
        meq[16] = R(0);
        meq[17] = R(0);
        meq[18] = R(0);
        const R s_nu = omega;
        const R s[19] = {R(0),    R(1.19), R(1.4), R(0),  R(1.2), R(0),    R(1.2),
                         R(0),    R(1.2),  s_nu,   R(1.4), s_nu,  R(1.4),  s_nu,
                         s_nu,    s_nu,    R(1.98), R(1.98), R(1.98)};
#pragma unroll
        for (int k = 0; k < 19; k++) m[k] = m[k] - s[k] * (m[k] - meq[k]);
        mrt_inverse<R>(m, fn);
    } else {
        // :618-625
#pragma unroll
        for (int i = 0; i < 19; i++) fn[i] = f[i] - omega * (f[i] - fe[i]);
    }
}

}  // namespace lbm
