// The fused step with two neighbouring cells per thread and the collision of
// both evaluated by sm_100's paired single-precision instructions
// (add / sub / mul / fma .rn.f32x2): lane x of every pair is cell x0, lane y
// cell x0 + 1 (x0 even).  Each lane performs exactly the scalar rounding
// sequence of collide() in lbm_d3q19.cuh -- which is the shader's,
// lbm_collide.comp:313-626 -- so the results are bit-identical to the
// one-cell kernel, while the instruction stream per cell is much shorter.
//
// Two rules keep the pairing exact:
//  * every product whose result feeds an addition is issued as a paired fma
//    with a runtime (-0, -0) addend (PairTable::nz): fma(a, b, -0) rounds
//    a*b exactly once, and an fma cannot be contracted with the addition
//    that follows (a paired multiply can be: measured on sm_100, see
//    lbm_d3q19.cuh);
//  * a product by +-2, +-4 or +-8 is exact and is fused into its sum, as
//    the scalar code does.
// Division and square root stay scalar, once per lane, with the scalar
// code's IEEE operations.
//
// Memory: a warp covers 64 consecutive x of one row.  Directions with
// e_x == 0 load, and every direction stores, the two cells with one aligned
// 64-bit (FP32) or 32-bit (FP16 / BF16) access; the e_x != 0 directions
// load the two cells separately (the pair is shifted by one element).
// Addresses are 32-bit cell indices added to per-direction base pointers
// held in the kernel parameter (PairTable).
//
// Pairs that hold a solid body cell take the scalar per-cell code; Zou-He
// cells and guard resets stay on the paired path (per-lane rewrite before
// the moments, per-lane select after the collision).  Included by
// lbm_step.cuh after the per-cell pieces it uses.
#pragma once

#include "lbm_d3q19.cuh"
#include "lbm_internal.h"

namespace lbm {
namespace LBM_ARITH_NS {

using P = float2;

__device__ __forceinline__ P pc(float v) { return make_float2(v, v); }

// a * b rounded once, never fused with the sum it feeds (nz = (-0, -0))
__device__ __forceinline__ P pmulz(P a, P b, P nz) {
#ifdef LBM_FAST_ARITH
    (void)nz;
    return pmul(a, b);
#else
    return pfma(a, b, nz);
#endif
}

// x / y for a constant y, given ny = (-y, -y) and zh = RN(1 / y): the
// Markstein sequence of cdiv() on both lanes (r = fma(q1, -y, x) is the
// scalar fma(-q1, y, x))
__device__ __forceinline__ P pcdiv(P x, P ny, P zh) {
#ifdef LBM_FAST_ARITH
    (void)ny;
    return pmul(x, zh);
#else
    const P q1 = pmul(x, zh);
    const P r = pfma(q1, ny, x);
    return pfma(r, zh, q1);
#endif
}
__device__ __forceinline__ P pcdiv(P x, float y) { return pcdiv(x, pc(-y), pc(1.0f / y)); }

// Left-to-right signed sums of populations: psum<a, b, -c, d>(F) is
// ((F[a] + F[b]) - F[c]) + F[d]; pchain<...>(s, F) continues from s.
template <int I>
__device__ __forceinline__ P pacc(P acc, const P (&F)[19]) {
    if constexpr (I < 0)
        return psub(acc, F[-I]);
    else
        return padd(acc, F[I]);
}
template <int... Rest>
__device__ __forceinline__ P pchain(P acc, const P (&F)[19]) {
    ((acc = pacc<Rest>(acc, F)), ...);
    return acc;
}
template <int First, int... Rest>
__device__ __forceinline__ P psum(const P (&F)[19]) {
    static_assert(First >= 0, "a sum starts with a positive term");
    return pchain<Rest...>(F[First], F);
}

// ---------------------------------------------------------------------------
// Paired collision: the lane-wise image of collide() and its helpers
// ---------------------------------------------------------------------------
// rho and momenta (:411-424), each in index order (moments())
__device__ __forceinline__ void pmoments(const P (&F)[19], P &rho, P &jx, P &jy, P &jz) {
    rho = psum<0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18>(F);
    jx = psum<1, -2, 7, -8, 9, -10, 11, -12, 13, -14>(F);
    jy = psum<3, -4, 7, 8, -9, -10, 15, -16, 17, -18>(F);
    jz = psum<5, -6, 11, 12, -13, -14, 15, 16, -17, -18>(F);
}

// equilibria() on both lanes: fe_i = (w_i rho) (((1 +- a) + b) - cu)
__device__ __forceinline__ void pequilibria(P rho, P ux, P uy, P uz, P u2, P nz, P (&fe)[19]) {
    constexpr float cs2 = 1.0f / 3.0f;
    constexpr float c1 = 2.0f * cs2;
    constexpr float c2 = 2.0f * cs2 * cs2;
    const P ONE = pc(1.0f);
    const P cu = pcdiv(u2, c1);
    const P wr0 = pmulz(pc(wgt<float>(0)), rho, nz);
    const P wr1 = pmulz(pc(wgt<float>(1)), rho, nz);
    const P wr2 = pmulz(pc(wgt<float>(7)), rho, nz);
    fe[0] = pmulz(wr0, psub(ONE, cu), nz);
    auto pair = [&](P e, P wr, P &fi, P &fj) {
        const P a = pcdiv(e, cs2);
        const P b = pcdiv(pmul(e, e), c2);
        fi = pmulz(wr, psub(padd(padd(ONE, a), b), cu), nz);
        fj = pmulz(wr, psub(padd(psub(ONE, a), b), cu), nz);
    };
    pair(ux, wr1, fe[1], fe[2]);
    pair(uy, wr1, fe[3], fe[4]);
    pair(uz, wr1, fe[5], fe[6]);
    pair(padd(ux, uy), wr2, fe[7], fe[10]);
    pair(psub(uy, ux), wr2, fe[8], fe[9]);
    pair(padd(ux, uz), wr2, fe[11], fe[14]);
    pair(psub(uz, ux), wr2, fe[12], fe[13]);
    pair(padd(uy, uz), wr2, fe[15], fe[18]);
    pair(psub(uz, uy), wr2, fe[16], fe[17]);
}

// stress(): Pi_ab = sum_i e_ia e_ib (f_i - feq_i), nonzero terms in index order
__device__ __forceinline__ void pstress(const P (&F)[19], const P (&fe)[19], P &Pxx, P &Pyy,
                                        P &Pzz, P &Pxy, P &Pxz, P &Pyz) {
    P n[19];
#pragma unroll
    for (int i = 0; i < 19; i++) n[i] = psub(F[i], fe[i]);
    Pxx = psum<1, 2, 7, 8, 9, 10, 11, 12, 13, 14>(n);
    Pyy = psum<3, 4, 7, 8, 9, 10, 15, 16, 17, 18>(n);
    Pzz = psum<5, 6, 11, 12, 13, 14, 15, 16, 17, 18>(n);
    Pxy = psum<7, -8, -9, 10>(n);
    Pxz = psum<11, -12, -13, 14>(n);
    Pyz = psum<15, -16, -17, 18>(n);
}

// The non-equilibrium stress of both lanes with the equilibria streamed in
// (for MRT + Smagorinsky, which needs feq only here): every f_i - feq_i is
// formed in index order and added at once to each sum it belongs to, so each
// sum receives its terms in the order stress() adds them and no array of
// equilibria stays live.  feq_i is evaluated as in pequilibria; f_i is
// get(i).
template <class Get>
__device__ __forceinline__ void pstress_streamed(Get get, P rho, P ux, P uy, P uz, P u2, P nz,
                                                 P &Pxx, P &Pyy, P &Pzz, P &Pxy, P &Pxz, P &Pyz) {
    constexpr float cs2 = 1.0f / 3.0f;
    constexpr float c1 = 2.0f * cs2;
    constexpr float c2 = 2.0f * cs2 * cs2;
    const P ONE = pc(1.0f);
    const P cu = pcdiv(u2, c1);
    const P wr1 = pmulz(pc(wgt<float>(1)), rho, nz);
    const P wr2 = pmulz(pc(wgt<float>(7)), rho, nz);
    // the quotients e/cs2 and e^2/(2 cs2^2) of one direction pair
    struct Q {
        P a, b;
    };
    auto quot = [&](P e) { return Q{pcdiv(e, cs2), pcdiv(pmul(e, e), c2)}; };
    auto nplus = [&](int i, P wr, Q q) {
        return psub(get(i), pmulz(wr, psub(padd(padd(ONE, q.a), q.b), cu), nz));
    };
    auto nminus = [&](int i, P wr, Q q) {
        return psub(get(i), pmulz(wr, psub(padd(psub(ONE, q.a), q.b), cu), nz));
    };
    P n;
    Q q = quot(ux);
    Pxx = padd(nplus(1, wr1, q), nminus(2, wr1, q));
    q = quot(uy);
    Pyy = padd(nplus(3, wr1, q), nminus(4, wr1, q));
    q = quot(uz);
    Pzz = padd(nplus(5, wr1, q), nminus(6, wr1, q));
    Q qa = quot(padd(ux, uy)), qb = quot(psub(uy, ux));
    n = nplus(7, wr2, qa);
    Pxx = padd(Pxx, n), Pyy = padd(Pyy, n), Pxy = n;
    n = nplus(8, wr2, qb);
    Pxx = padd(Pxx, n), Pyy = padd(Pyy, n), Pxy = psub(Pxy, n);
    n = nminus(9, wr2, qb);
    Pxx = padd(Pxx, n), Pyy = padd(Pyy, n), Pxy = psub(Pxy, n);
    n = nminus(10, wr2, qa);
    Pxx = padd(Pxx, n), Pyy = padd(Pyy, n), Pxy = padd(Pxy, n);
    qa = quot(padd(ux, uz)), qb = quot(psub(uz, ux));
    n = nplus(11, wr2, qa);
    Pxx = padd(Pxx, n), Pzz = padd(Pzz, n), Pxz = n;
    n = nplus(12, wr2, qb);
    Pxx = padd(Pxx, n), Pzz = padd(Pzz, n), Pxz = psub(Pxz, n);
    n = nminus(13, wr2, qb);
    Pxx = padd(Pxx, n), Pzz = padd(Pzz, n), Pxz = psub(Pxz, n);
    n = nminus(14, wr2, qa);
    Pxx = padd(Pxx, n), Pzz = padd(Pzz, n), Pxz = padd(Pxz, n);
    qa = quot(padd(uy, uz)), qb = quot(psub(uz, uy));
    n = nplus(15, wr2, qa);
    Pyy = padd(Pyy, n), Pzz = padd(Pzz, n), Pyz = n;
    n = nplus(16, wr2, qb);
    Pyy = padd(Pyy, n), Pzz = padd(Pzz, n), Pyz = psub(Pyz, n);
    n = nminus(17, wr2, qb);
    Pyy = padd(Pyy, n), Pzz = padd(Pzz, n), Pyz = psub(Pyz, n);
    n = nminus(18, wr2, qa);
    Pyy = padd(Pyy, n), Pzz = padd(Pzz, n), Pyz = padd(Pyz, n);
}

// mrt_forward() on both lanes (lbm_collide.comp:110-181)
__device__ __forceinline__ void pmrt_forward(const P (&F)[19], P nz, P (&m)[19]) {
    const P sf = psum<1, 2, 3, 4, 5, 6>(F);
    const P se = psum<7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18>(F);
    m[0] = padd(padd(F[0], sf), se);
    m[1] = pfma(pc(8.0f), se, psub(pmulz(pc(-30.0f), F[0], nz), pmulz(pc(11.0f), sf, nz)));
    m[2] = padd(pfma(pc(-4.0f), sf, pmulz(pc(12.0f), F[0], nz)), se);
    const P d12 = psub(F[1], F[2]), d34 = psub(F[3], F[4]), d56 = psub(F[5], F[6]);
    m[3] = pchain<7, -8, 9, -10, 11, -12, 13, -14>(d12, F);
    m[4] = pchain<-8, 9, -10, 11, -12, 13, -14>(pfma(pc(-4.0f), d12, F[7]), F);
    m[5] = pchain<7, 8, -9, -10, 15, -16, 17, -18>(d34, F);
    m[6] = pchain<8, -9, -10, 15, -16, 17, -18>(pfma(pc(-4.0f), d34, F[7]), F);
    m[7] = pchain<11, 12, -13, -14, 15, 16, -17, -18>(d56, F);
    m[8] = pchain<12, -13, -14, 15, 16, -17, -18>(pfma(pc(-4.0f), d56, F[11]), F);
    const P sXY = psum<7, 8, 9, 10>(F);
    const P sXZ = psum<11, 12, 13, 14>(F);
    const P sYZ = psum<15, 16, 17, 18>(F);
    const P s12 = padd(F[1], F[2]), s34 = padd(F[3], F[4]), s56 = padd(F[5], F[6]);
    m[9] = pfma(pc(-2.0f), sYZ,
                padd(padd(psub(pfma(pc(2.0f), s12, pneg(s34)), s56), sXY), sXZ));
    m[10] = pfma(pc(-2.0f), sYZ,
                 padd(padd(pfma(pc(2.0f), s56, pfma(pc(2.0f), s34, pmul(pc(-4.0f), s12))), sXY),
                      sXZ));
    m[11] = psub(padd(psub(s34, s56), sXY), sXZ);
    m[12] = psub(padd(pfma(pc(2.0f), s56, pmul(pc(-2.0f), s34)), sXY), sXZ);
    m[13] = psum<7, -8, -9, 10>(F);
    m[14] = psum<15, -16, -17, 18>(F);
    m[15] = psum<11, -12, -13, 14>(F);
    m[16] = psum<7, -8, 9, -10, -11, 12, -13, 14>(F);
    m[17] = pchain<-8, 9, 10, 15, -16, 17, -18>(pneg(F[7]), F);
    m[18] = psum<11, 12, -13, -14, -15, -16, 17, 18>(F);
}

// mrt_inverse() on both lanes in the reference's order (lbm_collide.comp:
// 185-311): moments scaled by their constant norms, then per population a
// left-to-right sum, products by 2, 4, 8 fused
__device__ __forceinline__ void pmrt_inverse(const P (&m)[19], P nz, P (&fi)[19]) {
    P ms[19];
    ms[0] = pcdiv(m[0], 19.0f);
    ms[1] = pcdiv(m[1], 2394.0f);
    ms[2] = pcdiv(m[2], 252.0f);
    ms[3] = pcdiv(m[3], 10.0f);
    ms[4] = pcdiv(m[4], 40.0f);
    ms[5] = pcdiv(m[5], 10.0f);
    ms[6] = pcdiv(m[6], 40.0f);
    ms[7] = pcdiv(m[7], 10.0f);
    ms[8] = pcdiv(m[8], 40.0f);
    ms[9] = pcdiv(m[9], 36.0f);
    ms[10] = pcdiv(m[10], 72.0f);
    ms[11] = pcdiv(m[11], 12.0f);
    ms[12] = pcdiv(m[12], 24.0f);
    ms[13] = pmul(m[13], pc(0.25f));  // division by a power of two is exact
    ms[14] = pmul(m[14], pc(0.25f));
    ms[15] = pmul(m[15], pc(0.25f));
    ms[16] = pmul(m[16], pc(0.125f));
    ms[17] = pmul(m[17], pc(0.125f));
    ms[18] = pmul(m[18], pc(0.125f));

    const P C2 = pc(2.0f), C4 = pc(4.0f), CM2 = pc(-2.0f), CM4 = pc(-4.0f);
    fi[0] = padd(psub(ms[0], pmulz(pc(30.0f), ms[1], nz)), pmulz(pc(12.0f), ms[2], nz));
    const P a0 = pfma(CM4, ms[2], psub(ms[0], pmulz(pc(11.0f), ms[1], nz)));
    fi[1] = pfma(CM4, ms[10], pfma(C2, ms[9], pfma(CM4, ms[4], padd(a0, ms[3]))));
    fi[2] = pfma(CM4, ms[10], pfma(C2, ms[9], pfma(C4, ms[4], psub(a0, ms[3]))));
    fi[3] = pfma(CM2, ms[12], padd(pfma(C2, ms[10], psub(pfma(CM4, ms[6], padd(a0, ms[5])), ms[9])),
                                   ms[11]));
    fi[4] = pfma(CM2, ms[12], padd(pfma(C2, ms[10], psub(pfma(C4, ms[6], psub(a0, ms[5])), ms[9])),
                                   ms[11]));
    fi[5] = pfma(C2, ms[12], psub(pfma(C2, ms[10], psub(pfma(CM4, ms[8], padd(a0, ms[7])), ms[9])),
                                  ms[11]));
    fi[6] = pfma(C2, ms[12], psub(pfma(C2, ms[10], psub(pfma(C4, ms[8], psub(a0, ms[7])), ms[9])),
                                  ms[11]));
    const P b0 = padd(pfma(pc(8.0f), ms[1], ms[0]), ms[2]);
    fi[7] = pchain<3, 4, 5, 6, 9, 10, 11, 12, 13, 16, -17>(b0, ms);
    fi[8] = pchain<-3, -4, 5, 6, 9, 10, 11, 12, -13, -16, -17>(b0, ms);
    fi[9] = pchain<3, 4, -5, -6, 9, 10, 11, 12, -13, 16, 17>(b0, ms);
    fi[10] = pchain<-3, -4, -5, -6, 9, 10, 11, 12, 13, -16, 17>(b0, ms);
    fi[11] = pchain<3, 4, 7, 8, 9, 10, -11, -12, 15, -16, 18>(b0, ms);
    fi[12] = pchain<-3, -4, 7, 8, 9, 10, -11, -12, -15, 16, 18>(b0, ms);
    fi[13] = pchain<3, 4, -7, -8, 9, 10, -11, -12, -15, -16, -18>(b0, ms);
    fi[14] = pchain<-3, -4, -7, -8, 9, 10, -11, -12, 15, 16, -18>(b0, ms);
    fi[15] = pchain<14, 17, -18>(pfma(CM2, ms[10], pfma(CM2, ms[9], pchain<5, 6, 7, 8>(b0, ms))), ms);
    fi[16] = pchain<-14, -17, -18>(pfma(CM2, ms[10], pfma(CM2, ms[9], pchain<-5, -6, 7, 8>(b0, ms))),
                                   ms);
    fi[17] = pchain<-14, 17, 18>(pfma(CM2, ms[10], pfma(CM2, ms[9], pchain<5, 6, -7, -8>(b0, ms))),
                                 ms);
    fi[18] = pchain<14, -17, 18>(pfma(CM2, ms[10], pfma(CM2, ms[9], pchain<-5, -6, -7, -8>(b0, ms))),
                                 ms);
}

// MRT relaxation (:559-610) of the moments m and the inverse transform into
// fn: meq from rho and u, m - s (m - meq) with s_nu = omega on the stress
// moments, the conserved moments kept, the ghost moments relaxed to 0.
__device__ __forceinline__ void pmrt_relax_inverse(P (&m)[19], P rho, P ux, P uy, P uz, P u2,
                                                   P omega, P nz, P (&fn)[19]) {
    P meq[19];
    const P uyy = pmulz(uy, uy, nz), uzz = pmulz(uz, uz, nz);
    const P pxx = psub(psub(pmulz(pmul(pc(2.0f), ux), ux, nz), uyy), uzz);
    const P pww = psub(uyy, uzz);
    meq[1] = padd(pmulz(pc(-11.0f), rho, nz), pmulz(pmulz(pc(19.0f), rho, nz), u2, nz));
    meq[2] = psub(pmulz(pc(3.0f), rho, nz), pmulz(pmulz(pc(5.5f), rho, nz), u2, nz));
    const P r23 = pmulz(pc(-2.0f / 3.0f), rho, nz);
    meq[4] = pmulz(r23, ux, nz);
    meq[6] = pmulz(r23, uy, nz);
    meq[8] = pmulz(r23, uz, nz);
    const P rh = pmulz(pc(-0.5f), rho, nz);
    meq[9] = pmulz(rho, pxx, nz);
    meq[10] = pmulz(rh, pxx, nz);
    meq[11] = pmulz(rho, pww, nz);
    meq[12] = pmulz(rh, pww, nz);
    const P rux = pmulz(rho, ux, nz);
    meq[13] = pmulz(rux, uy, nz);
    meq[14] = pmulz(pmulz(rho, uy, nz), uz, nz);
    meq[15] = pmulz(rux, uz, nz);
    auto relax = [&](int k, P s) { m[k] = psub(m[k], pmulz(s, psub(m[k], meq[k]), nz)); };
    relax(1, pc(1.19f));
    relax(2, pc(1.4f));
    relax(4, pc(1.2f));
    relax(6, pc(1.2f));
    relax(8, pc(1.2f));
    relax(9, omega);
    relax(10, pc(1.4f));
    relax(11, omega);
    relax(12, pc(1.4f));
    relax(13, omega);
    relax(14, omega);
    relax(15, omega);
    m[16] = psub(m[16], pmulz(pc(1.98f), m[16], nz));
    m[17] = psub(m[17], pmulz(pc(1.98f), m[17], nz));
    m[18] = psub(m[18], pmulz(pc(1.98f), m[18], nz));
    pmrt_inverse(m, nz, fn);
}

// Smagorinsky omega per lane (:472-484) from the non-equilibrium stress:
// the Frobenius norm paired, square roots and divisions per lane
__device__ __forceinline__ P psmag_omega(P Pxx, P Pyy, P Pzz, P Pxy, P Pxz, P Pyz, P rho,
                                         float tau, float smag18, P nz) {
    const P A = padd(padd(pmulz(Pxx, Pxx, nz), pmulz(Pyy, Pyy, nz)), pmulz(Pzz, Pzz, nz));
    const P B = padd(padd(pmulz(Pxy, Pxy, nz), pmulz(Pxz, Pxz, nz)), pmulz(Pyz, Pyz, nz));
    const P N2 = pfma(pc(2.0f), B, A);
    const float tt = tau * tau;
    auto lane = [&](float n2, float r) {
        const float pin = dsqrt<float>(n2);
        const float te = 0.5f * (tau + dsqrt<float>(tt + ddiv<float>(smag18 * pin, r + 1e-10f)));
        return ddiv<float>(1.0f, te);
    };
    return make_float2(lane(N2.x, rho.x), lane(N2.y, rho.y));
}

// collide() on both lanes; rho, u and u2 are the lanes' moments (u2 =
// (ux ux + uy uy) + uz uz), omega_tau the lanes' 1/tau when SMAG is off.
template <int OP, bool SMAG>
__device__ __forceinline__ void pcollide(const P (&F)[19], P (&fn)[19], P rho, P ux, P uy, P uz,
                                         P u2, float tau, float omega_tau, float smag18, P nz) {
    P fe[19];
    P omega = pc(omega_tau);
    P Pxx, Pyy, Pzz, Pxy, Pxz, Pyz;
    if (OP == OP_MRT) {
        // MRT needs the equilibria only for the Smagorinsky stress
        if (SMAG)
            pstress_streamed([&](int i) { return F[i]; }, rho, ux, uy, uz, u2, nz, Pxx, Pyy, Pzz,
                             Pxy, Pxz, Pyz);
    } else {
        pequilibria(rho, ux, uy, uz, u2, nz, fe);
        if (SMAG || OP == OP_REG) pstress(F, fe, Pxx, Pyy, Pzz, Pxy, Pxz, Pyz);
    }
    if (SMAG) omega = psmag_omega(Pxx, Pyy, Pzz, Pxy, Pxz, Pyz, rho, tau, smag18, nz);
    if (OP == OP_REG) {
        // :517-543
        constexpr float cs2 = 1.0f / 3.0f;
        const P K1 = pc(1.0f - cs2), K0 = pc(0.0f - cs2);
        const P om = psub(pc(1.0f), omega);
        const P k0x = pmulz(K0, Pxx, nz), k0y = pmulz(K0, Pyy, nz), k0z = pmulz(K0, Pzz, nz);
        const P k1x = pmulz(K1, Pxx, nz), k1y = pmulz(K1, Pyy, nz), k1z = pmulz(K1, Pzz, nz);
        const P Q0 = padd(padd(k0x, k0y), k0z);
        const P Qx = padd(padd(k1x, k0y), k0z);
        const P Qy = padd(padd(k0x, k1y), k0z);
        const P Qz = padd(padd(k0x, k0y), k1z);
        const P Txy = padd(padd(k1x, k1y), k0z);
        const P Txz = padd(padd(k1x, k0y), k1z);
        const P Tyz = padd(padd(k0x, k1y), k1z);
        P Q[19];
        Q[0] = Q0;
        Q[1] = Q[2] = Qx;
        Q[3] = Q[4] = Qy;
        Q[5] = Q[6] = Qz;
        Q[7] = Q[10] = pfma(pc(2.0f), Pxy, Txy);
        Q[8] = Q[9] = pfma(pc(-2.0f), Pxy, Txy);
        Q[11] = Q[14] = pfma(pc(2.0f), Pxz, Txz);
        Q[12] = Q[13] = pfma(pc(-2.0f), Pxz, Txz);
        Q[15] = Q[18] = pfma(pc(2.0f), Pyz, Tyz);
        Q[16] = Q[17] = pfma(pc(-2.0f), Pyz, Tyz);
#pragma unroll
        for (int i = 0; i < 19; i++)
            fn[i] = padd(fe[i], pmulz(om, pmulz(pc(wgt<float>(i) * 4.5f), Q[i], nz), nz));
    } else if (OP == OP_MRT) {
        // :550-616
        P m[19];
        pmrt_forward(F, nz, m);
        pmrt_relax_inverse(m, rho, ux, uy, uz, u2, omega, nz, fn);
    } else {
        // :618-625
#pragma unroll
        for (int i = 0; i < 19; i++) fn[i] = psub(F[i], pmulz(omega, psub(F[i], fe[i]), nz));
    }
}

// u /= rho when rho > 1e-4 (IEEE division per lane), u2, and the stability
// guard (:421-430) per lane
__device__ __forceinline__ void pvelocity_guard(P rho, P &ux, P &uy, P &uz, P &u2, P nz,
                                                bool &resetA, bool &resetB) {
    if (rho.x > 0.0001f) {
        ux.x = ddiv<float>(ux.x, rho.x);
        uy.x = ddiv<float>(uy.x, rho.x);
        uz.x = ddiv<float>(uz.x, rho.x);
    }
    if (rho.y > 0.0001f) {
        ux.y = ddiv<float>(ux.y, rho.y);
        uy.y = ddiv<float>(uy.y, rho.y);
        uz.y = ddiv<float>(uz.y, rho.y);
    }
    u2 = padd(padd(pmulz(ux, ux, nz), pmulz(uy, uy, nz)), pmulz(uz, uz, nz));
    auto guard = [](float r, float v2) {
        return r < 0.3f || r > 2.0f || speed_exceeds(v2) || isinf(r) || isnan(r);
    };
    resetA = guard(rho.x, u2.x);
    resetB = guard(rho.y, u2.y);
}

// The collision of a pair of fluid (or ground) cells after the stream:
// Zou-He on lane x (inlet plane) or lane y (outlet plane), the moments, the
// per-lane division and stability guard, the paired operator, and feq(1, 0)
// = w_i on a lane the guard resets (prepare_cell() + collide() per lane).
template <int OP, bool SMAG>
__device__ __forceinline__ void pair_collide_fluid(float (&fa)[19], float (&fb)[19], bool inletA,
                                                   bool outletB, float inX, float inY, float inZ,
                                                   float tau, float omega, float smag18, P nz,
                                                   P (&fn)[19], bool &resetA, bool &resetB) {
    // Zou-He (:336-408) on the lane that sits on the inlet / outlet plane
    if (inletA) zou_he_inlet<float>(fa, inX, inY, inZ);
    if (outletB) zou_he_outlet<float>(fb);
    P F[19];
#pragma unroll
    for (int i = 0; i < 19; i++) F[i] = make_float2(fa[i], fb[i]);
    P rho, ux, uy, uz, u2;
    pmoments(F, rho, ux, uy, uz);
    pvelocity_guard(rho, ux, uy, uz, u2, nz, resetA, resetB);
    pcollide<OP, SMAG>(F, fn, rho, ux, uy, uz, u2, tau, omega, smag18, nz);
#pragma unroll
    for (int i = 0; i < 19; i++) {
        if (resetA) fn[i].x = wgt<float>(i);
        if (resetB) fn[i].y = wgt<float>(i);
    }
}

// ---------------------------------------------------------------------------
// The kernels
// ---------------------------------------------------------------------------
constexpr int PAIR_THREADS = 128;  // threads per block (two cells each)
// Blocks resident per SM the paired kernels are compiled for (register cap
// 65536 / (PAIR_THREADS * blocks)), measured on B200 at 256x128x128: 7 (72
// registers) for the operators without Smagorinsky (FP32 BGK 41.0k, FP16
// BGK 53.1k MLUPS against 41.0k / 48.7k at 6), 6 (80 registers) with it (MRT
// + Smagorinsky 31.8k against 30.7k at 5 and 31.6k at 7; regularized +
// Smagorinsky 37.3k against 34.8k at 5).  LBM_PAIR_MINB overrides all of them
// (measurements).
template <int OP, bool SMAG>
__host__ __device__ constexpr int pair_minb() {
#ifdef LBM_PAIR_MINB
    return LBM_PAIR_MINB;
#else
    return SMAG ? 6 : 7;
#endif
}
// Batched launches of one operator take that operator's cap; a launch that
// switches between operators at run time holds the largest of them and is
// capped at 96 registers (5 blocks per SM).  LBM_PAIR_MINB_BATCH overrides
// (measurements).
__host__ __device__ constexpr int pair_minb_set(int set) {
#ifdef LBM_PAIR_MINB_BATCH
    return (void)set, LBM_PAIR_MINB_BATCH;
#else
    return set == BATCH_SET_BGK || set == BATCH_SET_REG || set == BATCH_SET_MRT ? 7
           : set < BATCH_SET_BGK_REG                                          ? 6
                                                                               : 5;
#endif
}

// Where the scalar fallback parks the second cell of a pair (one array per
// kernel, whichever operators the kernel instantiates).
__shared__ float pair_park[19 * PAIR_THREADS];

// Where a pair's populations come from and go to.  TabParam reads the
// per-direction pointers precomputed in a kernel parameter (constant-bank
// operands, no registers); TabCalc computes them from the two buffers'
// bases and the grid's extents, holding a few scalars instead of 57
// pointers -- for kernels whose grid is chosen at run time.
struct TabParam {
    const PairTable &t;
    __device__ __forceinline__ const void *pull(int i) const { return t.pull[i]; }
    __device__ __forceinline__ const void *own(int i) const { return t.own[i]; }
    __device__ __forceinline__ void *dst(int i) const { return t.dst[i]; }
    __device__ __forceinline__ float2 nz() const { return t.nz; }
};

template <class T>
struct TabCalc {
    const T *src;
    T *dstb;
    int n, nx, plane;
    float2 z;
    __device__ __forceinline__ const void *own(int i) const { return src + (long long)i * n; }
    __device__ __forceinline__ const void *pull(int i) const {
        return src + ((long long)i * n - cx(i) - cy(i) * nx - cz(i) * plane);
    }
    __device__ __forceinline__ void *dst(int i) const { return dstb + (long long)i * n; }
    __device__ __forceinline__ float2 nz() const { return z; }
};

template <class S>
__device__ __forceinline__ void pair_load(const void *base, unsigned cell, int i, float &a,
                                          float &b, bool aligned) {
    const typename S::T *p = static_cast<const typename S::T *>(base) + cell;
    if (aligned) {
        S::load2(p, i, a, b);
    } else {
        a = S::load(p, i);
        b = S::load(p + 1, i);
    }
}

// The pull of one pair in an interior row (y and z away from the grid
// faces) at warp-uniform offsets.  The inlet / outlet pairs of the row take
// the reference's x-edge rule by a per-lane pointer select: a cell whose
// source x lies outside the grid keeps its own value (lbm_stream.comp:
// 116-127).  Calls copy(i, lane-x source, lane-y source, aligned pair).
template <class S, class Tab, class Copy>
__device__ __forceinline__ void pair_pull_interior(const StepArgs &a, const Tab &t, int x0,
                                                   unsigned cell0, Copy copy) {
    using T = typename S::T;
    const bool edgeA = x0 == 0, edgeB = x0 + 2 == a.nx;
#pragma unroll
    for (int i = 0; i < 19; i++) {
        const T *pull = static_cast<const T *>(t.pull(i)) + cell0;
        if (cx(i) == 0) {
            copy(i, pull, pull + 1, true);
        } else {
            const T *own = static_cast<const T *>(t.own(i)) + cell0;
            const bool keepA = cx(i) == 1 && edgeA, keepB = cx(i) == -1 && edgeB;
            copy(i, keepA ? own : pull, keepB ? own + 1 : pull + 1, false);
        }
    }
}

// The populations of one pair before Bouzidi: FUSED, the pull (interior
// row or, on a y / z face row, the wrap / clamp rules of gather_pull);
// otherwise the buffer's own values (the first step after initialisation).
template <class S, bool FUSED, class Tab>
__device__ __forceinline__ void pair_gather(const StepArgs &a, const Tab &t, int x0, int y,
                                            int z, unsigned cell0, float (&fa)[19],
                                            float (&fb)[19]) {
    using T = typename S::T;
    if (FUSED) {
        // a warp covers one row, so this test is uniform across the warp
        if (y > 0 && y + 1 < a.ny && z > 0 && z + 1 < a.nz) {
            pair_pull_interior<S>(a, t, x0, cell0, [&](int i, const T *pa, const T *pb, bool al) {
                if (al) {
                    S::load2(pa, i, fa[i], fb[i]);
                } else {
                    fa[i] = S::load(pa, i);
                    fb[i] = S::load(pb, i);
                }
            });
        } else {
            const Rows rw = neighbour_rows(a, y, z);
            const T *src = static_cast<const T *>(a.src);
            gather_pull<S>(a, src, x0, rw, (long long)cell0, fa);
            gather_pull<S>(a, src, x0 + 1, rw, (long long)cell0 + 1, fb);
        }
    } else {
#pragma unroll
        for (int i = 0; i < 19; i++) pair_load<S>(t.own(i), cell0, i, fa[i], fb[i], true);
    }
}

// Bouzidi on the pair's link-owning cells (FUSED), the collision and the
// store of one pair; returns the pair's guard resets.
template <class S, int OP, bool SMAG, bool FUSED, class Tab>
__device__ __forceinline__ int pair_finish(const StepArgs &a, const Tab &t, int x0, int y,
                                           int z, unsigned cell0, uint8_t flagA, uint8_t flagB,
                                           float (&fa)[19], float (&fb)[19]) {
    using T = typename S::T;
    if (FUSED && ((flagA | flagB) & FLAG_BOUNDARY)) {
        const Rows rw = neighbour_rows(a, y, z);
        const T *src = static_cast<const T *>(a.src);
        if (flagA & FLAG_BOUNDARY) bouzidi<S>(a, src, x0, rw, (long long)cell0, fa);
        if (flagB & FLAG_BOUNDARY) bouzidi<S>(a, src, x0 + 1, rw, (long long)cell0 + 1, fb);
    }
    int resets = 0;
    const int solidA = flagA & FLAG_SOLID_MASK, solidB = flagB & FLAG_SOLID_MASK;
    if (solidA == 1 || solidB == 1) {
        // A body cell in the pair: the scalar per-cell code for both cells,
        // one after the other (one code instance).  The second cell's
        // populations wait in shared memory meanwhile (stride PAIR_THREADS:
        // conflict-free), so this rare path does not raise the kernel's
        // register demand.
        float *park = pair_park;
        const int slot = threadIdx.x + blockDim.x * threadIdx.y;
#pragma unroll
        for (int i = 0; i < 19; i++) park[i * PAIR_THREADS + slot] = fb[i];
#pragma unroll 1
        for (int c = 0; c < 2; c++) {
            if (c == 1) {
#pragma unroll
                for (int i = 0; i < 19; i++) fa[i] = park[i * PAIR_THREADS + slot];
            }
            float fn[19];
            const int kind = collide_cell<S, OP, SMAG>(a, fa, fn, x0 + c, c ? flagB : flagA);
            resets += kind == 2;
#pragma unroll
            for (int i = 0; i < 19; i++)
                S::store(static_cast<T *>(t.dst(i)) + cell0 + c, fn[i], i);
        }
    } else {
        P fn[19];
        bool resetA, resetB;
        pair_collide_fluid<OP, SMAG>(fa, fb, x0 == 0, x0 + 1 == a.nx - 1, a.inX, a.inY, a.inZ,
                                     a.tau, a.omega, a.smag18, t.nz(), fn, resetA, resetB);
        resets = (int)resetA + (int)resetB;
#pragma unroll
        for (int i = 0; i < 19; i++)
            S::store2(static_cast<T *>(t.dst(i)) + cell0, fn[i].x, fn[i].y, i);
    }
    return resets;
}

// guard resets of the warp added to the grid's counter (one atomic)
__device__ __forceinline__ void pair_count_resets(const StepArgs &a, int resets) {
    const unsigned active = __activemask();
    const unsigned any = __ballot_sync(active, resets > 0);
    if (any) {
        int v = resets;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(active, v, o);
        const unsigned lane = (threadIdx.x + blockDim.x * threadIdx.y) & 31u;
        if (lane == (unsigned)(__ffs(active) - 1) && v) atomicAdd(a.guard, (unsigned long long)v);
    }
}

// One thread: the cells (x0, y, z) and (x0 + 1, y, z), x0 even.  FUSED:
// pull-stream (+ Bouzidi) then collide; otherwise collide the buffer's own
// values (the first step after initialisation).
template <class S, int OP, bool SMAG, bool FUSED, class Tab>
__device__ __forceinline__ void step_pair(const StepArgs &a, const Tab &t, int x0, int y, int z) {
    if (x0 >= a.nx || y >= a.ny) return;
    const unsigned cell0 = (unsigned)x0 + (unsigned)a.nx * ((unsigned)y + (unsigned)a.ny * z);
    const uchar2 fl = *reinterpret_cast<const uchar2 *>(a.flags + cell0);
    float fa[19], fb[19];
    pair_gather<S, FUSED>(a, t, x0, y, z, cell0, fa, fb);
    const int resets = pair_finish<S, OP, SMAG, FUSED>(a, t, x0, y, z, cell0, fl.x, fl.y, fa, fb);
    pair_count_resets(a, resets);
}

// Blocks of PAIR_THREADS threads, blockDim.x along x (two cells each) and
// blockDim.y rows.
template <class S, int OP, bool SMAG, bool FUSED>
__global__ void __launch_bounds__(PAIR_THREADS, pair_minb<OP, SMAG>())
    k_step_pair(const StepArgs a, const __grid_constant__ PairTable t) {
    step_pair<S, OP, SMAG, FUSED>(a, TabParam{t}, 2 * (blockIdx.x * blockDim.x + threadIdx.x),
                                  blockIdx.y * blockDim.y + threadIdx.y, blockIdx.z);
}

// Batched paired step: one launch advances up to BATCH_LAUNCH_MAX grids by
// one fused step.  Work unit: one tile of one z-plane of one grid, one
// PAIR_THREADS block per unit; the block finds its grid by binary search over
// the unit offsets and copies that grid's entry (step arguments, operator,
// tile shape; 160 bytes) from the device table into shared memory, so
// nothing is indexed at run time in the parameter space; the per-direction
// pointers are computed from the buffers' bases (TabCalc) rather than read
// from a table, which would hold 57 pointers in registers.  The per-cell
// code is k_step_pair's, so every grid's result is bit-identical to a solo
// step.  (Blocks that walk several units to share the set-up were measured
// slower: the loop raised the spills.)
template <class S, int SET>
__global__ void __launch_bounds__(PAIR_THREADS, pair_minb_set(SET))
    k_step_batch_pair(const __grid_constant__ BatchPairParams p) {
    __shared__ BatchGridDev g;
    const unsigned b = blockIdx.x;
    int lo = 0, hi = p.count - 1;  // largest grid index with starts <= b
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (p.starts[mid] <= b) lo = mid; else hi = mid - 1;
    }
    {
        static_assert(sizeof(BatchGridDev) % 16 == 0, "entry copied in 16-byte words");
        const uint4 *src = reinterpret_cast<const uint4 *>(p.grids + lo);
        uint4 *dst = reinterpret_cast<uint4 *>(&g);
        for (int k = threadIdx.x; k < (int)(sizeof(BatchGridDev) / 16); k += PAIR_THREADS)
            dst[k] = __ldg(src + k);
    }
    __syncthreads();
    const unsigned local = b - p.starts[lo];
    const unsigned tx = local % (unsigned)g.tiles_x;
    const unsigned rest = local / (unsigned)g.tiles_x;
    const int ty = (int)(rest % (unsigned)g.tiles_y);
    const int z = (int)(rest / (unsigned)g.tiles_y);
    const int bxt = 1 << g.lbx;
    const int x0 = 2 * ((int)tx * bxt + (int)(threadIdx.x & (bxt - 1)));
    const int y = ty * (PAIR_THREADS >> g.lbx) + (int)(threadIdx.x >> g.lbx);
    using T = typename S::T;
    const TabCalc<T> t{static_cast<const T *>(g.a.src), static_cast<T *>(g.a.dst), (int)g.a.n,
                       g.a.nx, g.a.nx * g.a.ny, g.nz};
    constexpr unsigned M = batch_set_mask(SET);
    switch (g.combo) {
        case 0: if constexpr ((M & 1u) != 0) step_pair<S, OP_BGK, false, true>(g.a, t, x0, y, z); break;
        case 1: if constexpr ((M & 2u) != 0) step_pair<S, OP_BGK, true, true>(g.a, t, x0, y, z); break;
        case 2: if constexpr ((M & 4u) != 0) step_pair<S, OP_REG, false, true>(g.a, t, x0, y, z); break;
        case 3: if constexpr ((M & 8u) != 0) step_pair<S, OP_REG, true, true>(g.a, t, x0, y, z); break;
        case 4: if constexpr ((M & 16u) != 0) step_pair<S, OP_MRT, false, true>(g.a, t, x0, y, z); break;
        default: if constexpr ((M & 32u) != 0) step_pair<S, OP_MRT, true, true>(g.a, t, x0, y, z); break;
    }
}

}  // namespace LBM_ARITH_NS
}  // namespace lbm
