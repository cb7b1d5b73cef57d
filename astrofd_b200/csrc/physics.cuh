// physics.cuh -- pointwise SRHD / RMHD physics of AstroFD's right-hand side,
// as device functions templated on the arithmetic type R (double for the
// FP64 path, float for the mixed-precision reconstruction/Riemann path).
//
// Formulas, clamps and evaluation order follow the reference (paths relative
// to the AstroFD checkout):
//   core/srhd_core.py  prim_to_cons :47, cons_to_prim :62, sound_speed :134,
//                      eig_speeds :143, flux_* :157, hlle :172, hllc_flux_* :189,
//                      minmod/mc_lim :306,314, ppm_reconstruct :328,
//                      weno5_left/right :344,362, floor_prim :380
//   core/rmhd_core.py  limiter :61, floor_prim_rmhd :126, prim_to_cons_rmhd :138,
//                      _cons_to_prim_hydro :171, rmhd_f_of_Z :229,
//                      cons_to_prim_rmhd :249, flux_rmhd_* :344, rmhd_fast_speed :420,
//                      hllc_hydro_flux_* :474, riemann_flux_rmhd_* :570,
//                      hllc_contact_speed_* :581, hll_d_flux_dir :602
// Directions are a runtime index n (0 = x, 1 = y, 2 = z); the per-direction
// copies of the reference differ only in which component is normal.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include "../../include/astrofd.h"

#define AHD __host__ __device__ __forceinline__

namespace astro {

template <typename R> struct C {
    static constexpr R small = R(1e-12);
};

template <typename R> AHD R rmax(R a, R b) { return a > b ? a : b; }
template <typename R> AHD R rmin(R a, R b) { return a < b ? a : b; }
template <typename R> AHD R rsqrt_(R x) { return sqrt(x); }
template <typename R> AHD R rabs(R x) { return x < R(0) ? -x : x; }

// The float32 face path takes one approximate reciprocal per shared
// denominator (rcp.approx.ftz.f32, one MUFU operation, relative error about
// one ulp) and rsqrt.approx.ftz.f32 for 1/sqrt, where a division compiles to
// a reciprocal plus range fix-ups; the float64 path keeps the reference's
// IEEE divisions and square roots exactly as written.
template <typename R> AHD R rcp_(R x) {
#ifdef __CUDA_ARCH__
    if constexpr (sizeof(R) == 4) {
        float y;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
        return y;
    }
#endif
    return R(1) / x;
}
template <typename R> AHD R rsq_(R x) {
#ifdef __CUDA_ARCH__
    if constexpr (sizeof(R) == 4) {
        float y;
        asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
        return y;
    }
#endif
    return R(1) / sqrt(x);
}
// Float64 reciprocal for the learned con2prim's polish (not the reference's
// own solve, which keeps IEEE divisions): the hardware approximation
// rcp.approx.ftz.f64 refined by two Newton-Raphson steps for 1/x,
// r <- r + r (1 - x r), each of which squares the relative error, which ends
// at float64 rounding (within 2 ulp of 1/x, checked on the device against the
// IEEE quotient).  For normal, non-zero x, which is all its callers pass; a
// subnormal x is flushed to zero.
AHD double rcp_nr(double x) {
#ifdef __CUDA_ARCH__
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
#else
    return 1.0 / x;
#endif
}

// a / b: float32 as a * rcp(b), float64 as the IEEE quotient
template <typename R> AHD R qdiv(R a, R b) {
    if constexpr (sizeof(R) == 4) return a * rcp_(b);
    else return a / b;
}

// Physical parameters in the arithmetic type of the caller.
template <typename R> struct Phys {
    R gamma, srhd_gamma, p_max, v_max, glm_ch, glm_cp;
    int limiter, riemann;
    AHD static Phys from(const AstroParams& p) {
        Phys q;
        q.gamma = R(p.gamma); q.srhd_gamma = R(p.srhd_gamma);
        q.p_max = R(p.p_max); q.v_max = R(p.v_max);
        q.glm_ch = R(p.glm_ch); q.glm_cp = R(p.glm_cp);
        q.limiter = p.limiter; q.riemann = p.riemann;
        return q;
    }
};

// ---------------------------------------------------------------- recon ---
template <typename R> AHD R minmod(R a, R b) {
    if (a * b <= R(0)) return R(0);
    return rabs(a) < rabs(b) ? a : b;
}

template <typename R> AHD R limiter(int id, R dqL, R dqR) {
    if (id == ASTRO_LIM_MINMOD) return minmod(dqL, dqR);
    if (id == ASTRO_LIM_VANLEER) {
        if (dqL * dqR <= R(0)) return R(0);
        R denom = dqL + dqR;
        if (denom == R(0)) return R(0);
        return (R(2) * dqL * dqR) / denom;
    }
    R mm = minmod(dqL, dqR);
    return minmod(R(0.5) * (dqL + dqR), R(2) * mm);
}

template <typename R> AHD void ppm(R q_im2, R q_im1, R q_i, R q_ip1, R q_ip2, R& oL, R& oR) {
    R qL = R(7.0 / 12.0) * (q_im1 + q_i) - R(1.0 / 12.0) * (q_im2 + q_ip1);
    R qR = R(7.0 / 12.0) * (q_i + q_ip1) - R(1.0 / 12.0) * (q_im1 + q_ip2);
    R qmax = rmax(rmax(q_im1, q_i), q_ip1);
    R qmin = rmin(rmin(q_im1, q_i), q_ip1);
    if (qL > qmax) qL = qmax;
    if (qL < qmin) qL = qmin;
    if (qR > qmax) qR = qmax;
    if (qR < qmin) qR = qmin;
    if ((qR - q_i) * (q_i - qL) <= R(0)) { qL = q_i; qR = q_i; }
    oL = qL; oR = qR;
}

// Jiang-Shu WENO5 value at the face on the (a..e) side; weno5_right of the
// reference is the same formula with the stencil reversed.
template <typename R> AHD R weno5(R a, R b, R c, R d, R e) {
    const R eps = R(1e-12);
    R t0 = a - R(2) * b + c, u0 = a - R(4) * b + R(3) * c;
    R t1 = b - R(2) * c + d, u1 = b - d;
    R t2 = c - R(2) * d + e, u2 = R(3) * c - R(4) * d + e;
    R IS0 = R(13.0 / 12.0) * (t0 * t0) + R(0.25) * (u0 * u0);
    R IS1 = R(13.0 / 12.0) * (t1 * t1) + R(0.25) * (u1 * u1);
    R IS2 = R(13.0 / 12.0) * (t2 * t2) + R(0.25) * (u2 * u2);
    R p0 = R(1.0 / 3.0) * a - R(7.0 / 6.0) * b + R(11.0 / 6.0) * c;
    R p1 = R(-1.0 / 6.0) * b + R(5.0 / 6.0) * c + R(1.0 / 3.0) * d;
    R p2 = R(1.0 / 3.0) * c + R(5.0 / 6.0) * d - R(1.0 / 6.0) * e;
    if constexpr (sizeof(R) == 4) {
        // four reciprocals instead of six divisions; a weight whose
        // (eps + IS)^2 overflows goes to 0 as in the quotient form
        const R a0 = R(0.1) * rcp_((eps + IS0) * (eps + IS0));
        const R a1 = R(0.6) * rcp_((eps + IS1) * (eps + IS1));
        const R a2 = R(0.3) * rcp_((eps + IS2) * (eps + IS2));
        return (a0 * p0 + a1 * p1 + a2 * p2) * rcp_(a0 + a1 + a2);
    } else {
        R a0 = R(0.1) / ((eps + IS0) * (eps + IS0));
        R a1 = R(0.6) / ((eps + IS1) * (eps + IS1));
        R a2 = R(0.3) / ((eps + IS2) * (eps + IS2));
        R s = a0 + a1 + a2;
        R w0 = a0 / s, w1 = a1 / s, w2 = a2 / s;
        return w0 * p0 + w1 * p1 + w2 * p2;
    }
}

#ifdef __CUDA_ARCH__
// Both WENO5 face values of a float32 stencil s[0..5] at once: lane x is the
// left-biased value weno5(s0..s4), lane y the right-biased weno5(s5..s1), the
// same formula on mirrored stencils, so every add/multiply is one packed
// float32x2 instruction (FADD2/FMUL2/FFMA2) and only the reciprocals are
// scalar.
__device__ __forceinline__ float2 weno5_pair(const float* s) {
    const float2 A = make_float2(s[0], s[5]), B = make_float2(s[1], s[4]);
    const float2 Cc = make_float2(s[2], s[3]), D = make_float2(s[3], s[2]);
    const float2 E = make_float2(s[4], s[1]);
    auto k2 = [](float c) { return make_float2(c, c); };
    const float2 m2 = k2(-2.f);
    const float2 t0 = __fadd2_rn(__ffma2_rn(B, m2, A), Cc);
    const float2 u0 = __ffma2_rn(Cc, k2(3.f), __ffma2_rn(B, k2(-4.f), A));
    const float2 t1 = __fadd2_rn(__ffma2_rn(Cc, m2, B), D);
    const float2 u1 = __fadd2_rn(B, __fmul2_rn(D, k2(-1.f)));
    const float2 t2 = __fadd2_rn(__ffma2_rn(D, m2, Cc), E);
    const float2 u2 = __fadd2_rn(__ffma2_rn(D, k2(-4.f), __fmul2_rn(Cc, k2(3.f))), E);
    const float2 c13 = k2(13.f / 12.f), q = k2(0.25f), eps = k2(1e-12f);
    const float2 w0 = __ffma2_rn(__fmul2_rn(t0, c13), t0, __ffma2_rn(__fmul2_rn(u0, q), u0, eps));
    const float2 w1 = __ffma2_rn(__fmul2_rn(t1, c13), t1, __ffma2_rn(__fmul2_rn(u1, q), u1, eps));
    const float2 w2 = __ffma2_rn(__fmul2_rn(t2, c13), t2, __ffma2_rn(__fmul2_rn(u2, q), u2, eps));
    const float2 v0 = __fmul2_rn(w0, w0), v1 = __fmul2_rn(w1, w1), v2 = __fmul2_rn(w2, w2);
    const float2 a0 = __fmul2_rn(make_float2(rcp_(v0.x), rcp_(v0.y)), k2(0.1f));
    const float2 a1 = __fmul2_rn(make_float2(rcp_(v1.x), rcp_(v1.y)), k2(0.6f));
    const float2 a2 = __fmul2_rn(make_float2(rcp_(v2.x), rcp_(v2.y)), k2(0.3f));
    const float2 p0 = __ffma2_rn(Cc, k2(11.f / 6.f), __ffma2_rn(B, k2(-7.f / 6.f), __fmul2_rn(A, k2(1.f / 3.f))));
    const float2 p1 = __ffma2_rn(D, k2(1.f / 3.f), __ffma2_rn(Cc, k2(5.f / 6.f), __fmul2_rn(B, k2(-1.f / 6.f))));
    const float2 p2 = __ffma2_rn(E, k2(-1.f / 6.f), __ffma2_rn(D, k2(5.f / 6.f), __fmul2_rn(Cc, k2(1.f / 3.f))));
    const float2 num = __ffma2_rn(a2, p2, __ffma2_rn(a1, p1, __fmul2_rn(a0, p0)));
    const float2 den = __fadd2_rn(__fadd2_rn(a0, a1), a2);
    return __fmul2_rn(num, make_float2(rcp_(den.x), rcp_(den.y)));
}
#endif

// Left/right states at the face between cell c-1 and c from a stencil
// a[0..5] = q(c-3) .. q(c+2).  MUSCL uses a[1..4].
template <int RECON, typename R> AHD void recon_face(const R* a, int lim, R& qL, R& qR) {
    if (RECON == ASTRO_RECON_MUSCL) {
        R slL = limiter(lim, a[2] - a[1], a[3] - a[2]);
        R slR = limiter(lim, a[3] - a[2], a[4] - a[3]);
        qL = a[2] + R(0.5) * slL;
        qR = a[3] - R(0.5) * slR;
    } else if (RECON == ASTRO_RECON_PPM) {
        R l0, r0, l1, r1;
        ppm(a[0], a[1], a[2], a[3], a[4], l0, r0);
        ppm(a[1], a[2], a[3], a[4], a[5], l1, r1);
        qL = r0; qR = l1;
    } else {
#ifdef __CUDA_ARCH__
        if constexpr (sizeof(R) == 4) {
            const float2 lr = weno5_pair(a);
            qL = lr.x;
            qR = lr.y;
            return;
        }
#endif
        qL = weno5(a[0], a[1], a[2], a[3], a[4]);
        qR = weno5(a[5], a[4], a[3], a[2], a[1]);
    }
}

template <typename R> AHD R hlle_scalar(R qL, R qR, R fL, R fR, R sL, R sR) {
    if (sL >= R(0)) return fL;
    if (sR <= R(0)) return fR;
    return (sR * fL - sL * fR + sL * sR * (qR - qL)) / (sR - sL + C<R>::small);
}

// HLLE flux of components [V0, N)
template <int N, typename R, int V0 = 0>
AHD void hlle(const R* UL, const R* UR, const R* FL, const R* FR, R sL, R sR, R* out) {
    if (sL >= R(0)) { for (int v = V0; v < N; ++v) out[v] = FL[v]; return; }
    if (sR <= R(0)) { for (int v = V0; v < N; ++v) out[v] = FR[v]; return; }
    R inv = sR - sL + C<R>::small;
    if constexpr (sizeof(R) == 4) {
        const R ri = rcp_(inv);
#pragma unroll
        for (int v = V0; v < N; ++v) out[v] = (sR * FL[v] - sL * FR[v] + sL * sR * (UR[v] - UL[v])) * ri;
    } else {
#pragma unroll
        for (int v = V0; v < N; ++v) out[v] = (sR * FL[v] - sL * FR[v] + sL * sR * (UR[v] - UL[v])) / inv;
    }
}

template <typename R> AHD void eig_speeds(R vn, R cs, R& lm, R& lp) {
    R dp = R(1) + vn * cs, dm = R(1) - vn * cs;
    if (dp == R(0)) dp = C<R>::small;
    if (dm == R(0)) dm = C<R>::small;
    R p, m;
    if constexpr (sizeof(R) == 4) {
        const R r = rcp_(dp * dm);
        p = (vn + cs) * dm * r;
        m = (vn - cs) * dp * r;
    } else {
        p = (vn + cs) / dp;
        m = (vn - cs) / dm;
    }
    if (p > R(1)) p = R(1);
    if (p < R(-1)) p = R(-1);
    if (m > R(1)) m = R(1);
    if (m < R(-1)) m = R(-1);
    lm = m; lp = p;
}

// ----------------------------------------------------------------- SRHD ---
template <typename R> AHD void s_p2c(const Phys<R>& P, const R* q, R* U) {
    const R gamma = P.srhd_gamma;
    R rho = q[0], vx = q[1], vy = q[2], vz = q[3], p = q[4];
    R v2 = vx * vx + vy * vy + vz * vz;
    if (v2 >= R(1)) v2 = R(1) - R(1e-14);
    R W = sizeof(R) == 4 ? rsq_(R(1) - v2) : R(1) / rsqrt_(R(1) - v2);
    R h = R(1) + qdiv(gamma / (gamma - R(1)) * p, rmax(rho, C<R>::small));
    R w = rho * h;
    U[0] = rho * W;
    R wW2 = w * W * W;
    U[1] = wW2 * vx;
    U[2] = wW2 * vy;
    U[3] = wW2 * vz;
    U[4] = wW2 - p - U[0];
}

template <typename R> AHD R s_sound_speed(const Phys<R>& P, R rho, R p) {
    const R gamma = P.srhd_gamma;
    R h = R(1) + qdiv(gamma / (gamma - R(1)) * p, rmax(rho, C<R>::small));
    R w = rho * h;
    R cs2 = qdiv(gamma * p, rmax(w, C<R>::small));
    if (cs2 < R(0)) cs2 = R(0);
    if (cs2 > R(1) - R(1e-14)) cs2 = R(1) - R(1e-14);
    return rsqrt_(cs2);
}

template <typename R> AHD void floor_prim(const Phys<R>& P, R* q) {
    if (q[0] < C<R>::small) q[0] = C<R>::small;
    if (q[4] < C<R>::small) q[4] = C<R>::small;
    if (q[4] > P.p_max) q[4] = P.p_max;
    R v2 = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    R vmax2 = P.v_max * P.v_max;
    if (v2 >= vmax2) {
        R fac = P.v_max / rsqrt_(v2 + R(1e-32));
        q[1] *= fac; q[2] *= fac; q[3] *= fac;
    }
}

// physical flux from primitives q and their conserved state U = p2c(q)
// (the reference recomputes p2c inside flux_x/y/z, srhd_core.py:157-169; the
// caller's U is the same value, so it is reused)
template <typename R> AHD void s_flux_u(const Phys<R>& P, int n, const R* q, const R* U, R* F) {
    R vn = q[1 + n], p = q[4];
    F[0] = U[0] * vn;
#pragma unroll
    for (int m = 0; m < 3; ++m) F[1 + m] = (m == n) ? U[1 + m] * vn + p : U[1 + m] * vn;
    F[4] = (U[4] + p) * vn;
}

template <typename R> AHD void s_flux(const Phys<R>& P, int n, const R* q, R* F) {
    R U[5];
    s_p2c(P, q, U);
    s_flux_u(P, n, q, U, F);
}

template <typename R> AHD R contact_speed(int n, const R* UL, const R* UR, R sL, R sR, R pL,
                                          R pR, R vL, R vR) {
    R denom = (UL[0] * (sL - vL) - UR[0] * (sR - vR)) + C<R>::small;
    return qdiv(pR - pL + UL[1 + n] * (sL - vL) - UR[1 + n] * (sR - vR), denom);
}

// HLLC for SRHD / the hydro block of RMHD "hlld"
template <typename R>
AHD void hllc5(int n, const R* UL, const R* UR, const R* FL, const R* FR, R sL, R sR, R pL,
               R pR, R vL, R vR, R* out) {
    if (sL >= R(0)) { for (int v = 0; v < 5; ++v) out[v] = FL[v]; return; }
    if (sR <= R(0)) { for (int v = 0; v < 5; ++v) out[v] = FR[v]; return; }
    R DL = UL[0], DR = UR[0];
    R denom = (DL * (sL - vL) - DR * (sR - vR)) + C<R>::small;
    R sM = qdiv(pR - pL + UL[1 + n] * (sL - vL) - UR[1 + n] * (sR - vR), denom);
    R pStar = R(0.5) * (pL + pR + DL * (sL - vL) * (sM - vL) + DR * (sR - vR) * (sM - vR));
    const bool left = sM >= R(0);
    const R* U = left ? UL : UR;
    const R* F = left ? FL : FR;
    R s = left ? sL : sR, pK = left ? pL : pR, vK = left ? vL : vR;
    R den = s - sM + C<R>::small;
    R fac, dpx, dex;
    if constexpr (sizeof(R) == 4) {
        const R rd = rcp_(den);
        fac = (s - vK) * rd;
        dpx = (pStar - pK) * rd;
        dex = (pStar * sM - pK * vK) * rd;
    } else {
        fac = (s - vK) / den;
        dpx = (pStar - pK) / den;
        dex = (pStar * sM - pK * vK) / den;
    }
    R Ust[5];
    Ust[0] = U[0] * fac;
#pragma unroll
    for (int m = 0; m < 3; ++m)
        Ust[1 + m] = (m == n) ? U[1 + m] * fac + dpx : U[1 + m] * fac;
    Ust[4] = U[4] * fac + dex;
#pragma unroll
    for (int v = 0; v < 5; ++v) out[v] = F[v] + s * (Ust[v] - U[v]);
}

// Israel-Stewart dissipation flux of one cell added to a face flux
// (add_diss_flux_x/y/z, srhd_core.py:417-442).  is = pi, pixx, piyy, pizz,
// pixy, pixz, piyz, qx, qy, qz of the cell; q the face primitives after the
// floor.  Stress row n: pi delta_nm + pi^nm; energy: v . row + q_n, summed in
// the reference's order.
template <typename R> AHD void s_diss_flux(int n, const R* q, const R* is, R* F) {
    constexpr int S[3][3] = {{1, 4, 5}, {4, 2, 6}, {5, 6, 3}};
    R row[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) row[m] = (m == n) ? is[0] + is[S[n][m]] : is[S[n][m]];
#pragma unroll
    for (int m = 0; m < 3; ++m) F[1 + m] += row[m];
    F[4] += q[1] * row[0] + q[2] * row[1] + q[3] * row[2] + is[7 + n];
}

// one SRHD face: floor, p2c, flux, (ndiss times the dissipation fluxes of the
// cells isL / isR), speeds, Riemann (srhd_core.py:517-550)
template <int RIEMANN, typename R>
AHD void s_face(const Phys<R>& P, int n, R* qL, R* qR, R* F, R& sL, R& sR, int ndiss = 0,
                const R* isL = nullptr, const R* isR = nullptr) {
    R UL[5], UR[5], FL[5], FR[5], lmL, lpL, lmR, lpR;
    floor_prim(P, qL);
    floor_prim(P, qR);
    s_p2c(P, qL, UL);
    s_p2c(P, qR, UR);
    s_flux_u(P, n, qL, UL, FL);
    s_flux_u(P, n, qR, UR, FR);
    for (int rep = 0; rep < ndiss; ++rep) {
        s_diss_flux(n, qL, isL, FL);
        s_diss_flux(n, qR, isR, FR);
    }
    R csL = s_sound_speed(P, qL[0], qL[4]), csR = s_sound_speed(P, qR[0], qR[4]);
    eig_speeds(qL[1 + n], csL, lmL, lpL);
    eig_speeds(qR[1 + n], csR, lmR, lpR);
    sL = rmin(lmL, lmR);
    sR = rmax(lpL, lpR);
    if (RIEMANN == ASTRO_RIEMANN_HLLC)
        hllc5(n, UL, UR, FL, FR, sL, sR, qL[4], qR[4], qL[1 + n], qR[1 + n], F);
    else
        hlle<5>(UL, UR, FL, FR, sL, sR, F);
}

// ----------------------------------------------------------------- RMHD ---
// rhoh_out / b2_out: rho h and b^2 of the state, for the fast speed of the
// same (floored) state on the float32 faces
template <typename R>
AHD void r_p2c(const Phys<R>& P, const R* qin, R* U, R* rhoh_out = nullptr,
               R* b2_out = nullptr, R* B2_out = nullptr, R* vb_out = nullptr) {
    const R gamma = P.gamma;
    R rho = qin[0], vx = qin[1], vy = qin[2], vz = qin[3], p = qin[4];
    R Bx = qin[5], By = qin[6], Bz = qin[7];
    R v2 = vx * vx + vy * vy + vz * vz;
    R vmax2 = P.v_max * P.v_max;
    if (v2 >= vmax2) {
        R fac = P.v_max / rsqrt_(v2 + R(1e-32));
        vx *= fac; vy *= fac; vz *= fac;
    }
    if (p < C<R>::small) p = C<R>::small;
    if (p > P.p_max) p = P.p_max;
    R B2 = Bx * Bx + By * By + Bz * Bz;
    R W, bx, by, bz;
    R h = R(1) + qdiv(gamma / (gamma - R(1)) * p, rmax(rho, C<R>::small));
    R rhoh = rho * h;
    R vb = vx * Bx + vy * By + vz * Bz;
    if constexpr (sizeof(R) == 4) {
        const R om = R(1) - (vx * vx + vy * vy + vz * vz);
        W = rsq_(om);
        const R iW = om * W;  // sqrt(1 - v^2)
        const R b0 = W * vb;
        bx = (Bx + b0 * vx) * iW; by = (By + b0 * vy) * iW; bz = (Bz + b0 * vz) * iW;
    } else {
        W = R(1) / rsqrt_(R(1) - (vx * vx + vy * vy + vz * vz));
        const R b0 = W * vb;  // divisions kept as in the reference
        bx = (Bx + b0 * vx) / W; by = (By + b0 * vy) / W; bz = (Bz + b0 * vz) / W;
    }
    R b0 = W * vb;
    R b2 = (bx * bx + by * by + bz * bz) - b0 * b0;
    R rhohW2 = rhoh * W * W;
    R wtot = rhohW2 + B2;
    R D = rho * W;
    U[0] = D;
    U[1] = wtot * vx - (Bx * vb);
    U[2] = wtot * vy - (By * vb);
    U[3] = wtot * vz - (Bz * vb);
    U[4] = rhohW2 - p + R(0.5) * B2 + R(0.5) * b2 - D;
    U[5] = Bx; U[6] = By; U[7] = Bz; U[8] = qin[8];
    if (rhoh_out) *rhoh_out = rhoh;
    if (b2_out) *b2_out = b2;
    if (B2_out) *B2_out = B2;
    if (vb_out) *vb_out = vb;
}

// physical flux from primitives q and U = p2c(q) (flux_rmhd_x/y/z,
// rmhd_core.py:344-395, recompute p2c internally; reused here)
// B2, Bv: B^2 and B . v of q when the caller has them (p2c of the same q)
template <typename R>
AHD void r_flux_u(const Phys<R>& P, int n, const R* q, const R* U, R* F, R B2 = R(-1),
                  R Bv = R(0)) {
    R v[3] = {q[1], q[2], q[3]}, B[3] = {q[5], q[6], q[7]};
    R p = q[4], psi = q[8];
    if (B2 < R(0)) {
        B2 = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
        Bv = B[0] * v[0] + B[1] * v[1] + B[2] * v[2];
    }
    R pt = p + R(0.5) * B2;
    R vn = v[n], Bn = B[n];
    F[0] = U[0] * vn;
#pragma unroll
    for (int m = 0; m < 3; ++m)
        F[1 + m] = (m == n) ? U[1 + m] * vn + pt - Bn * Bn : U[1 + m] * vn - Bn * B[m];
    F[4] = (U[4] + pt) * vn - (Bn * Bv);
#pragma unroll
    for (int m = 0; m < 3; ++m) F[5 + m] = (m == n) ? psi : v[m] * Bn - vn * B[m];
    F[8] = P.glm_ch * P.glm_ch * Bn;
}

template <typename R> AHD void r_flux(const Phys<R>& P, int n, const R* q, R* F) {
    R U[9];
    r_p2c(P, q, U);
    r_flux_u(P, n, q, U, F);
}

// fast magnetosonic speed from rho h and b^2 (rmhd_fast_speed,
// rmhd_core.py:420-458, after its b-vector)
template <typename R> AHD R r_fast_speed_from(const Phys<R>& P, R p, R rhoh, R b2) {
    const R G = P.gamma;
    R cs2 = qdiv(G * p, rmax(rhoh, C<R>::small));
    if (cs2 < R(0)) cs2 = R(0);
    if (cs2 > R(1) - R(1e-14)) cs2 = R(1) - R(1e-14);
    R ca2 = qdiv(b2, rmax(rhoh + b2, C<R>::small));
    if (ca2 < R(0)) ca2 = R(0);
    if (ca2 > R(1) - R(1e-14)) ca2 = R(1) - R(1e-14);
    R a = cs2 + ca2 - cs2 * ca2;
    R disc = a * a - R(4) * cs2 * ca2;
    if (disc < R(0)) disc = R(0);
    R cf2 = R(0.5) * (a + rsqrt_(disc));
    if (cf2 < R(0)) cf2 = R(0);
    if (cf2 > R(1) - R(1e-14)) cf2 = R(1) - R(1e-14);
    return rsqrt_(cf2);
}

template <typename R> AHD R r_fast_speed(const Phys<R>& P, const R* q) {
    const R G = P.gamma;
    R rho = q[0], vx = q[1], vy = q[2], vz = q[3], p = q[4];
    R Bx = q[5], By = q[6], Bz = q[7];
    R v2 = vx * vx + vy * vy + vz * vz;
    if (v2 >= P.v_max * P.v_max) v2 = P.v_max * P.v_max - R(1e-14);
    if (rho < C<R>::small) rho = C<R>::small;
    if (p < C<R>::small) p = C<R>::small;
    if (p > P.p_max) p = P.p_max;
    R h = R(1) + qdiv(G / (G - R(1)) * p, rmax(rho, C<R>::small));
    R rhoh = rho * h;
    R vb = vx * Bx + vy * By + vz * Bz;
    R W, bx, by, bz;
    if constexpr (sizeof(R) == 4) {
        W = rsq_(R(1) - v2);
        const R iW = (R(1) - v2) * W;
        const R b0 = W * vb;
        bx = (Bx + b0 * vx) * iW; by = (By + b0 * vy) * iW; bz = (Bz + b0 * vz) * iW;
    } else {
        W = R(1) / rsqrt_(R(1) - v2);
        const R b0 = W * vb;
        bx = (Bx + b0 * vx) / W; by = (By + b0 * vy) / W; bz = (Bz + b0 * vz) / W;
    }
    R b0 = W * vb;
    R b2 = (bx * bx + by * by + bz * bz) - b0 * b0;
    return r_fast_speed_from(P, p, rhoh, b2);
}

// hll_d_flux_dir (rmhd_core.py:602-724): approximate HLLD, HLLE on degenerate states
template <typename R>
AHD void r_hlld_full(const Phys<R>& P, int n, const R* UL, const R* UR, const R* FL,
                     const R* FR, R sL, R sR, R pL, R pR, R vL, R vR, R* out) {
    if (sL >= R(0)) { for (int v = 0; v < 9; ++v) out[v] = FL[v]; return; }
    if (sR <= R(0)) { for (int v = 0; v < 9; ++v) out[v] = FR[v]; return; }
    const R SM = C<R>::small;
    const int t1 = (n == 0) ? 1 : 0, t2 = (n == 2) ? 1 : 2;
    if (UL[0] <= SM || UR[0] <= SM) { hlle<9>(UL, UR, FL, FR, sL, sR, out); return; }
    R Bn = R(0.5) * (UL[5 + n] + UR[5 + n]);
    if (rabs(Bn) < R(1e-8)) { hlle<9>(UL, UR, FL, FR, sL, sR, out); return; }
    R Bt1L = UL[5 + t1], Bt2L = UL[5 + t2], Bt1R = UR[5 + t1], Bt2R = UR[5 + t2];
    R sM = contact_speed(n, UL, UR, sL, sR, pL, pR, vL, vR);
    R DL = UL[0], DR = UR[0];
    R dLs = sL - sM + SM, dRs = sR - sM + SM;
    R DstarL = DL * (sL - vL) / dLs;
    R DstarR = DR * (sR - vR) / dRs;
    if (DstarL <= SM || DstarR <= SM) { hlle<9>(UL, UR, FL, FR, sL, sR, out); return; }
    R Bt1Ls = Bt1L * (sL - vL) / dLs, Bt2Ls = Bt2L * (sL - vL) / dLs;
    R Bt1Rs = Bt1R * (sR - vR) / dRs, Bt2Rs = Bt2R * (sR - vR) / dRs;
    R denomL = DL * (sL - vL) - Bn * Bn;
    R denomR = DR * (sR - vR) - Bn * Bn;
    if (rabs(denomL) < SM || rabs(denomR) < SM) { hlle<9>(UL, UR, FL, FR, sL, sR, out); return; }
    R vt1L = UL[1 + t1] / rmax(DL, SM), vt2L = UL[1 + t2] / rmax(DL, SM);
    R vt1R = UR[1 + t1] / rmax(DR, SM), vt2R = UR[1 + t2] / rmax(DR, SM);
    R vt1Ls = vt1L - Bn * (Bt1L - Bt1Ls) / denomL;
    R vt2Ls = vt2L - Bn * (Bt2L - Bt2Ls) / denomL;
    R vt1Rs = vt1R - Bn * (Bt1R - Bt1Rs) / denomR;
    R vt2Rs = vt2R - Bn * (Bt2R - Bt2Rs) / denomR;
    R sLs = sM - rabs(Bn) / rsqrt_(DstarL + SM);
    R sRs = sM + rabs(Bn) / rsqrt_(DstarR + SM);
    R sqL = rsqrt_(DstarL), sqR = rsqrt_(DstarR);
    R sgn = (Bn >= R(0)) ? R(1) : R(-1);
    R den = sqL + sqR + SM;
    // which fan region: only the needed star states are built
    int region;
    if (sL <= R(0) && R(0) <= sLs) region = 0;
    else if (sLs <= R(0) && R(0) <= sM) region = 1;
    else if (sM <= R(0) && R(0) <= sRs) region = 2;
    else if (sRs <= R(0) && R(0) <= sR) region = 3;
    else { hlle<9>(UL, UR, FL, FR, sL, sR, out); return; }
    const bool leftside = region <= 1;
    const R* UK = leftside ? UL : UR;
    const R* FK = leftside ? FL : FR;
    R sK = leftside ? sL : sR;
    R DK = leftside ? DstarL : DstarR;
    R q[9], UKs[9];
    // star state on the chosen side (build_state, rmhd_core.py:671-693)
    q[0] = rmax(DK, SM);
    q[1 + n] = sM;
    q[1 + t1] = leftside ? vt1Ls : vt1Rs;
    q[1 + t2] = leftside ? vt2Ls : vt2Rs;
    q[4] = (DK == DstarL) ? pL : pR;
    q[5 + n] = Bn;
    q[5 + t1] = leftside ? Bt1Ls : Bt1Rs;
    q[5 + t2] = leftside ? Bt2Ls : Bt2Rs;
    q[8] = UK[8];
    r_p2c(P, q, UKs);
    if (region == 0 || region == 3) {
#pragma unroll
        for (int v = 0; v < 9; ++v) out[v] = FK[v] + sK * (UKs[v] - UK[v]);
        return;
    }
    R Dss = R(0.5) * (DstarL + DstarR);
    R qs[9], Us[9];
    qs[0] = rmax(Dss, SM);
    qs[1 + n] = sM;
    qs[1 + t1] = (sqL * vt1Ls + sqR * vt1Rs + sgn * (Bt1Rs - Bt1Ls)) / den;
    qs[1 + t2] = (sqL * vt2Ls + sqR * vt2Rs + sgn * (Bt2Rs - Bt2Ls)) / den;
    qs[4] = (Dss == DstarL) ? pL : pR;
    qs[5 + n] = Bn;
    qs[5 + t1] = (sqL * Bt1Rs + sqR * Bt1Ls + sgn * sqL * sqR * (vt1Ls - vt1Rs)) / den;
    qs[5 + t2] = (sqL * Bt2Rs + sqR * Bt2Ls + sgn * sqL * sqR * (vt2Ls - vt2Rs)) / den;
    qs[8] = R(0.5) * (UL[8] + UR[8]);
    r_p2c(P, qs, Us);
    R sKs = leftside ? sLs : sRs;
#pragma unroll
    for (int v = 0; v < 9; ++v) out[v] = FK[v] + sK * (UKs[v] - UK[v]) + sKs * (Us[v] - UKs[v]);
}

// Riemann dispatch with given speeds; MUSCL_OVR adds the MUSCL-only upwind
// override of the induction/GLM fluxes for "hlld" (rmhd_core.py:811-831).
template <int RIEMANN, bool MUSCL_OVR, typename R>
AHD void r_riemann(const Phys<R>& P, int n, const R* qL, const R* qR, const R* UL,
                   const R* UR, const R* FL, const R* FR, R sL, R sR, R* out) {
    R pL = qL[4], pR = qR[4], vL = qL[1 + n], vR = qR[1 + n];
    if (RIEMANN == ASTRO_RIEMANN_HLLD_FULL) {
        r_hlld_full(P, n, UL, UR, FL, FR, sL, sR, pL, pR, vL, vR, out);
    } else if (RIEMANN == ASTRO_RIEMANN_HLLD) {
        // HLLE for the field and psi, HLLC for the hydro block (which the
        // reference computes with HLLE first and then overwrites)
        hlle<9, R, 5>(UL, UR, FL, FR, sL, sR, out);
        hllc5(n, UL, UR, FL, FR, sL, sR, pL, pR, vL, vR, out);
        if (MUSCL_OVR) {
            R sM = contact_speed(n, UL, UR, sL, sR, pL, pR, vL, vR);
            const R* Fm = (sM >= R(0)) ? FL : FR;
#pragma unroll
            for (int v = 5; v < 9; ++v) out[v] = Fm[v];
        }
    } else {
        hlle<9>(UL, UR, FL, FR, sL, sR, out);
    }
}

template <typename R>
AHD void r_speeds(const Phys<R>& P, int n, const R* qL, const R* qR, R& sL, R& sR) {
    R lmL, lpL, lmR, lpR;
    R cfL = r_fast_speed(P, qL), cfR = r_fast_speed(P, qR);
    eig_speeds(qL[1 + n], cfL, lmL, lpL);
    eig_speeds(qR[1 + n], cfR, lmR, lpR);
    sL = rmin(lmL, lmR);
    sR = rmax(lpL, lpR);
}

// one RMHD face.  GIVEN: use the supplied (sL, sR) instead of the face's own
// speeds (the reference's loop-carried x-face speeds, rmhd_core.py:1445,1468).
template <int RIEMANN, bool MUSCL_OVR, bool GIVEN, typename R>
AHD void r_face(const Phys<R>& P, int n, R* qL, R* qR, R* F, R& sL, R& sR) {
    R UL[9], UR[9], FL[9], FR[9];
    floor_prim(P, qL);
    floor_prim(P, qR);
    if constexpr (sizeof(R) == 4) {
        // float32 faces: the fast speeds from p2c's rho h and b^2 of the
        // same floored states (equal to recomputing them, to rounding)
        R rhL, b2L, rhR, b2R, BBL, BBR, vbL, vbR;
        r_p2c(P, qL, UL, &rhL, &b2L, &BBL, &vbL);
        r_p2c(P, qR, UR, &rhR, &b2R, &BBR, &vbR);
        r_flux_u(P, n, qL, UL, FL, BBL, vbL);
        r_flux_u(P, n, qR, UR, FR, BBR, vbR);
        if (!GIVEN) {
            R lmL, lpL, lmR, lpR;
            eig_speeds(qL[1 + n], r_fast_speed_from(P, qL[4], rhL, b2L), lmL, lpL);
            eig_speeds(qR[1 + n], r_fast_speed_from(P, qR[4], rhR, b2R), lmR, lpR);
            sL = rmin(lmL, lmR);
            sR = rmax(lpL, lpR);
        }
    } else {
        r_p2c(P, qL, UL);
        r_p2c(P, qR, UR);
        r_flux_u(P, n, qL, UL, FL);
        r_flux_u(P, n, qR, UR, FR);
        if (!GIVEN) r_speeds(P, n, qL, qR, sL, sR);
    }
    r_riemann<RIEMANN, MUSCL_OVR>(P, n, qL, qR, UL, UR, FL, FR, sL, sR, F);
}

// ------------------------------------------------------- con2prim (FP64) ---
struct C2PCount {
    unsigned newton = 0, bisect = 0, hydro_fallback = 0;
};

AHD void s_c2p(const Phys<double>& P, const double* U, double* q) {
    const double gamma = P.srhd_gamma, SM = 1e-12;
    double D = U[0], Sx = U[1], Sy = U[2], Sz = U[3], tau = U[4];
    double E = tau + D;
    double S2 = Sx * Sx + Sy * Sy + Sz * Sz;
    double p = (gamma - 1.0) * (E - D);
    if (p < SM) p = SM;
    if (p > P.p_max) p = P.p_max;
    bool ok = false;
    const double vmax2 = P.v_max * P.v_max;
    for (int it = 0; it < 60; ++it) {
        double Wm = E + p;
        double v2 = S2 / (Wm * Wm + SM);
        if (v2 >= vmax2) v2 = vmax2 - 1e-14;
        double W = 1.0 / sqrt(1.0 - v2);
        double rho = D / rmax(W, SM);
        double h = 1.0 + gamma / (gamma - 1.0) * p / rmax(rho, SM);
        double f = Wm - rho * h * W * W;
        double dp = -f;
        if (dp > 0.5 * p) dp = 0.5 * p;
        if (dp < -0.5 * p) dp = -0.5 * p;
        double pn = p + dp;
        if (pn < SM) pn = SM;
        if (pn > P.p_max) pn = P.p_max;
        if (fabs(dp) < 1e-12 * rmax(1.0, pn)) { p = pn; ok = true; break; }
        p = pn;
    }
    if (!ok) {
        p = (gamma - 1.0) * (E - D);
        if (p < SM) p = SM;
        if (p > P.p_max) p = P.p_max;
    }
    double Wm = E + p;
    double vx = Sx / rmax(Wm, SM), vy = Sy / rmax(Wm, SM), vz = Sz / rmax(Wm, SM);
    double v2 = vx * vx + vy * vy + vz * vz;
    if (v2 >= vmax2) {
        double fac = P.v_max / sqrt(v2 + 1e-32);
        vx *= fac; vy *= fac; vz *= fac;
    }
    v2 = vx * vx + vy * vy + vz * vz;
    if (v2 >= 1.0) v2 = 1.0 - 1e-14;
    double W = 1.0 / sqrt(1.0 - v2);
    double rho = D / rmax(W, SM);
    if (rho < SM) rho = SM;
    if (p < SM) p = SM;
    if (p > P.p_max) p = P.p_max;
    q[0] = rho; q[1] = vx; q[2] = vy; q[3] = vz; q[4] = p;
}

// _cons_to_prim_hydro (rmhd_core.py:171): the hydro fixed point on p
AHD void r_c2p_hydro(const Phys<double>& P, double D, double Sx, double Sy, double Sz,
                     double tau, double* q) {
    Phys<double> Q = P;
    Q.srhd_gamma = P.gamma;
    double U[5] = {D, Sx, Sy, Sz, tau};
    s_c2p(Q, U, q);
}

AHD double r_f_df_of_Z(const Phys<double>& P, double Z, double D, double tau, double B2,
                       double SB, double S2, double* df, double tol = 0.0);

AHD double r_f_of_Z(const Phys<double>& P, double Z, double D, double tau, double B2,
                    double SB, double S2) {
    const double G = P.gamma, SM = 1e-12;
    double denomZ = rmax(Z, SM);
    double vb = SB / denomZ;
    double ZpB = Z + B2;
    double v2 = (S2 + (SB * SB) * (2.0 * Z + B2) / (denomZ * denomZ)) / (ZpB * ZpB + SM);
    double vmax2 = P.v_max * P.v_max;
    if (v2 >= vmax2) v2 = vmax2 - 1e-14;
    double W2 = 1.0 / (1.0 - v2);
    double W = sqrt(W2);
    double rho = D / rmax(W, SM);
    double h = Z / rmax(rho * W2, SM);
    double p = (h - 1.0) * rho * (G - 1.0) / G;
    if (p < SM) p = SM;
    if (p > P.p_max) p = P.p_max;
    double b2 = B2 / W2 + vb * vb;
    double tau_calc = Z - p + 0.5 * B2 + 0.5 * b2 - D;
    return tau_calc - tau;
}

// f(Z) in the reference's operation order (float64 reference mode), or
// (FAST) the same expressions with the divisions regrouped (r_f_df_of_Z):
// equal to rounding, with a dependency chain about half as long, for the
// learned path's fallback solves, whose time is the latency of its slowest
// cells
template <bool FAST>
AHD double r_f_eval(const Phys<double>& P, double Z, double D, double tau, double B2,
                    double SB, double S2) {
    if constexpr (FAST) return r_f_df_of_Z(P, Z, D, tau, B2, SB, S2, nullptr);
    else return r_f_of_Z(P, Z, D, tau, B2, SB, S2);
}

// The reference's Newton on Z from a starting value: up to 50 steps with the
// forward-difference derivative and +-Z/2 step clamp (rmhd_core.py:268-292).
// Returns true when |f| < 1e-10 max(1, tau).
template <bool FAST = false>
AHD bool r_newton(const Phys<double>& P, double& Z, int max_it, double D, double tau,
                  double B2, double SB, double S2, int* steps = nullptr) {
    const double tol = 1e-10 * rmax(1.0, tau);
    for (int it = 0; it < max_it; ++it) {
        double f = r_f_eval<FAST>(P, Z, D, tau, B2, SB, S2);
        if (fabs(f) < tol) {
            if (steps) *steps = it;
            return true;
        }
        double eps = 1e-6 * rmax(1.0, Z);
        double fp = r_f_eval<FAST>(P, Z + eps, D, tau, B2, SB, S2);
        double dfdZ = (fp - f) / eps;
        if (dfdZ == 0.0) break;
        double dZ = -f / dfdZ;
        if (dZ > 0.5 * Z) dZ = 0.5 * Z;
        if (dZ < -0.5 * Z) dZ = -0.5 * Z;
        Z += dZ;
        if (Z < 1e-12) Z = 1e-12;
    }
    if (steps) *steps = max_it;
    return false;
}

// Primitive recovery once Z is known (rmhd_core.py:320-341); FAST as in
// r_f_eval
template <bool FAST = false>
AHD void r_prims_from_Z(const Phys<double>& P, double Z, const double* U, const double* q0,
                        double* q, C2PCount& cnt) {
    const double G = P.gamma, SM = 1e-12;
    double Sx = U[1], Sy = U[2], Sz = U[3], D = U[0];
    double Bx = U[5], By = U[6], Bz = U[7];
    double B2 = Bx * Bx + By * By + Bz * Bz;
    double SB = Sx * Bx + Sy * By + Sz * Bz;
    double ZpB = Z + B2;
    double vx, vy, vz, rho, h, p;
    if constexpr (FAST) {
        const double vb = SB * (1.0 / rmax(Z, SM));
        const double iZB = 1.0 / rmax(ZpB, SM);
        vx = (Sx + vb * Bx) * iZB;
        vy = (Sy + vb * By) * iZB;
        vz = (Sz + vb * Bz) * iZB;
    } else {
        double vb = SB / rmax(Z, SM);
        vx = (Sx + vb * Bx) / rmax(ZpB, SM);
        vy = (Sy + vb * By) / rmax(ZpB, SM);
        vz = (Sz + vb * Bz) / rmax(ZpB, SM);
    }
    double v2 = vx * vx + vy * vy + vz * vz;
    double vmax2 = P.v_max * P.v_max;
    if (v2 >= vmax2) {
        double fac = P.v_max / sqrt(v2 + 1e-32);
        vx *= fac; vy *= fac; vz *= fac;
    }
    if constexpr (FAST) {
        const double om = 1.0 - (vx * vx + vy * vy + vz * vz);
        rho = D * sqrt(om);
        h = Z / rmax(rho / om, SM);
        p = (h - 1.0) * rho * ((G - 1.0) / G);
    } else {
        double W = 1.0 / sqrt(1.0 - (vx * vx + vy * vy + vz * vz));
        rho = D / rmax(W, SM);
        h = Z / rmax(rho * W * W, SM);
        p = (h - 1.0) * rho * (G - 1.0) / G;
    }
    if (!isfinite(rho) || !isfinite(p) || rho <= 0.0 || p <= 0.0) {
        cnt.hydro_fallback++;
        rho = q0[0]; vx = q0[1]; vy = q0[2]; vz = q0[3]; p = q0[4];
    }
    q[0] = rho; q[1] = vx; q[2] = vy; q[3] = vz; q[4] = p;
    q[5] = Bx; q[6] = By; q[7] = Bz; q[8] = U[8];
    floor_prim(P, q);
}

// Bisection fallback (rmhd_core.py:294-318); Z holds the last Newton iterate
template <bool FAST = false>
AHD void r_bisect(const Phys<double>& P, double& Z, double Z1, double D, double tau, double B2,
                  double SB, double S2) {
    double Zmin = 1e-12;
    double Zmax = rmax(rmax(Z, Z1), 1.0);
    double fmin = r_f_eval<FAST>(P, Zmin, D, tau, B2, SB, S2);
    double fmax = r_f_eval<FAST>(P, Zmax, D, tau, B2, SB, S2);
    for (int it = 0; it < 40; ++it) {
        if (fmin * fmax <= 0.0) break;
        Zmax *= 2.0;
        fmax = r_f_eval<FAST>(P, Zmax, D, tau, B2, SB, S2);
    }
    if (fmin * fmax <= 0.0) {
        const double tol = 1e-10 * rmax(1.0, tau);
        for (int it = 0; it < 60; ++it) {
            double Zmid = 0.5 * (Zmin + Zmax);
            double fmid = r_f_eval<FAST>(P, Zmid, D, tau, B2, SB, S2);
            if (fabs(fmid) < tol) { Z = Zmid; break; }
            if (fmin * fmid <= 0.0) { Zmax = Zmid; fmax = fmid; }
            else { Zmin = Zmid; fmin = fmid; }
            Z = 0.5 * (Zmin + Zmax);
        }
    }
}

// Hydro initial guess and the two Newton starting points Z0, Z1
AHD void r_c2p_start(const Phys<double>& P, const double* U, double* q0, double& Z0,
                     double& Z1) {
    const double G = P.gamma, SM = 1e-12;
    double D = U[0], tau = U[4];
    double B2 = U[5] * U[5] + U[6] * U[6] + U[7] * U[7];
    double tau_h = tau - 0.5 * B2;
    if (tau_h < SM) tau_h = SM;
    r_c2p_hydro(P, D, U[1], U[2], U[3], tau_h, q0);
    double v20 = q0[1] * q0[1] + q0[2] * q0[2] + q0[3] * q0[3];
    if (v20 >= P.v_max * P.v_max) v20 = P.v_max * P.v_max - 1e-14;
    double W0 = 1.0 / sqrt(1.0 - v20);
    double h0 = 1.0 + G / (G - 1.0) * q0[4] / rmax(q0[0], SM);
    Z0 = rmax(q0[0] * h0 * W0 * W0, SM);
    Z1 = rmax(D + tau + B2, SM);
}

// f(Z) of the reference's con2prim equation (the same arithmetic as
// r_f_of_Z) and, when df is non-null, its analytic derivative from the same
// intermediates: v^2 = A / Bq with A = S^2 + (S.B)^2 (2Z + B^2) / Z^2 and
// Bq = (Z + B^2)^2, W^2 = 1 / (1 - v^2), rho = D / W, p = (G-1)/G (Z / W^2 - rho),
// b^2 = B^2 / W^2 + (S.B / Z)^2.  Where the reference clamps v^2 or p the
// clamped quantity is constant and contributes nothing.
AHD double r_f_df_of_Z(const Phys<double>& P, double Z, double D, double tau, double B2,
                       double SB, double S2, double* df, double tol) {
    // the reference's divisions regrouped: one division (1/Z and
    // 1/(Z+B^2)^2 from their product), one reciprocal square root (W), and
    // p = (G-1)/G (Z / W^2 - rho), the reference's (h - 1) rho (G-1)/G with
    // h = Z / (rho W^2) written without a quotient: the same residual to
    // rounding, far inside the Newton tolerance
    const double G = P.gamma, SM = 1e-12;
    const double Zf = rmax(Z, SM);
    const double ZpB = Z + B2;
    const double Bq = ZpB * ZpB + SM;
    // 1/Z and 1/(Z+B^2)^2 from one division (of their product), unless the
    // product leaves the float64 range
    double iZ, iBq;
    const double ZB = Zf * Bq;
    if (ZB < 1e300) {
        const double t = rcp_nr(ZB);
        iZ = t * Bq;
        iBq = t * Zf;
    } else {
        iZ = 1.0 / Zf;
        iBq = 1.0 / Bq;
    }
    const double vb = SB * iZ;
    double v2 = (S2 + (SB * SB) * (2.0 * Z + B2) * (iZ * iZ)) * iBq;
    const double vmax2 = P.v_max * P.v_max;
    const bool vcap = v2 >= vmax2;
    if (vcap) v2 = vmax2 - 1e-14;
    const double om = 1.0 - v2;  // 1 / W^2 >= 1 - v_max^2 > 0
    const double W = rsqrt(om);
    const double W2 = W * W;
    const double rho = D * (om * W);  // D / W, W >= 1
    const double gm = (G - 1.0) / G;
    // (h - 1) rho with h = Z / (rho W^2) is Z / W^2 - rho: no division
    double p = (Z * om - rho) * gm;
    bool pcap = false;
    if (p < SM) { p = SM; pcap = true; }
    if (p > P.p_max) { p = P.p_max; pcap = true; }
    const double b2 = B2 * om + vb * vb;
    const double f = (Z - p + 0.5 * B2 + 0.5 * b2 - D) - tau;
    // |f| < tol: the caller stops here, the derivative is not needed
    if (df && !(fabs(f) < tol)) {
        const bool zfloor = Z < SM;
        const double dA = zfloor ? 0.0 : -2.0 * SB * SB * ZpB * (iZ * iZ * iZ);
        const double dv2 = vcap ? 0.0 : (dA - v2 * 2.0 * ZpB) * iBq;
        const double dW2 = W2 * W2 * dv2;
        const double om2 = om * om;
        const double drho = -0.5 * rho * dW2 * om;  // rho = D W2^-1/2
        const double dp = pcap ? 0.0 : gm * (om - Z * dW2 * om2 - drho);
        const double dvb = zfloor ? 0.0 : -vb * iZ;
        const double db2 = -B2 * dW2 * om2 + 2.0 * vb * dvb;
        *df = 1.0 - dp + 0.5 * db2;
    }
    return f;
}

// At most max_steps Newton steps on the reference's con2prim equation with its
// +-Z/2 step clamp and Z floor, the derivative analytic (r_f_df_of_Z: one
// evaluation per step instead of the reference's two for a forward
// difference), testing |f| < 1e-10 max(1, tau) before each step and after
// the last.  *steps = steps taken when converged.  The converged Z meets the
// reference's own criterion, so the result agrees with the reference's to
// its tolerance.
AHD bool r_newton_polish(const Phys<double>& P, double& Z, int max_steps, double D, double tau,
                         double B2, double SB, double S2, int* steps) {
    const double tol = 1e-10 * rmax(1.0, tau);
    for (int s = 0;; ++s) {
        double dfdZ = 0.0;
        const double f =
            r_f_df_of_Z(P, Z, D, tau, B2, SB, S2, s < max_steps ? &dfdZ : nullptr, tol);
        if (fabs(f) < tol) {
            *steps = s;
            return true;
        }
        if (s == max_steps) break;
        if (dfdZ == 0.0 || !isfinite(dfdZ)) break;
        double dZ = -f * rcp_nr(dfdZ);
        if (dZ > 0.5 * Z) dZ = 0.5 * Z;
        if (dZ < -0.5 * Z) dZ = -0.5 * Z;
        Z += dZ;
        if (Z < 1e-12) Z = 1e-12;
    }
    *steps = max_steps;
    return false;
}

// The same polish with a second start Zb: unless the first start's Newton
// step |f / f'| is already under 1e-2 of Z (the start is next to a root; on
// jet states that holds for 99.6 % of cells, so whole warps skip the second
// evaluation), f and f' are evaluated at Zb too and the iteration continues
// from the start with the shorter first step (a start that meets the
// tolerance ends it at once; a start with f' zero or not finite loses).  Z
// holds the first start on entry and the result on return; steps are counted
// as r_newton_polish counts them.
AHD bool r_newton_polish2(const Phys<double>& P, double& Z, double Zb, int max_steps, double D,
                          double tau, double B2, double SB, double S2, int* steps) {
    const double tol = 1e-10 * rmax(1.0, tau);
    double df = 0.0;
    double f = r_f_df_of_Z(P, Z, D, tau, B2, SB, S2, max_steps > 0 ? &df : nullptr, tol);
    *steps = 0;
    if (fabs(f) < tol) return true;
    const bool a_ok = isfinite(f) && isfinite(df) && df != 0.0;
    if (!(a_ok && fabs(f) < 1e-2 * Z * fabs(df))) {
        double dfb = 0.0;
        const double fb = r_f_df_of_Z(P, Zb, D, tau, B2, SB, S2, max_steps > 0 ? &dfb : nullptr, tol);
        if (fabs(fb) < tol) {
            Z = Zb;
            return true;
        }
        const bool b_ok = isfinite(fb) && isfinite(dfb) && dfb != 0.0;
        // |fb / dfb| < |f / df| without the two divisions
        if (b_ok && (!a_ok || fabs(fb) * fabs(df) < fabs(f) * fabs(dfb))) {
            Z = Zb;
            f = fb;
            df = dfb;
        }
    }
    for (int s = 1; s <= max_steps; ++s) {
        if (df == 0.0 || !isfinite(df)) break;
        double dZ = -f * rcp_nr(df);
        if (dZ > 0.5 * Z) dZ = 0.5 * Z;
        if (dZ < -0.5 * Z) dZ = -0.5 * Z;
        Z += dZ;
        if (Z < 1e-12) Z = 1e-12;
        f = r_f_df_of_Z(P, Z, D, tau, B2, SB, S2, s < max_steps ? &df : nullptr, tol);
        if (fabs(f) < tol) {
            *steps = s;
            return true;
        }
    }
    *steps = max_steps;
    return false;
}

// Primitives from a converged Z (rmhd_core.py:320-341) without the hydro
// fallback: returns false when the result is invalid (the caller then runs
// the reference's full con2prim, which owns that fallback).
AHD bool r_prims_from_Z_checked(const Phys<double>& P, double Z, const double* U, double* q) {
    const double G = P.gamma, SM = 1e-12;
    double Sx = U[1], Sy = U[2], Sz = U[3], D = U[0];
    double Bx = U[5], By = U[6], Bz = U[7];
    double B2 = Bx * Bx + By * By + Bz * Bz;
    double SB = Sx * Bx + Sy * By + Sz * Bz;
    // divisions regrouped as in r_f_df_of_Z (same values to rounding): 1/Z
    // and 1/(Z+B^2) from one division unless their product leaves the range
    double ZpB = Z + B2;
    const double Zf = rmax(Z, SM), ZBf = rmax(ZpB, SM);
    double iZ, iZB;
    if (Zf * ZBf < 1e300) {
        const double t = rcp_nr(Zf * ZBf);
        iZ = t * ZBf;
        iZB = t * Zf;
    } else {
        iZ = 1.0 / Zf;
        iZB = 1.0 / ZBf;
    }
    double vb = SB * iZ;
    double vx = (Sx + vb * Bx) * iZB;
    double vy = (Sy + vb * By) * iZB;
    double vz = (Sz + vb * Bz) * iZB;
    double v2 = vx * vx + vy * vy + vz * vz;
    double vmax2 = P.v_max * P.v_max;
    if (v2 >= vmax2) {
        double fac = P.v_max / sqrt(v2 + 1e-32);
        vx *= fac; vy *= fac; vz *= fac;
    }
    const double om = 1.0 - (vx * vx + vy * vy + vz * vz);  // 1 / W^2
    const double W = rsqrt(om);
    double rho = D * (om * W);                               // D / W, W >= 1
    // (h - 1) rho with h = Z / (rho W^2) is Z / W^2 - rho: no division
    double p = (Z * om - rho) * ((G - 1.0) / G);
    if (!isfinite(rho) || !isfinite(p) || rho <= 0.0 || p <= 0.0) return false;
    q[0] = rho; q[1] = vx; q[2] = vy; q[3] = vz; q[4] = p;
    q[5] = Bx; q[6] = By; q[7] = Bz; q[8] = U[8];
    floor_prim(P, q);
    return true;
}

// Full reference con2prim (cons_to_prim_rmhd, rmhd_core.py:249-341); FAST:
// its f(Z) and primitive recovery with the regrouped divisions (the learned
// path's fallback), otherwise the reference's operation order
template <bool FAST = false>
AHD void r_c2p(const Phys<double>& P, const double* U, double* q, C2PCount& cnt) {
    double D = U[0], tau = U[4];
    double B2 = U[5] * U[5] + U[6] * U[6] + U[7] * U[7];
    double SB = U[1] * U[5] + U[2] * U[6] + U[3] * U[7];
    double S2 = U[1] * U[1] + U[2] * U[2] + U[3] * U[3];
    double q0[5], Z0, Z1;
    r_c2p_start(P, U, q0, Z0, Z1);
    double Z = Z0;
    bool ok = r_newton<FAST>(P, Z, 50, D, tau, B2, SB, S2);
    if (!ok) {
        Z = Z1;
        ok = r_newton<FAST>(P, Z, 50, D, tau, B2, SB, S2);
    }
    if (ok) cnt.newton++;
    else {
        cnt.bisect++;
        r_bisect<FAST>(P, Z, Z1, D, tau, B2, SB, S2);
    }
    r_prims_from_Z<FAST>(P, Z, U, q0, q, cnt);
}

}  // namespace astro
