/*
 * astro_oracle.c -- CPU restatement of AstroFD's per-step finite-volume
 * right-hand side, written in plain C as the parity oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the astrofd_b200 product links,
 * imports or calls this file.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py use it, and only as the checker
 * or as the timed CPU baseline.
 *
 * It restates, loop for loop and quirk for quirk, the reference's Numba
 * kernels (paths relative to the AstroFD checkout):
 *   core/srhd_core.py   prim_to_cons :47, cons_to_prim :62, sound_speed :134,
 *                       eig_speeds :143, flux_x/y/z :157-169, hlle :172,
 *                       hllc_flux_x/y/z :189-282, minmod/mc_lim :306,314,
 *                       ppm_reconstruct :328, weno5_left/right :344,362,
 *                       floor_prim :380, compute_rhs_muscl :469,
 *                       compute_rhs_ppm :927, compute_rhs_weno :1167,
 *                       max_char_speed :1268, step_ssprk2/3 :1286,1334
 *   core/rmhd_core.py   limiter :61, floor_prim_rmhd :126,
 *                       prim_to_cons_rmhd :138, _cons_to_prim_hydro :171,
 *                       rmhd_f_of_Z :229, cons_to_prim_rmhd :249,
 *                       flux_rmhd_x/y/z :344-395, hlle :403,
 *                       rmhd_fast_speed :420, rmhd_eig_speeds :460,
 *                       hllc_hydro_flux_* :474-567, riemann_flux_rmhd_* :570,727,738,
 *                       hllc_contact_speed_* :581-599, hll_d_flux_dir :602,
 *                       compute_rhs_rmhd :749, compute_rhs_ppm :1280,
 *                       compute_rhs_weno :1440, step_ssprk2/3 :1559,1609
 *   core/boundary.py    apply_periodic_yz :4, apply_outflow_right_x :10
 *   core/nozzle.py      nozzle_weight :5, apply_nozzle_left_x :27
 *   core/source_terms.py apply_cooling_heating :5, apply_two_temperature :30
 *
 * Array layout: pr[v][i][j][k], C-contiguous float64, k fastest, extents
 * (nv, nx, ny, nz) including ghosts -- the reference's own layout.
 */
#include <math.h>
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define SMALL 1e-12

typedef struct {
    int physics;        /* 0 = SRHD, 1 = RMHD                               */
    int recon;          /* 0 = muscl, 1 = ppm, 2 = weno                     */
    int limiter;        /* 0 = mc, 1 = minmod, 2 = vanleer                  */
    int riemann;        /* SRHD 0 hlle 1 hllc; RMHD 0 hlle 1 hlld 2 hlld_full */
    int n_passive;
    int passive_offset;
    int resistive;
    int flux_mode;      /* 0 = the reference's own arithmetic; 1 = each RMHD
                           PPM/WENO x face with its own speeds and the
                           resistive term applied once for every recon      */
    double gamma;       /* RMHD gamma; SRHD kernels always use 5/3 (quirk)  */
    double p_max, v_max, glm_ch, glm_cp, resistivity;
} OParams;

typedef struct { int nv, nx, ny, nz; } OGrid;

static inline size_t IX(const OGrid* g, int v, int i, int j, int k) {
    return (((size_t)v * g->nx + i) * g->ny + j) * g->nz + k;
}
#define P(v, i, j, k) pr[IX(g, (v), (i), (j), (k))]

/* Passive stencils in the MUSCL right-hand sides reach i-3 / i+3 although the
 * loop bounds only guarantee +-2.  Numba wraps negative indices per axis and
 * does not bound-check positive ones, so an index n aliases the next row of
 * the C-contiguous block (core/srhd_core.py:550-560, core/rmhd_core.py:832-940).
 * This restates that addressing; a read past the end of the block is
 * undefined in the reference and returns NaN here. */
static inline double pget(const OGrid* g, const double* pr, int v, int i, int j, int k) {
    if (i < 0) i += g->nx;
    if (j < 0) j += g->ny;
    if (k < 0) k += g->nz;
    size_t flat = (((size_t)v * g->nx + i) * g->ny + j) * g->nz + k;
    size_t total = (size_t)g->nv * g->nx * g->ny * g->nz;
    if (flat >= total) return NAN;
    return pr[flat];
}

static inline double dmax(double a, double b) { return a > b ? a : b; }
static inline double dmin(double a, double b) { return a < b ? a : b; }

/* ------------------------------------------------------------------ */
/* reconstruction (srhd_core.py:306-378, rmhd_core.py:53-124)          */
/* ------------------------------------------------------------------ */
static double minmod(double a, double b) {
    if (a * b <= 0.0) return 0.0;
    return fabs(a) < fabs(b) ? a : b;
}

static double limiter(int id, double dqL, double dqR) {
    if (id == 1) return minmod(dqL, dqR);
    if (id == 2) {
        if (dqL * dqR <= 0.0) return 0.0;
        double denom = dqL + dqR;
        if (denom == 0.0) return 0.0;
        return (2.0 * dqL * dqR) / denom;
    }
    double mm = minmod(dqL, dqR);
    return minmod(0.5 * (dqL + dqR), 2.0 * mm);
}

static void ppm(double q_im2, double q_im1, double q_i, double q_ip1, double q_ip2,
                double* oL, double* oR) {
    double qL = (7.0 / 12.0) * (q_im1 + q_i) - (1.0 / 12.0) * (q_im2 + q_ip1);
    double qR = (7.0 / 12.0) * (q_i + q_ip1) - (1.0 / 12.0) * (q_im1 + q_ip2);
    double qmax = dmax(dmax(q_im1, q_i), q_ip1);
    double qmin = dmin(dmin(q_im1, q_i), q_ip1);
    if (qL > qmax) qL = qmax;
    if (qL < qmin) qL = qmin;
    if (qR > qmax) qR = qmax;
    if (qR < qmin) qR = qmin;
    if ((qR - q_i) * (q_i - qL) <= 0.0) { qL = q_i; qR = q_i; }
    *oL = qL; *oR = qR;
}

static double weno5(double a, double b, double c, double d, double e) {
    /* weno5_left(a..e) == weno5_right with the stencil reversed */
    const double eps = 1e-12;
    double t0 = a - 2.0 * b + c, u0 = a - 4.0 * b + 3.0 * c;
    double t1 = b - 2.0 * c + d, u1 = b - d;
    double t2 = c - 2.0 * d + e, u2 = 3.0 * c - 4.0 * d + e;
    double IS0 = (13.0 / 12.0) * (t0 * t0) + 0.25 * (u0 * u0);
    double IS1 = (13.0 / 12.0) * (t1 * t1) + 0.25 * (u1 * u1);
    double IS2 = (13.0 / 12.0) * (t2 * t2) + 0.25 * (u2 * u2);
    double a0 = 0.1 / ((eps + IS0) * (eps + IS0));
    double a1 = 0.6 / ((eps + IS1) * (eps + IS1));
    double a2 = 0.3 / ((eps + IS2) * (eps + IS2));
    double s = a0 + a1 + a2;
    double w0 = a0 / s, w1 = a1 / s, w2 = a2 / s;
    double p0 = (1.0 / 3.0) * a - (7.0 / 6.0) * b + (11.0 / 6.0) * c;
    double p1 = (-1.0 / 6.0) * b + (5.0 / 6.0) * c + (1.0 / 3.0) * d;
    double p2 = (1.0 / 3.0) * c + (5.0 / 6.0) * d - (1.0 / 6.0) * e;
    return w0 * p0 + w1 * p1 + w2 * p2;
}

static inline double hlle_scalar(double qL, double qR, double fL, double fR,
                                 double sL, double sR) {
    if (sL >= 0.0) return fL;
    if (sR <= 0.0) return fR;
    return (sR * fL - sL * fR + sL * sR * (qR - qL)) / (sR - sL + SMALL);
}

static void hlle_vec(int n, const double* UL, const double* UR, const double* FL,
                     const double* FR, double sL, double sR, double* out) {
    if (sL >= 0.0) { memcpy(out, FL, n * sizeof(double)); return; }
    if (sR <= 0.0) { memcpy(out, FR, n * sizeof(double)); return; }
    for (int v = 0; v < n; ++v)
        out[v] = (sR * FL[v] - sL * FR[v] + sL * sR * (UR[v] - UL[v])) / (sR - sL + SMALL);
}

static void eig_speeds(double vn, double cs, double* lm, double* lp) {
    double dp = 1.0 + vn * cs, dm = 1.0 - vn * cs;
    if (dp == 0.0) dp = SMALL;
    if (dm == 0.0) dm = SMALL;
    double p = (vn + cs) / dp, m = (vn - cs) / dm;
    if (p > 1.0) p = 1.0;
    if (p < -1.0) p = -1.0;
    if (m > 1.0) m = 1.0;
    if (m < -1.0) m = -1.0;
    *lm = m; *lp = p;
}

/* ------------------------------------------------------------------ */
/* SRHD (gamma always 5/3: default argument frozen at import,          */
/* srhd_core.py:47,62,134)                                             */
/* ------------------------------------------------------------------ */
#define SRHD_GAMMA (5.0 / 3.0)

static void s_p2c(const double* q, double* U) {
    const double gamma = SRHD_GAMMA;
    double rho = q[0], vx = q[1], vy = q[2], vz = q[3], p = q[4];
    double v2 = vx * vx + vy * vy + vz * vz;
    if (v2 >= 1.0) v2 = 1.0 - 1e-14;
    double W = 1.0 / sqrt(1.0 - v2);
    double h = 1.0 + gamma / (gamma - 1.0) * p / dmax(rho, SMALL);
    double w = rho * h;
    U[0] = rho * W;
    U[1] = w * W * W * vx;
    U[2] = w * W * W * vy;
    U[3] = w * W * W * vz;
    U[4] = w * W * W - p - U[0];
}

static void s_c2p(const OParams* pa, const double* U, double* q) {
    const double gamma = SRHD_GAMMA;
    double D = U[0], Sx = U[1], Sy = U[2], Sz = U[3], tau = U[4];
    double E = tau + D;
    double S2 = Sx * Sx + Sy * Sy + Sz * Sz;
    double p = (gamma - 1.0) * (E - D);
    if (p < SMALL) p = SMALL;
    if (p > pa->p_max) p = pa->p_max;
    int ok = 0;
    for (int it = 0; it < 60; ++it) {
        double Wm = E + p;
        double v2 = S2 / (Wm * Wm + SMALL);
        if (v2 >= pa->v_max * pa->v_max) v2 = pa->v_max * pa->v_max - 1e-14;
        double W = 1.0 / sqrt(1.0 - v2);
        double rho = D / dmax(W, SMALL);
        double h = 1.0 + gamma / (gamma - 1.0) * p / dmax(rho, SMALL);
        double w = rho * h;
        double f = Wm - w * W * W;
        double dp = -f / 1.0;
        if (dp > 0.5 * p) dp = 0.5 * p;
        if (dp < -0.5 * p) dp = -0.5 * p;
        double pn = p + dp;
        if (pn < SMALL) pn = SMALL;
        if (pn > pa->p_max) pn = pa->p_max;
        if (fabs(dp) < 1e-12 * dmax(1.0, pn)) { p = pn; ok = 1; break; }
        p = pn;
    }
    if (!ok) {
        p = (gamma - 1.0) * (E - D);
        if (p < SMALL) p = SMALL;
        if (p > pa->p_max) p = pa->p_max;
    }
    double Wm = E + p;
    double vx = Sx / dmax(Wm, SMALL), vy = Sy / dmax(Wm, SMALL), vz = Sz / dmax(Wm, SMALL);
    double v2 = vx * vx + vy * vy + vz * vz;
    double vmax2 = pa->v_max * pa->v_max;
    if (v2 >= vmax2) {
        double fac = pa->v_max / sqrt(v2 + 1e-32);
        vx *= fac; vy *= fac; vz *= fac;
    }
    v2 = vx * vx + vy * vy + vz * vz;
    if (v2 >= 1.0) v2 = 1.0 - 1e-14;
    double W = 1.0 / sqrt(1.0 - v2);
    double rho = D / dmax(W, SMALL);
    if (rho < SMALL) rho = SMALL;
    if (p < SMALL) p = SMALL;
    if (p > pa->p_max) p = pa->p_max;
    q[0] = rho; q[1] = vx; q[2] = vy; q[3] = vz; q[4] = p;
}

static double s_sound_speed(double rho, double p) {
    const double gamma = SRHD_GAMMA;
    double h = 1.0 + gamma / (gamma - 1.0) * p / dmax(rho, SMALL);
    double w = rho * h;
    double cs2 = gamma * p / dmax(w, SMALL);
    if (cs2 < 0.0) cs2 = 0.0;
    if (cs2 > 1.0 - 1e-14) cs2 = 1.0 - 1e-14;
    return sqrt(cs2);
}

static void s_floor(const OParams* pa, double* q) {
    if (q[0] < SMALL) q[0] = SMALL;
    if (q[4] < SMALL) q[4] = SMALL;
    if (q[4] > pa->p_max) q[4] = pa->p_max;
    double v2 = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    double vmax2 = pa->v_max * pa->v_max;
    if (v2 >= vmax2) {
        double fac = pa->v_max / sqrt(v2 + 1e-32);
        q[1] *= fac; q[2] *= fac; q[3] *= fac;
    }
}

static void s_flux(int n, const double* q, double* F) {
    double U[5];
    s_p2c(q, U);
    double vn = q[1 + n], p = q[4];
    F[0] = U[0] * vn;
    for (int m = 0; m < 3; ++m) F[1 + m] = (m == n) ? U[1 + m] * vn + p : U[1 + m] * vn;
    F[4] = (U[4] + p) * vn;
}

/* HLLC for SRHD and the hydro part of RMHD "hlld" (srhd_core.py:189-282,
 * rmhd_core.py:474-567); direction n selects the normal momentum. */
static void hllc5(int n, const double* UL, const double* UR, const double* FL,
                  const double* FR, double sL, double sR, double pL, double pR,
                  double vL, double vR, double* out) {
    double DL = UL[0], DR = UR[0];
    double SnL = UL[1 + n], SnR = UR[1 + n];
    double denom = (DL * (sL - vL) - DR * (sR - vR)) + SMALL;
    double sM = (pR - pL + SnL * (sL - vL) - SnR * (sR - vR)) / denom;
    double pStar = 0.5 * (pL + pR + DL * (sL - vL) * (sM - vL) + DR * (sR - vR) * (sM - vR));
    if (sL >= 0.0) { memcpy(out, FL, 5 * sizeof(double)); return; }
    if (sR <= 0.0) { memcpy(out, FR, 5 * sizeof(double)); return; }
    double Ust[5];
    if (sM >= 0.0) {
        double fac = (sL - vL) / (sL - sM + SMALL);
        Ust[0] = DL * fac;
        for (int m = 0; m < 3; ++m)
            Ust[1 + m] = (m == n) ? UL[1 + m] * fac + (pStar - pL) / (sL - sM + SMALL)
                                  : UL[1 + m] * fac;
        Ust[4] = UL[4] * fac + (pStar * sM - pL * vL) / (sL - sM + SMALL);
        for (int v = 0; v < 5; ++v) out[v] = FL[v] + sL * (Ust[v] - UL[v]);
    } else {
        double fac = (sR - vR) / (sR - sM + SMALL);
        Ust[0] = DR * fac;
        for (int m = 0; m < 3; ++m)
            Ust[1 + m] = (m == n) ? UR[1 + m] * fac + (pStar - pR) / (sR - sM + SMALL)
                                  : UR[1 + m] * fac;
        Ust[4] = UR[4] * fac + (pStar * sM - pR * vR) / (sR - sM + SMALL);
        for (int v = 0; v < 5; ++v) out[v] = FR[v] + sR * (Ust[v] - UR[v]);
    }
}

static double contact_speed(int n, const double* UL, const double* UR, double sL,
                            double sR, double pL, double pR, double vL, double vR) {
    double denom = (UL[0] * (sL - vL) - UR[0] * (sR - vR)) + SMALL;
    return (pR - pL + UL[1 + n] * (sL - vL) - UR[1 + n] * (sR - vR)) / denom;
}

typedef struct { double F[9]; double sL, sR, vL, vR; } Face;

/* Israel-Stewart dissipation flux of one cell added to a face flux
 * (add_diss_flux_x/y/z, srhd_core.py:417-442): is = pi, pixx, piyy, pizz,
 * pixy, pixz, piyz, qx, qy, qz of the cell, q the face primitives after the
 * floor.  Row n of the stress: pi delta_nm + pi^nm; energy: v.row + q_n. */
static void s_diss_flux(int n, const double* q, const double* is, double* F) {
    static const int S[3][3] = {{1, 4, 5}, {4, 2, 6}, {5, 6, 3}};
    double row[3];
    for (int m = 0; m < 3; ++m) row[m] = (m == n) ? is[0] + is[S[n][m]] : is[S[n][m]];
    for (int m = 0; m < 3; ++m) F[1 + m] += row[m];
    F[4] += q[1] * row[0] + q[2] * row[1] + q[3] * row[2] + is[7 + n];
}

/* One SRHD face from reconstructed left/right primitives: floor, p2c, flux,
 * (ndiss times the dissipation fluxes of the cells isL / isR), speeds,
 * Riemann (the repeated block of srhd_core.py:517-550 etc.). */
static void s_face_is(const OParams* pa, int n, double* qL, double* qR, int ndiss,
                      const double* isL, const double* isR, Face* f) {
    double UL[5], UR[5], FL[5], FR[5], lmL, lpL, lmR, lpR;
    s_floor(pa, qL);
    s_floor(pa, qR);
    s_p2c(qL, UL);
    s_p2c(qR, UR);
    s_flux(n, qL, FL);
    s_flux(n, qR, FR);
    for (int rep = 0; rep < ndiss; ++rep) {
        s_diss_flux(n, qL, isL, FL);
        s_diss_flux(n, qR, isR, FR);
    }
    double csL = s_sound_speed(qL[0], qL[4]), csR = s_sound_speed(qR[0], qR[4]);
    eig_speeds(qL[1 + n], csL, &lmL, &lpL);
    eig_speeds(qR[1 + n], csR, &lmR, &lpR);
    double sL = dmin(lmL, lmR), sR = dmax(lpL, lpR);
    if (pa->riemann == 1)
        hllc5(n, UL, UR, FL, FR, sL, sR, qL[4], qR[4], qL[1 + n], qR[1 + n], f->F);
    else
        hlle_vec(5, UL, UR, FL, FR, sL, sR, f->F);
    f->sL = sL; f->sR = sR; f->vL = qL[1 + n]; f->vR = qR[1 + n];
}

static void s_face(const OParams* pa, int n, double* qL, double* qR, Face* f) {
    s_face_is(pa, n, qL, qR, 0, NULL, NULL, f);
}

/* ------------------------------------------------------------------ */
/* RMHD (rmhd_core.py)                                                  */
/* ------------------------------------------------------------------ */
static void r_floor(const OParams* pa, double* q) {
    if (q[0] < SMALL) q[0] = SMALL;
    if (q[4] < SMALL) q[4] = SMALL;
    if (q[4] > pa->p_max) q[4] = pa->p_max;
    double v2 = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    double vmax2 = pa->v_max * pa->v_max;
    if (v2 >= vmax2) {
        double fac = pa->v_max / sqrt(v2 + 1e-32);
        q[1] *= fac; q[2] *= fac; q[3] *= fac;
    }
}

static void r_p2c(const OParams* pa, const double* qin, double* U) {
    const double gamma = pa->gamma;
    double rho = qin[0], vx = qin[1], vy = qin[2], vz = qin[3], p = qin[4];
    double Bx = qin[5], By = qin[6], Bz = qin[7], psi = qin[8];
    double v2 = vx * vx + vy * vy + vz * vz;
    double vmax2 = pa->v_max * pa->v_max;
    if (v2 >= vmax2) {
        double fac = pa->v_max / sqrt(v2 + 1e-32);
        vx *= fac; vy *= fac; vz *= fac;
    }
    if (p < SMALL) p = SMALL;
    if (p > pa->p_max) p = pa->p_max;
    double B2 = Bx * Bx + By * By + Bz * Bz;
    double W = 1.0 / sqrt(1.0 - (vx * vx + vy * vy + vz * vz));
    double h = 1.0 + gamma / (gamma - 1.0) * p / dmax(rho, SMALL);
    double rhoh = rho * h;
    double vb = vx * Bx + vy * By + vz * Bz;
    double b0 = W * vb;
    double bx = (Bx + b0 * vx) / W, by = (By + b0 * vy) / W, bz = (Bz + b0 * vz) / W;
    double b2 = (bx * bx + by * by + bz * bz) - b0 * b0;
    double wtot = rhoh * W * W + B2;
    double D = rho * W;
    U[0] = D;
    U[1] = wtot * vx - (Bx * vb);
    U[2] = wtot * vy - (By * vb);
    U[3] = wtot * vz - (Bz * vb);
    U[4] = rhoh * W * W - p + 0.5 * B2 + 0.5 * b2 - D;
    U[5] = Bx; U[6] = By; U[7] = Bz; U[8] = psi;
}

static void r_c2p_hydro(const OParams* pa, double D, double Sx, double Sy, double Sz,
                        double tau, double* q) {
    const double gamma = pa->gamma;
    double E = tau + D;
    double S2 = Sx * Sx + Sy * Sy + Sz * Sz;
    double p = (gamma - 1.0) * (E - D);
    if (p < SMALL) p = SMALL;
    if (p > pa->p_max) p = pa->p_max;
    int ok = 0;
    for (int it = 0; it < 60; ++it) {
        double Wm = E + p;
        double v2 = S2 / (Wm * Wm + SMALL);
        if (v2 >= pa->v_max * pa->v_max) v2 = pa->v_max * pa->v_max - 1e-14;
        double W = 1.0 / sqrt(1.0 - v2);
        double rho = D / dmax(W, SMALL);
        double h = 1.0 + gamma / (gamma - 1.0) * p / dmax(rho, SMALL);
        double w = rho * h;
        double f = Wm - w * W * W;
        double dp = -f / 1.0;
        if (dp > 0.5 * p) dp = 0.5 * p;
        if (dp < -0.5 * p) dp = -0.5 * p;
        double pn = p + dp;
        if (pn < SMALL) pn = SMALL;
        if (pn > pa->p_max) pn = pa->p_max;
        if (fabs(dp) < 1e-12 * dmax(1.0, pn)) { p = pn; ok = 1; break; }
        p = pn;
    }
    if (!ok) {
        p = (gamma - 1.0) * (E - D);
        if (p < SMALL) p = SMALL;
        if (p > pa->p_max) p = pa->p_max;
    }
    double Wm = E + p;
    double vx = Sx / dmax(Wm, SMALL), vy = Sy / dmax(Wm, SMALL), vz = Sz / dmax(Wm, SMALL);
    double v2 = vx * vx + vy * vy + vz * vz;
    double vmax2 = pa->v_max * pa->v_max;
    if (v2 >= vmax2) {
        double fac = pa->v_max / sqrt(v2 + 1e-32);
        vx *= fac; vy *= fac; vz *= fac;
    }
    v2 = vx * vx + vy * vy + vz * vz;
    if (v2 >= 1.0) v2 = 1.0 - 1e-14;
    double W = 1.0 / sqrt(1.0 - v2);
    double rho = D / dmax(W, SMALL);
    if (rho < SMALL) rho = SMALL;
    if (p < SMALL) p = SMALL;
    if (p > pa->p_max) p = pa->p_max;
    q[0] = rho; q[1] = vx; q[2] = vy; q[3] = vz; q[4] = p;
}

static double r_f_of_Z(const OParams* pa, double Z, double D, double tau, double B2,
                       double SB, double S2) {
    const double G = pa->gamma;
    double denomZ = dmax(Z, SMALL);
    double vb = SB / denomZ;
    double ZpB = Z + B2;
    double v2 = (S2 + (SB * SB) * (2.0 * Z + B2) / (denomZ * denomZ)) / (ZpB * ZpB + SMALL);
    double vmax2 = pa->v_max * pa->v_max;
    if (v2 >= vmax2) v2 = vmax2 - 1e-14;
    double W2 = 1.0 / (1.0 - v2);
    double W = sqrt(W2);
    double rho = D / dmax(W, SMALL);
    double h = Z / dmax(rho * W2, SMALL);
    double p = (h - 1.0) * rho * (G - 1.0) / G;
    if (p < SMALL) p = SMALL;
    if (p > pa->p_max) p = pa->p_max;
    double b2 = B2 / W2 + vb * vb;
    double tau_calc = Z - p + 0.5 * B2 + 0.5 * b2 - D;
    return tau_calc - tau;
}

/* Counters of the con2prim paths taken (converged by Newton, bisection,
 * invalid -> hydro fallback), summed over calls since the last reset. */
static long g_c2p_newton = 0, g_c2p_bisect = 0, g_c2p_hydro_fallback = 0;

static void r_c2p(const OParams* pa, const double* U, double* q) {
    const double G = pa->gamma;
    double D = U[0], Sx = U[1], Sy = U[2], Sz = U[3], tau = U[4];
    double Bx = U[5], By = U[6], Bz = U[7], psi = U[8];
    double B2 = Bx * Bx + By * By + Bz * Bz;
    double SB = Sx * Bx + Sy * By + Sz * Bz;
    double S2 = Sx * Sx + Sy * Sy + Sz * Sz;
    double tau_h = tau - 0.5 * B2;
    if (tau_h < SMALL) tau_h = SMALL;
    double q0[5];
    r_c2p_hydro(pa, D, Sx, Sy, Sz, tau_h, q0);
    double v20 = q0[1] * q0[1] + q0[2] * q0[2] + q0[3] * q0[3];
    if (v20 >= pa->v_max * pa->v_max) v20 = pa->v_max * pa->v_max - 1e-14;
    double W0 = 1.0 / sqrt(1.0 - v20);
    double h0 = 1.0 + G / (G - 1.0) * q0[4] / dmax(q0[0], SMALL);
    double Z0 = dmax(q0[0] * h0 * W0 * W0, SMALL);
    double Z1 = dmax(D + tau + B2, SMALL);
    int ok = 0;
    double Z = Z0;
    for (int attempt = 0; attempt < 2; ++attempt) {
        if (attempt == 1) Z = Z1;
        for (int it = 0; it < 50; ++it) {
            double f = r_f_of_Z(pa, Z, D, tau, B2, SB, S2);
            if (fabs(f) < 1e-10 * dmax(1.0, tau)) { ok = 1; break; }
            double eps = 1e-6 * dmax(1.0, Z);
            double fp = r_f_of_Z(pa, Z + eps, D, tau, B2, SB, S2);
            double dfdZ = (fp - f) / eps;
            if (dfdZ == 0.0) break;
            double dZ = -f / dfdZ;
            if (dZ > 0.5 * Z) dZ = 0.5 * Z;
            if (dZ < -0.5 * Z) dZ = -0.5 * Z;
            Z += dZ;
            if (Z < SMALL) Z = SMALL;
        }
        if (ok) break;
    }
    if (ok) g_c2p_newton++;
    if (!ok) {
        g_c2p_bisect++;
        double Zmin = SMALL;
        double Zmax = dmax(dmax(Z, Z1), 1.0);
        double fmin = r_f_of_Z(pa, Zmin, D, tau, B2, SB, S2);
        double fmax = r_f_of_Z(pa, Zmax, D, tau, B2, SB, S2);
        for (int it = 0; it < 40; ++it) {
            if (fmin * fmax <= 0.0) break;
            Zmax *= 2.0;
            fmax = r_f_of_Z(pa, Zmax, D, tau, B2, SB, S2);
        }
        if (fmin * fmax <= 0.0) {
            for (int it = 0; it < 60; ++it) {
                double Zmid = 0.5 * (Zmin + Zmax);
                double fmid = r_f_of_Z(pa, Zmid, D, tau, B2, SB, S2);
                if (fabs(fmid) < 1e-10 * dmax(1.0, tau)) { Z = Zmid; break; }
                if (fmin * fmid <= 0.0) { Zmax = Zmid; fmax = fmid; }
                else { Zmin = Zmid; fmin = fmid; }
                Z = 0.5 * (Zmin + Zmax);
            }
        }
    }
    double ZpB = Z + B2;
    double vb = SB / dmax(Z, SMALL);
    double vx = (Sx + vb * Bx) / dmax(ZpB, SMALL);
    double vy = (Sy + vb * By) / dmax(ZpB, SMALL);
    double vz = (Sz + vb * Bz) / dmax(ZpB, SMALL);
    double v2 = vx * vx + vy * vy + vz * vz;
    double vmax2 = pa->v_max * pa->v_max;
    if (v2 >= vmax2) {
        double fac = pa->v_max / sqrt(v2 + 1e-32);
        vx *= fac; vy *= fac; vz *= fac;
    }
    double W = 1.0 / sqrt(1.0 - (vx * vx + vy * vy + vz * vz));
    double rho = D / dmax(W, SMALL);
    double h = Z / dmax(rho * W * W, SMALL);
    double p = (h - 1.0) * rho * (G - 1.0) / G;
    if (!isfinite(rho) || !isfinite(p) || rho <= 0.0 || p <= 0.0) {
        g_c2p_hydro_fallback++;
        rho = q0[0]; vx = q0[1]; vy = q0[2]; vz = q0[3]; p = q0[4];
    }
    q[0] = rho; q[1] = vx; q[2] = vy; q[3] = vz; q[4] = p;
    q[5] = Bx; q[6] = By; q[7] = Bz; q[8] = psi;
    r_floor(pa, q);
}

static void r_flux(const OParams* pa, int n, const double* q, double* F) {
    double U[9];
    r_p2c(pa, q, U);
    double vx = q[1], vy = q[2], vz = q[3], p = q[4];
    double Bx = q[5], By = q[6], Bz = q[7], psi = q[8];
    double v[3] = {vx, vy, vz}, B[3] = {Bx, By, Bz};
    double B2 = Bx * Bx + By * By + Bz * Bz;
    double pt = p + 0.5 * B2;
    double vn = v[n], Bn = B[n];
    F[0] = U[0] * vn;
    for (int m = 0; m < 3; ++m)
        F[1 + m] = (m == n) ? U[1 + m] * vn + pt - Bn * Bn : U[1 + m] * vn - Bn * B[m];
    F[4] = (U[4] + pt) * vn - (Bn * (Bx * vx + By * vy + Bz * vz));
    for (int m = 0; m < 3; ++m)
        F[5 + m] = (m == n) ? psi : v[m] * Bn - vn * B[m];
    F[8] = pa->glm_ch * pa->glm_ch * Bn;
}

static double r_fast_speed(const OParams* pa, const double* q) {
    const double G = pa->gamma;
    double rho = q[0], vx = q[1], vy = q[2], vz = q[3], p = q[4];
    double Bx = q[5], By = q[6], Bz = q[7];
    double v2 = vx * vx + vy * vy + vz * vz;
    if (v2 >= pa->v_max * pa->v_max) v2 = pa->v_max * pa->v_max - 1e-14;
    double W = 1.0 / sqrt(1.0 - v2);
    if (rho < SMALL) rho = SMALL;
    if (p < SMALL) p = SMALL;
    if (p > pa->p_max) p = pa->p_max;
    double h = 1.0 + G / (G - 1.0) * p / dmax(rho, SMALL);
    double rhoh = rho * h;
    double vb = vx * Bx + vy * By + vz * Bz;
    double b0 = W * vb;
    double bx = (Bx + b0 * vx) / W, by = (By + b0 * vy) / W, bz = (Bz + b0 * vz) / W;
    double b2 = (bx * bx + by * by + bz * bz) - b0 * b0;
    double cs2 = G * p / dmax(rhoh, SMALL);
    if (cs2 < 0.0) cs2 = 0.0;
    if (cs2 > 1.0 - 1e-14) cs2 = 1.0 - 1e-14;
    double ca2 = b2 / dmax(rhoh + b2, SMALL);
    if (ca2 < 0.0) ca2 = 0.0;
    if (ca2 > 1.0 - 1e-14) ca2 = 1.0 - 1e-14;
    double a = cs2 + ca2 - cs2 * ca2;
    double disc = a * a - 4.0 * cs2 * ca2;
    if (disc < 0.0) disc = 0.0;
    double cf2 = 0.5 * (a + sqrt(disc));
    if (cf2 < 0.0) cf2 = 0.0;
    if (cf2 > 1.0 - 1e-14) cf2 = 1.0 - 1e-14;
    return sqrt(cf2);
}

/* hll_d_flux_dir (rmhd_core.py:602-724), the experimental HLLD */
static void r_hlld_full(const OParams* pa, int n, const double* UL, const double* UR,
                        const double* FL, const double* FR, double sL, double sR,
                        double pL, double pR, double vL, double vR, double* out) {
    if (sL >= 0.0) { memcpy(out, FL, 9 * sizeof(double)); return; }
    if (sR <= 0.0) { memcpy(out, FR, 9 * sizeof(double)); return; }
    int t1 = (n == 0) ? 1 : 0, t2 = (n == 2) ? 1 : 2;
    int vt1 = 1 + t1, vt2 = 1 + t2, bn = 5 + n, bt1 = 5 + t1, bt2 = 5 + t2;
    if (UL[0] <= SMALL || UR[0] <= SMALL) { hlle_vec(9, UL, UR, FL, FR, sL, sR, out); return; }
    double BnL = UL[bn], BnR = UR[bn];
    double Bt1L = UL[bt1], Bt2L = UL[bt2], Bt1R = UR[bt1], Bt2R = UR[bt2];
    double Bn = 0.5 * (BnL + BnR);
    if (fabs(Bn) < 1e-8) { hlle_vec(9, UL, UR, FL, FR, sL, sR, out); return; }
    double sM = contact_speed(n, UL, UR, sL, sR, pL, pR, vL, vR);
    double DL = UL[0], DR = UR[0];
    double DstarL = DL * (sL - vL) / (sL - sM + SMALL);
    double DstarR = DR * (sR - vR) / (sR - sM + SMALL);
    if (DstarL <= SMALL || DstarR <= SMALL) { hlle_vec(9, UL, UR, FL, FR, sL, sR, out); return; }
    double Bt1Ls = Bt1L * (sL - vL) / (sL - sM + SMALL);
    double Bt2Ls = Bt2L * (sL - vL) / (sL - sM + SMALL);
    double Bt1Rs = Bt1R * (sR - vR) / (sR - sM + SMALL);
    double Bt2Rs = Bt2R * (sR - vR) / (sR - sM + SMALL);
    double denomL = DL * (sL - vL) - Bn * Bn;
    double denomR = DR * (sR - vR) - Bn * Bn;
    if (fabs(denomL) < SMALL || fabs(denomR) < SMALL) { hlle_vec(9, UL, UR, FL, FR, sL, sR, out); return; }
    double vt1L = UL[vt1] / dmax(DL, SMALL), vt2L = UL[vt2] / dmax(DL, SMALL);
    double vt1R = UR[vt1] / dmax(DR, SMALL), vt2R = UR[vt2] / dmax(DR, SMALL);
    double vt1Ls = vt1L - Bn * (Bt1L - Bt1Ls) / denomL;
    double vt2Ls = vt2L - Bn * (Bt2L - Bt2Ls) / denomL;
    double vt1Rs = vt1R - Bn * (Bt1R - Bt1Rs) / denomR;
    double vt2Rs = vt2R - Bn * (Bt2R - Bt2Rs) / denomR;
    double sLs = sM - fabs(Bn) / sqrt(DstarL + SMALL);
    double sRs = sM + fabs(Bn) / sqrt(DstarR + SMALL);
    double sqL = sqrt(DstarL), sqR = sqrt(DstarR);
    double sgn = (Bn >= 0.0) ? 1.0 : -1.0;
    double vt1ss = (sqL * vt1Ls + sqR * vt1Rs + sgn * (Bt1Rs - Bt1Ls)) / (sqL + sqR + SMALL);
    double vt2ss = (sqL * vt2Ls + sqR * vt2Rs + sgn * (Bt2Rs - Bt2Ls)) / (sqL + sqR + SMALL);
    double Bt1ss = (sqL * Bt1Rs + sqR * Bt1Ls + sgn * sqL * sqR * (vt1Ls - vt1Rs)) / (sqL + sqR + SMALL);
    double Bt2ss = (sqL * Bt2Rs + sqR * Bt2Ls + sgn * sqL * sqR * (vt2Ls - vt2Rs)) / (sqL + sqR + SMALL);
    double qLs[9], qRs[9], qss[9];
    double Dss = 0.5 * (DstarL + DstarR);
    double* qs[3] = {qLs, qRs, qss};
    double Ds[3] = {DstarL, DstarR, Dss};
    double a1[3] = {vt1Ls, vt1Rs, vt1ss}, a2[3] = {vt2Ls, vt2Rs, vt2ss};
    double b1[3] = {Bt1Ls, Bt1Rs, Bt1ss}, b2[3] = {Bt2Ls, Bt2Rs, Bt2ss};
    double ps[3] = {UL[8], UR[8], 0.5 * (UL[8] + UR[8])};
    for (int s = 0; s < 3; ++s) {
        double* q = qs[s];
        q[0] = dmax(Ds[s], SMALL);
        q[1 + n] = sM; q[1 + t1] = a1[s]; q[1 + t2] = a2[s];
        q[4] = (Ds[s] == DstarL) ? pL : pR;
        q[5 + n] = Bn; q[5 + t1] = b1[s]; q[5 + t2] = b2[s];
        q[8] = ps[s];
    }
    double ULs[9], URs[9], Us[9], FLs[9], FRs[9], Fs[9];
    r_p2c(pa, qLs, ULs);
    r_p2c(pa, qRs, URs);
    r_p2c(pa, qss, Us);
    r_flux(pa, n, qLs, FLs);
    r_flux(pa, n, qRs, FRs);
    r_flux(pa, n, qss, Fs);
    (void)FLs; (void)FRs; (void)Fs;
    if (sL <= 0.0 && 0.0 <= sLs) {
        for (int v = 0; v < 9; ++v) out[v] = FL[v] + sL * (ULs[v] - UL[v]);
        return;
    }
    if (sLs <= 0.0 && 0.0 <= sM) {
        for (int v = 0; v < 9; ++v) out[v] = FL[v] + sL * (ULs[v] - UL[v]) + sLs * (Us[v] - ULs[v]);
        return;
    }
    if (sM <= 0.0 && 0.0 <= sRs) {
        for (int v = 0; v < 9; ++v) out[v] = FR[v] + sR * (URs[v] - UR[v]) + sRs * (Us[v] - URs[v]);
        return;
    }
    if (sRs <= 0.0 && 0.0 <= sR) {
        for (int v = 0; v < 9; ++v) out[v] = FR[v] + sR * (URs[v] - UR[v]);
        return;
    }
    hlle_vec(9, UL, UR, FL, FR, sL, sR, out);
}

/* Riemann solve with given speeds (riemann_flux_rmhd_* :570,727,738), plus
 * the MUSCL-only upwind override of the induction/GLM fluxes for "hlld"
 * (compute_rhs_rmhd :811-831). */
static void r_riemann(const OParams* pa, int n, int muscl_override, const double* qL,
                      const double* qR, const double* UL, const double* UR,
                      const double* FL, const double* FR, double sL, double sR,
                      double* out) {
    double pL = qL[4], pR = qR[4], vL = qL[1 + n], vR = qR[1 + n];
    if (pa->riemann == 2) {
        r_hlld_full(pa, n, UL, UR, FL, FR, sL, sR, pL, pR, vL, vR, out);
    } else if (pa->riemann == 1) {
        double h5[5];
        hllc5(n, UL, UR, FL, FR, sL, sR, pL, pR, vL, vR, h5);
        hlle_vec(9, UL, UR, FL, FR, sL, sR, out);
        memcpy(out, h5, 5 * sizeof(double));
        if (muscl_override) {
            double sM = contact_speed(n, UL, UR, sL, sR, pL, pR, vL, vR);
            const double* Fm = (sM >= 0.0) ? FL : FR;
            for (int v = 5; v < 9; ++v) out[v] = Fm[v];
        }
    } else {
        hlle_vec(9, UL, UR, FL, FR, sL, sR, out);
    }
}

typedef struct { double q[9]; double U[9]; double F[9]; } RState;

static void r_prep(const OParams* pa, int n, double* q, RState* s) {
    r_floor(pa, q);
    memcpy(s->q, q, 9 * sizeof(double));
    r_p2c(pa, q, s->U);
    r_flux(pa, n, q, s->F);
}

static void r_speeds(const OParams* pa, int n, const RState* L, const RState* R,
                     double* sL, double* sR) {
    double lmL, lpL, lmR, lpR;
    double cfL = r_fast_speed(pa, L->q), cfR = r_fast_speed(pa, R->q);
    eig_speeds(L->q[1 + n], cfL, &lmL, &lpL);
    eig_speeds(R->q[1 + n], cfR, &lmR, &lpR);
    *sL = dmin(lmL, lmR);
    *sR = dmax(lpL, lpR);
}

/* RMHD face with its own speeds */
static void r_face(const OParams* pa, int n, int muscl_override, double* qL, double* qR,
                   Face* f) {
    RState L, R;
    r_prep(pa, n, qL, &L);
    r_prep(pa, n, qR, &R);
    double sL, sR;
    r_speeds(pa, n, &L, &R, &sL, &sR);
    r_riemann(pa, n, muscl_override, L.q, R.q, L.U, R.U, L.F, R.F, sL, sR, f->F);
    f->sL = sL; f->sR = sR; f->vL = L.q[1 + n]; f->vR = R.q[1 + n];
}

/* RMHD face with externally supplied speeds (the loop-carried x-left face) */
static void r_face_given(const OParams* pa, int n, double* qL, double* qR, double sL,
                         double sR, Face* f) {
    RState L, R;
    r_prep(pa, n, qL, &L);
    r_prep(pa, n, qR, &R);
    r_riemann(pa, n, 0, L.q, R.q, L.U, R.U, L.F, R.F, sL, sR, f->F);
    f->sL = sL; f->sR = sR; f->vL = L.q[1 + n]; f->vR = R.q[1 + n];
}

/* ------------------------------------------------------------------ */
/* face-state reconstruction helpers                                    */
/* ------------------------------------------------------------------ */
static const int DI[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};

/* value of variable v at offset o along direction n from (i,j,k) */
static inline double at(const OGrid* g, const double* pr, int v, int n, int i, int j, int k, int o) {
    return P(v, i + o * DI[n][0], j + o * DI[n][1], k + o * DI[n][2]);
}

/* MUSCL states at the face between cell c-1 and c (offset 0 is cell c):
 * qL from cell c-1, qR from cell c (srhd_core.py:482-528) */
static void muscl_states(const OParams* pa, const OGrid* g, const double* pr, int nvar,
                         int n, int i, int j, int k, double* qL, double* qR) {
    for (int v = 0; v < nvar; ++v) {
        double m2 = at(g, pr, v, n, i, j, k, -2), m1 = at(g, pr, v, n, i, j, k, -1);
        double c0 = at(g, pr, v, n, i, j, k, 0), p1 = at(g, pr, v, n, i, j, k, 1);
        double slL = limiter(pa->limiter, m1 - m2, c0 - m1);
        double slR = limiter(pa->limiter, c0 - m1, p1 - c0);
        qL[v] = m1 + 0.5 * slL;
        qR[v] = c0 - 0.5 * slR;
    }
}

static void ppm_states(const OGrid* g, const double* pr, int nvar, int n, int i, int j,
                       int k, double* qL, double* qR) {
    for (int v = 0; v < nvar; ++v) {
        double a[6];
        for (int o = -3; o <= 2; ++o) a[o + 3] = at(g, pr, v, n, i, j, k, o);
        double l0, r0, l1, r1;
        ppm(a[0], a[1], a[2], a[3], a[4], &l0, &r0);
        ppm(a[1], a[2], a[3], a[4], a[5], &l1, &r1);
        qL[v] = r0;
        qR[v] = l1;
    }
}

static void weno_states(const OGrid* g, const double* pr, int nvar, int n, int i, int j,
                        int k, double* qL, double* qR) {
    for (int v = 0; v < nvar; ++v) {
        double a[6];
        for (int o = -3; o <= 2; ++o) a[o + 3] = at(g, pr, v, n, i, j, k, o);
        qL[v] = weno5(a[0], a[1], a[2], a[3], a[4]);
        qR[v] = weno5(a[5], a[4], a[3], a[2], a[1]);
    }
}

/* reconstructed face states at the face between (cell - e_n) and cell */
static void face_states(const OParams* pa, const OGrid* g, const double* pr, int nvar,
                        int n, int i, int j, int k, double* qL, double* qR) {
    if (pa->recon == 0) muscl_states(pa, g, pr, nvar, n, i, j, k, qL, qR);
    else if (pa->recon == 1) ppm_states(g, pr, nvar, n, i, j, k, qL, qR);
    else weno_states(g, pr, nvar, n, i, j, k, qL, qR);
}

/* ------------------------------------------------------------------ */
/* passive scalars (the triple-evaluation quirk, srhd_core.py:534-660,  */
/* rmhd_core.py:832-940)                                                */
/* ------------------------------------------------------------------ */
enum { PW = 0, PP = 1, PM = 2 };

/* passive face flux of kind K at the face between (c - e_n) and c */
static double passive_face(const OParams* pa, const OGrid* g, const double* pr, int idx,
                           int kind, int n, int i, int j, int k, double vL, double vR,
                           double sL, double sR) {
    double a[6];
    for (int o = -3; o <= 2; ++o)
        a[o + 3] = pget(g, pr, idx, i + o * DI[n][0], j + o * DI[n][1], k + o * DI[n][2]);
    double tL, tR;
    if (kind == PW) {
        tL = weno5(a[0], a[1], a[2], a[3], a[4]);
        tR = weno5(a[5], a[4], a[3], a[2], a[1]);
    } else if (kind == PP) {
        double l0, r0, l1, r1;
        ppm(a[0], a[1], a[2], a[3], a[4], &l0, &r0);
        ppm(a[1], a[2], a[3], a[4], a[5], &l1, &r1);
        tL = r0; tR = l1;
    } else {
        double slL = limiter(pa->limiter, a[2] - a[1], a[3] - a[2]);
        double slR = limiter(pa->limiter, a[3] - a[2], a[4] - a[3]);
        tL = a[2] + 0.5 * slL;
        tR = a[3] - 0.5 * slR;
    }
    return hlle_scalar(tL, tR, tL * vL, tR * vR, sL, sR);
}

/* ------------------------------------------------------------------ */
/* right-hand sides                                                     */
/* ------------------------------------------------------------------ */
static int bounds_lo(const OParams* pa) { return pa->recon == 0 ? 2 : 3; }
static int bounds_hi_off(const OParams* pa) {
    if (pa->recon != 0) return 3;
    return pa->physics == 0 ? 3 : 2; /* SRHD MUSCL [2,n-3), RMHD MUSCL [2,n-2) */
}

static void s_rhs(const OParams* pa, const OGrid* g, const double* pr, double dd[3],
                  double* rhs) {
    const int nr = 5 + pa->n_passive;
    OGrid gr = {nr, g->nx, g->ny, g->nz};
    memset(rhs, 0, sizeof(double) * (size_t)nr * g->nx * g->ny * g->nz);
    int lo = bounds_lo(pa), ho = bounds_hi_off(pa);
    int i1 = g->nx - ho, j1 = g->ny - ho, k1 = g->nz - ho;
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = lo; i < i1; ++i)
        for (int j = lo; j < j1; ++j)
            for (int k = lo; k < k1; ++k) {
                double r[5] = {0, 0, 0, 0, 0};
                for (int n = 0; n < 3; ++n) {
                    int o[3] = {i + DI[n][0], j + DI[n][1], k + DI[n][2]};
                    double qL[5], qR[5], qL2[5], qR2[5];
                    Face fa, fb;
                    face_states(pa, g, pr, 5, n, i, j, k, qL, qR);
                    face_states(pa, g, pr, 5, n, o[0], o[1], o[2], qL2, qR2);
                    if (pa->recon == 0 && pa->passive_offset > 5) {
                        /* add_pi_lr (srhd_core.py:394-398) */
                        qL[4] += P(5, i - DI[n][0], j - DI[n][1], k - DI[n][2]);
                        qR[4] += P(5, i, j, k);
                        qL2[4] += P(5, i, j, k);
                        qR2[4] += P(5, o[0], o[1], o[2]);
                    }
                    /* dissipation fluxes of blocks of 15+ variables: once in
                     * MUSCL, twice in PPM (srhd_core.py:543-544, 958-961),
                     * none in WENO */
                    const int nd = g->nv >= 15 ? (pa->recon == 0 ? 1 : (pa->recon == 1 ? 2 : 0)) : 0;
                    double isA[10], isB[10], isC[10];
                    if (nd)
                        for (int m = 0; m < 10; ++m) {
                            isA[m] = P(5 + m, i - DI[n][0], j - DI[n][1], k - DI[n][2]);
                            isB[m] = P(5 + m, i, j, k);
                            isC[m] = P(5 + m, o[0], o[1], o[2]);
                        }
                    s_face_is(pa, n, qL, qR, nd, isA, isB, &fa);
                    s_face_is(pa, n, qL2, qR2, nd, isB, isC, &fb);
                    for (int v = 0; v < 5; ++v) r[v] -= (fb.F[v] - fa.F[v]) / dd[n];
                    /* passives */
                    int kinds[3], nk = 0, lkind = -1;
                    if (pa->recon == 0 && n == 0) { kinds[0] = PW; kinds[1] = PP; kinds[2] = PM; nk = 3; lkind = PM; }
                    if (pa->recon == 0 && n == 2) { kinds[0] = PM; nk = 1; lkind = PM; }
                    if (pa->recon == 1 && n == 1) { kinds[0] = PW; kinds[1] = PP; kinds[2] = PM; nk = 3; lkind = PM; }
                    if (pa->recon == 1 && n == 2) { kinds[0] = PW; kinds[1] = PP; nk = 2; lkind = PP; }
                    for (int t = 0; t < pa->n_passive && nk > 0; ++t) {
                        int idx = pa->passive_offset + t;
                        double FLt = passive_face(pa, g, pr, idx, lkind, n, i, j, k,
                                                  fa.vL, fa.vR, fa.sL, fa.sR);
                        double acc = 0.0;
                        for (int q = 0; q < nk; ++q) {
                            double FRt = passive_face(pa, g, pr, idx, kinds[q], n, o[0], o[1],
                                                      o[2], fb.vL, fb.vR, fb.sL, fb.sR);
                            acc -= (FRt - FLt) / dd[n];
                        }
                        rhs[IX(&gr, 5 + t, i, j, k)] += acc;
                    }
                }
                for (int v = 0; v < 5; ++v) rhs[IX(&gr, v, i, j, k)] = r[v];
            }
}

/* z-back face speeds of cell (i,j,k) for the loop-carried RMHD PPM/WENO quirk */
static void r_zback_speeds(const OParams* pa, const OGrid* g, const double* pr, int i,
                           int j, int k, double* sL, double* sR) {
    double qL[9], qR[9];
    face_states(pa, g, pr, 9, 2, i, j, k, qL, qR);
    RState L, R;
    r_prep(pa, 2, qL, &L);
    r_prep(pa, 2, qR, &R);
    r_speeds(pa, 2, &L, &R, sL, sR);
}

static void r_rhs(const OParams* pa, const OGrid* g, const double* pr, double dd[3],
                  double* rhs) {
    const int nr = 9 + pa->n_passive;
    OGrid gr = {nr, g->nx, g->ny, g->nz};
    memset(rhs, 0, sizeof(double) * (size_t)nr * g->nx * g->ny * g->nz);
    int lo = bounds_lo(pa), ho = bounds_hi_off(pa);
    int i1 = g->nx - ho, j1 = g->ny - ho, k1 = g->nz - ho;
    const int muscl = (pa->recon == 0);
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = lo; i < i1; ++i) {
        for (int j = lo; j < j1; ++j) {
            /* loop-carried (sL, sR) entering row (i, j): +-1 for the very first
             * cell, else the z-back face speeds of the previous cell in the
             * reference's serial i-j-k order */
            double cL = -1.0, cR = 1.0;
            if (!muscl && j > lo) r_zback_speeds(pa, g, pr, i, j - 1, k1 - 1, &cL, &cR);
            else if (!muscl && i > lo) r_zback_speeds(pa, g, pr, i - 1, j1 - 1, k1 - 1, &cL, &cR);
            for (int k = lo; k < k1; ++k) {
                double r[9] = {0};
                for (int n = 0; n < 3; ++n) {
                    int o[3] = {i + DI[n][0], j + DI[n][1], k + DI[n][2]};
                    double qL[9], qR[9], qL2[9], qR2[9];
                    Face fa, fb;
                    face_states(pa, g, pr, 9, n, i, j, k, qL, qR);
                    face_states(pa, g, pr, 9, n, o[0], o[1], o[2], qL2, qR2);
                    if (!muscl && n == 0 && pa->flux_mode == 0) r_face_given(pa, 0, qL, qR, cL, cR, &fa);
                    else r_face(pa, n, muscl, qL, qR, &fa);
                    r_face(pa, n, muscl, qL2, qR2, &fb);
                    if (!muscl && n == 2) { cL = fa.sL; cR = fa.sR; }
                    for (int v = 0; v < 9; ++v) r[v] -= (fb.F[v] - fa.F[v]) / dd[n];
                    if (muscl) {
                        /* WENO, PPM and MC passive fluxes on the high face, all
                         * with the LOW face's speeds, minus the MC low-face flux */
                        for (int t = 0; t < pa->n_passive; ++t) {
                            int idx = pa->passive_offset + t;
                            double FLt = passive_face(pa, g, pr, idx, PM, n, i, j, k, fa.vL,
                                                      fa.vR, fa.sL, fa.sR);
                            double acc = 0.0;
                            for (int q = 0; q < 3; ++q) {
                                double FRt = passive_face(pa, g, pr, idx, q, n, o[0], o[1], o[2],
                                                          fb.vL, fb.vR, fa.sL, fa.sR);
                                acc -= (FRt - FLt) / dd[n];
                            }
                            rhs[IX(&gr, 9 + t, i, j, k)] += acc;
                        }
                    }
                }
                r[8] -= pa->glm_cp * pa->glm_cp * P(8, i, j, k);
                int nres = (pa->resistive && pa->resistivity > 0.0)
                               ? (pa->recon == 0 ? 1 : (pa->recon == 1 ? 2 : 0)) : 0;
                if (pa->flux_mode == 1) nres = (pa->resistive && pa->resistivity > 0.0) ? 1 : 0;
                for (int rep = 0; rep < nres; ++rep) {
                    double ix2 = 1.0 / (dd[0] * dd[0] + SMALL);
                    double iy2 = 1.0 / (dd[1] * dd[1] + SMALL);
                    double iz2 = 1.0 / (dd[2] * dd[2] + SMALL);
                    for (int c = 5; c < 8; ++c) {
                        double lap = (P(c, i + 1, j, k) - 2.0 * P(c, i, j, k) + P(c, i - 1, j, k)) * ix2 +
                                     (P(c, i, j + 1, k) - 2.0 * P(c, i, j, k) + P(c, i, j - 1, k)) * iy2 +
                                     (P(c, i, j, k + 1) - 2.0 * P(c, i, j, k) + P(c, i, j, k - 1)) * iz2;
                        r[c] += pa->resistivity * lap;
                    }
                }
                for (int v = 0; v < 9; ++v) rhs[IX(&gr, v, i, j, k)] = r[v];
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* exported API                                                         */
/* ------------------------------------------------------------------ */
int oracle_rhs(const OParams* pa, const double* pr, int nv, int nx, int ny, int nz,
               double dx, double dy, double dz, double* rhs) {
    OGrid g = {nv, nx, ny, nz};
    double dd[3] = {dx, dy, dz};
    if (pa->physics == 0) {
        s_rhs(pa, &g, pr, dd, rhs);
    } else {
        r_rhs(pa, &g, pr, dd, rhs);
    }
    return 0;
}

void oracle_p2c(const OParams* pa, const double* q, double* U, long count) {
    int nm = pa->physics == 0 ? 5 : 9;
    for (long c = 0; c < count; ++c) {
        double a[9], b[9];
        for (int v = 0; v < nm; ++v) a[v] = q[v * count + c];
        if (pa->physics == 0) s_p2c(a, b); else r_p2c(pa, a, b);
        for (int v = 0; v < nm; ++v) U[v * count + c] = b[v];
    }
}

void oracle_c2p(const OParams* pa, const double* U, double* q, long count) {
    int nm = pa->physics == 0 ? 5 : 9;
    for (long c = 0; c < count; ++c) {
        double a[9], b[9];
        for (int v = 0; v < nm; ++v) a[v] = U[v * count + c];
        if (pa->physics == 0) s_c2p(pa, a, b); else r_c2p(pa, a, b);
        for (int v = 0; v < nm; ++v) q[v * count + c] = b[v];
    }
}

void oracle_c2p_counters(long* out3, int reset) {
    out3[0] = g_c2p_newton; out3[1] = g_c2p_bisect; out3[2] = g_c2p_hydro_fallback;
    if (reset) g_c2p_newton = g_c2p_bisect = g_c2p_hydro_fallback = 0;
}

double oracle_max_char_speed(const double* pr, int nv, int nx, int ny, int nz) {
    OGrid g0 = {nv, nx, ny, nz};
    const OGrid* g = &g0;
    double amax = 0.0;
    for (int i = 1; i < nx - 1; ++i)
        for (int j = 1; j < ny - 1; ++j)
            for (int k = 1; k < nz - 1; ++k) {
                double cs = s_sound_speed(P(0, i, j, k), P(4, i, j, k));
                double loc = 0.0;
                for (int n = 0; n < 3; ++n) {
                    double lm, lp;
                    eig_speeds(P(1 + n, i, j, k), cs, &lm, &lp);
                    loc = dmax(loc, dmax(fabs(lm), fabs(lp)));
                }
                if (loc > amax) amax = loc;
            }
    if (amax < SMALL) amax = SMALL;
    return amax;
}

/* ------------------------------------------------------------------ */
/* fixed-metric GR wrappers (grhd_core.py, grmhd_core.py, gr_metric.py) */
/* ------------------------------------------------------------------ */
typedef struct { int metric, orthonormal, ng, offs_x; double mass, spin; } OGR;
enum { GR_MINK = 0, GR_SCHW = 1, GR_KS = 2, GR_OTHER = 3 };

/* gr_metric.py:19-36 (lapse of the Kerr-Schild form; shift unused) */
static void gr_ks(double x, double y, double z, double M, double* alpha, double g[3]) {
    double r = sqrt(x * x + y * y + z * z) + 1e-12;
    double H = M / r;
    *alpha = 1.0 / sqrt(1.0 + 2.0 * H);
    double lx = x / r, ly = y / r, lz = z / r;
    double dlnadr = H / (r * (1.0 + 2.0 * H));
    g[0] = dlnadr * lx; g[1] = dlnadr * ly; g[2] = dlnadr * lz;
}

/* gr_metric.py:6-16 */
static void gr_iso(double x, double y, double z, double M, double g[3]) {
    double r = sqrt(x * x + y * y + z * z) + 1e-12;
    double a = M / (2.0 * r);
    double denom = (1.0 - a * a);
    double dlnadr = denom == 0.0 ? 0.0 : (2.0 * a) / (r * denom);
    g[0] = dlnadr * (x / r); g[1] = dlnadr * (y / r); g[2] = dlnadr * (z / r);
}

/* compute_rhs_grhd / compute_rhs_grmhd (grhd_core.py:20-78,
 * grmhd_core.py:20-80): velocity rescale for the fluxes, core RHS, sources */
int oracle_rhs_gr(const OParams* pa, const OGR* gr, const double* pr, int nv, int nx, int ny,
                  int nz, double dx, double dy, double dz, double* rhs) {
    OGrid g0 = {nv, nx, ny, nz};
    const OGrid* g = &g0;
    const size_t nc = (size_t)nx * ny * nz;
    const int ng = gr->ng;
    const double* use = pr;
    double* copy = NULL;
    if (gr->orthonormal && (gr->metric == GR_SCHW || gr->metric == GR_KS)) {
        copy = malloc(sizeof(double) * nv * nc);
        if (!copy) return -1;
        memcpy(copy, pr, sizeof(double) * nv * nc);
        for (int i = ng; i < nx - ng; ++i)
            for (int j = ng; j < ny - ng; ++j)
                for (int k = ng; k < nz - ng; ++k) {
                    double x = (gr->offs_x + (i - ng) + 0.5) * dx;
                    double y = (j - ng + 0.5) * dy, z = (k - ng + 0.5) * dz;
                    double alpha, gg[3];
                    gr_ks(x, y, z, gr->mass, &alpha, gg);
                    double ax = dmax(alpha, 1e-12);
                    for (int v = 1; v <= 3; ++v) copy[IX(g, v, i, j, k)] = P(v, i, j, k) / ax;
                }
        use = copy;
    }
    int rc = oracle_rhs(pa, use, nv, nx, ny, nz, dx, dy, dz, rhs);
    free(copy);
    if (rc != 0 || gr->metric == GR_MINK) return rc;
    const int nr = (pa->physics == 0 ? 5 : 9) + pa->n_passive;
    OGrid gr_r = {nr, nx, ny, nz};
    for (int i = ng; i < nx - ng; ++i)
        for (int j = ng; j < ny - ng; ++j)
            for (int k = ng; k < nz - ng; ++k) {
                double x = (gr->offs_x + (i - ng) + 0.5) * dx;
                double y = (j - ng + 0.5) * dy, z = (k - ng + 0.5) * dz;
                double gg[3], alpha;
                if (gr->metric == GR_SCHW) gr_iso(x, y, z, gr->mass, gg);
                else gr_ks(x, y, z, gr->mass, &alpha, gg);
                double q[9], U[9];
                for (int v = 0; v < (pa->physics == 0 ? 5 : 9); ++v) q[v] = P(v, i, j, k);
                double v2 = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
                if (v2 >= 1.0) v2 = 1.0 - 1e-14;
                double W = 1.0 / sqrt(1.0 - v2);
                double h = 1.0 + pa->gamma / (pa->gamma - 1.0) * q[4] / dmax(q[0], SMALL);
                double w;
                if (pa->physics == 0) {
                    w = q[0] * h * W * W + q[4];
                    s_p2c(q, U);  /* srhd prim_to_cons: its default gamma 5/3 */
                } else {
                    double B2 = q[5] * q[5] + q[6] * q[6] + q[7] * q[7];
                    w = q[0] * h * W * W + B2 + q[4];
                    r_p2c(pa, q, U);
                }
                rhs[IX(&gr_r, 1, i, j, k)] += w * gg[0];
                rhs[IX(&gr_r, 2, i, j, k)] += w * gg[1];
                rhs[IX(&gr_r, 3, i, j, k)] += w * gg[2];
                rhs[IX(&gr_r, 4, i, j, k)] += U[1] * gg[0] + U[2] * gg[1] + U[3] * gg[2];
            }
    return 0;
}

static int step_impl(const OParams* pa, const OGR* gr, const double* pr, int nv, int nx, int ny,
                     int nz, double dx, double dy, double dz, double dt, int rk, double* out);

/* One SSPRK2/3 step (srhd_core.py:1286-1400, rmhd_core.py:1559-1677). */
int oracle_step(const OParams* pa, const double* pr, int nv, int nx, int ny, int nz,
                double dx, double dy, double dz, double dt, int rk, double* out) {
    return step_impl(pa, NULL, pr, nv, nx, ny, nz, dx, dy, dz, dt, rk, out);
}

static void block_p2c(const OParams* pa, const double* pr, size_t nc, double* U0);
static void stage_impl(const OParams* pa, const OGR* gr, const double* pr, const double* U0,
                       const double* cur, double* Uk, double* rhs, int nv, int nx, int ny,
                       int nz, double dx, double dy, double dz, double dt, int nst, int s,
                       double* dst);

/* Stage `stage` of an SSPRK step from pr (the step input), prk (this stage's
 * input), Uk (nm x nc: the previous stage's conserved state in, this stage's
 * out; ignored in at stage 0): what the stage loop of oracle_step does, for
 * callers that refresh ghosts between stages. */
int oracle_stage(const OParams* pa, const double* pr, const double* prk, double* Uk, int nv,
                 int nx, int ny, int nz, double dx, double dy, double dz, double dt, int rk,
                 int stage, double* out) {
    const int nm = pa->physics == 0 ? 5 : 9;
    const size_t nc = (size_t)nx * ny * nz;
    double* U0 = malloc(sizeof(double) * nm * nc);
    double* rhs = malloc(sizeof(double) * (nm + pa->n_passive) * nc);
    if (!U0 || !rhs) return -1;
    block_p2c(pa, pr, nc, U0);
    stage_impl(pa, NULL, pr, U0, prk, Uk, rhs, nv, nx, ny, nz, dx, dy, dz, dt,
               rk == 3 ? 3 : 2, stage, out);
    free(U0); free(rhs);
    return 0;
}

/* The GR wrappers' steps (grhd_core.py:76-166, grmhd_core.py:80-183): the
 * core step with the GR right-hand side. */
int oracle_step_gr(const OParams* pa, const OGR* gr, const double* pr, int nv, int nx, int ny,
                   int nz, double dx, double dy, double dz, double dt, int rk, double* out) {
    return step_impl(pa, gr, pr, nv, nx, ny, nz, dx, dy, dz, dt, rk, out);
}

/* U0 = prim_to_cons(pr) over the block (the steps' U0 loops) */
static void block_p2c(const OParams* pa, const double* pr, size_t nc, double* U0) {
    const int nm = pa->physics == 0 ? 5 : 9;
    for (size_t c = 0; c < nc; ++c) {
        double a[9], b[9];
        for (int v = 0; v < nm; ++v) a[v] = pr[v * nc + c];
        if (pa->physics == 0) s_p2c(a, b); else r_p2c(pa, a, b);
        for (int v = 0; v < nm; ++v) U0[v * nc + c] = b[v];
    }
}

/* Stage s of nst (srhd_core.py:1286-1400, rmhd_core.py:1559-1677): the
 * right-hand side of cur, Uk <- the stage's SSPRK combination with U0, dst <-
 * con2prim(Uk), the carried and passive fields; rhs is scratch. */
static void stage_impl(const OParams* pa, const OGR* gr, const double* pr, const double* U0,
                       const double* cur, double* Uk, double* rhs, int nv, int nx, int ny,
                       int nz, double dx, double dy, double dz, double dt, int nst, int s,
                       double* dst) {
    const int nm = pa->physics == 0 ? 5 : 9;
    const int np = pa->n_passive, po = pa->passive_offset;
    const size_t nc = (size_t)nx * ny * nz;
    {
        if (gr) oracle_rhs_gr(pa, gr, cur, nv, nx, ny, nz, dx, dy, dz, rhs);
        else oracle_rhs(pa, cur, nv, nx, ny, nz, dx, dy, dz, rhs);
        memset(dst, 0, sizeof(double) * (size_t)nv * nc);
#pragma omp parallel for schedule(static)
        for (long cl = 0; cl < (long)nc; ++cl) {
            size_t c = (size_t)cl;
            double Un[9], q[9];
            for (int v = 0; v < nm; ++v) {
                double r = rhs[v * nc + c], u0 = U0[v * nc + c];
                if (s == 0) Un[v] = u0 + dt * r;
                else if (nst == 2) Un[v] = 0.5 * ((u0 + Uk[v * nc + c]) + dt * r);
                else if (s == 1) Un[v] = 0.75 * u0 + 0.25 * (Uk[v * nc + c] + dt * r);
                else Un[v] = (1.0 / 3.0) * u0 + (2.0 / 3.0) * (Uk[v * nc + c] + dt * r);
                Uk[v * nc + c] = Un[v];
            }
            if (pa->physics == 0) s_c2p(pa, Un, q); else r_c2p(pa, Un, q);
            for (int v = 0; v < nm; ++v) dst[v * nc + c] = q[v];
            if (pa->physics == 0 && nv > 5 && po > 5)
                for (int v = 5; v < po; ++v) dst[v * nc + c] = cur[v * nc + c];
            for (int t = 0; t < np; ++t) {
                size_t o = (size_t)(po + t) * nc + c;
                double t0 = pr[o], r = rhs[(size_t)(nm + t) * nc + c];
                if (s == 0) dst[o] = t0 + dt * r;
                else if (nst == 2) dst[o] = 0.5 * ((t0 + cur[o]) + dt * r);
                else if (s == 1) dst[o] = 0.75 * t0 + 0.25 * (cur[o] + dt * r);
                else dst[o] = (1.0 / 3.0) * t0 + (2.0 / 3.0) * (cur[o] + dt * r);
            }
        }
    }
}

static int step_impl(const OParams* pa, const OGR* gr, const double* pr, int nv, int nx, int ny,
                     int nz, double dx, double dy, double dz, double dt, int rk, double* out) {
    const int nm = pa->physics == 0 ? 5 : 9;
    const size_t nc = (size_t)nx * ny * nz;
    const int nr = nm + pa->n_passive;
    double* U0 = malloc(sizeof(double) * nm * nc);
    double* Uk = malloc(sizeof(double) * nm * nc);
    double* rhs = malloc(sizeof(double) * nr * nc);
    double* prA = calloc((size_t)nv * nc, sizeof(double));
    double* prB = calloc((size_t)nv * nc, sizeof(double));
    if (!U0 || !Uk || !rhs || !prA || !prB) return -1;
    block_p2c(pa, pr, nc, U0);
    const double* cur = pr;
    const double* prev = NULL;   /* primitives of the previous stage */
    const int nst = (rk == 3) ? 3 : 2;
    double* bufs[2] = {prA, prB};
    for (int s = 0; s < nst; ++s) {
        double* dst = (s == nst - 1) ? out : bufs[s % 2];
        stage_impl(pa, gr, pr, U0, cur, Uk, rhs, nv, nx, ny, nz, dx, dy, dz, dt, nst, s, dst);
        prev = cur;
        cur = dst;
    }
    (void)prev;
    free(U0); free(Uk); free(rhs); free(prA); free(prB);
    return 0;
}

/* ------------------------------------------------------------------ */
/* ghost fills (boundary.py:4-11, nozzle.py:5-91)                       */
/* ------------------------------------------------------------------ */
void oracle_periodic_yz(double* pr, int nv, int nx, int ny, int nz, int ng) {
    OGrid g0 = {nv, nx, ny, nz};
    const OGrid* g = &g0;
    for (int v = 0; v < nv; ++v)
        for (int i = 0; i < nx; ++i) {
            for (int j = 0; j < ng; ++j)
                for (int k = 0; k < nz; ++k) P(v, i, j, k) = P(v, i, ny - 2 * ng + j, k);
            for (int j = 0; j < ng; ++j)
                for (int k = 0; k < nz; ++k) P(v, i, ny - ng + j, k) = P(v, i, ng + j, k);
        }
    for (int v = 0; v < nv; ++v)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                for (int k = 0; k < ng; ++k) P(v, i, j, k) = P(v, i, j, nz - 2 * ng + k);
                for (int k = 0; k < ng; ++k) P(v, i, j, nz - ng + k) = P(v, i, j, ng + k);
            }
}

/* extension, no reference counterpart: zero-gradient y faces, then z faces */
void oracle_outflow_yz(double* pr, int nv, int nx, int ny, int nz, int ng) {
    OGrid g0 = {nv, nx, ny, nz};
    const OGrid* g = &g0;
    for (int v = 0; v < nv; ++v)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ng; ++j)
                for (int k = 0; k < nz; ++k) {
                    P(v, i, j, k) = P(v, i, ng, k);
                    P(v, i, ny - 1 - j, k) = P(v, i, ny - 1 - ng, k);
                }
    for (int v = 0; v < nv; ++v)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < ng; ++k) {
                    P(v, i, j, k) = P(v, i, j, ng);
                    P(v, i, j, nz - 1 - k) = P(v, i, j, nz - 1 - ng);
                }
}

void oracle_outflow_right_x(double* pr, int nv, int nx, int ny, int nz, int ng) {
    OGrid g0 = {nv, nx, ny, nz};
    const OGrid* g = &g0;
    for (int v = 0; v < nv; ++v)
        for (int i = nx - ng; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < nz; ++k) P(v, i, j, k) = P(v, nx - ng - 1, j, k);
}

typedef struct {
    int ng, profile;          /* profile 0 top_hat, 1 taper/smooth, 2 parabolic */
    int perturb;              /* 0 none, else random                            */
    int physics;              /* 0 hydro, 1 rmhd                                */
    int b_init;               /* 0 none, 1 poloidal, 2 toroidal, 3 B_phi(r)     */
    int n_tracers, tracer_offset, two_temperature, thermo_offset;
    int ambient_bc;           /* s = 0 cells: 0 fixed ambient, 1 zero-gradient  */
    double radius, shear_thick, gamma_jet, eta_rho, p_eq, rho_amb;
    double vx_amb, vy_amb, vz_amb, turb_vamp, turb_pamp, b0, te, ti;
    double tracer_nozzle[8], tracer_amb[8];
    double b_amb_x;
    int chemistry, chem_offset;  /* CHEMISTRY_ENABLED, CHEM_OFFSET         */
    double chem_x[3];            /* CHEM_X_HII/HEII/HEIII_NOZZLE           */
} ONozzle;

static double nozzle_weight(double r, double radius, double shear, int profile) {
    if (radius <= 0.0) return 0.0;
    if (profile == 1) {
        if (r >= radius) return 0.0;
        return 0.5 * (1.0 + cos(M_PI * r / radius));
    }
    if (profile == 2) {
        if (r >= radius) return 0.0;
        double x = r / radius;
        return dmax(0.0, 1.0 - x * x);
    }
    if (shear > 0.0) return 0.5 * (1.0 - tanh((r - radius) / shear));
    return r <= radius ? 1.0 : 0.0;
}

/* rnd: host-drawn uniforms in the reference's draw order, 3 per perturbed
 * cell, or NULL when unperturbed.  Returns the number of draws consumed. */
long oracle_nozzle_left_x(double* pr, int nv, int nx, int ny, int nz, double dy,
                          double dz, int ny_loc, int nz_loc, double y0, double z0,
                          const ONozzle* c, const double* rnd) {
    OGrid g0 = {nv, nx, ny, nz};
    const OGrid* g = &g0;
    long used = 0;
    for (int gg = 0; gg < c->ng; ++gg)
        for (int j = c->ng; j < c->ng + ny_loc; ++j) {
            double y = (j - c->ng + 0.5) * dy;
            for (int k = c->ng; k < c->ng + nz_loc; ++k) {
                double z = (k - c->ng + 0.5) * dz;
                double rr = sqrt((y - y0) * (y - y0) + (z - z0) * (z - z0));
                double s = nozzle_weight(rr, c->radius, c->shear_thick, c->profile);
                /* extension, no reference counterpart: outflow outside the nozzle */
                if (c->ambient_bc == 1 && !(s > 0.0)) {
                    for (int v = 0; v < nv; ++v) P(v, gg, j, k) = P(v, c->ng, j, k);
                    continue;
                }
                double rho = c->eta_rho * c->rho_amb * s + c->rho_amb * (1.0 - s);
                double p = c->p_eq;
                double beta = sqrt(1.0 - 1.0 / (c->gamma_jet * c->gamma_jet));
                double vx = beta * s + c->vx_amb * (1.0 - s);
                double vy = c->vy_amb, vz = c->vz_amb;
                if (c->perturb && s > 0.0) {
                    vy += c->turb_vamp * (2.0 * rnd[used] - 1.0);
                    vz += c->turb_vamp * (2.0 * rnd[used + 1] - 1.0);
                    p *= (1.0 + c->turb_pamp * (2.0 * rnd[used + 2] - 1.0));
                    used += 3;
                }
                P(0, gg, j, k) = rho; P(1, gg, j, k) = vx; P(2, gg, j, k) = vy;
                P(3, gg, j, k) = vz; P(4, gg, j, k) = p;
                if (nv >= 15)
                    for (int v = 5; v < 15; ++v) P(v, gg, j, k) = 0.0;
                for (int t = 0; t < c->n_tracers; ++t) {
                    double tn = c->tracer_nozzle[t], ta = c->tracer_amb[t];
                    P(c->tracer_offset + t, gg, j, k) = ta + (tn - ta) * s;
                }
                if (c->two_temperature && nv > c->thermo_offset + 1) {
                    P(c->thermo_offset, gg, j, k) = c->te;
                    P(c->thermo_offset + 1, gg, j, k) = c->ti;
                }
                /* nozzle.py:77-82: the inflow's ionisation fractions */
                if (c->chemistry && nv > c->chem_offset + 2)
                    for (int m = 0; m < 3; ++m) P(c->chem_offset + m, gg, j, k) = c->chem_x[m];
                if (c->physics == 1) {
                    double Bx = 0.0, By = 0.0, Bz = 0.0;
                    if (c->b_init == 1) Bx = c->b0 * s;
                    else if (c->b_init == 2) By = c->b0 * s;
                    else if (c->b_init == 3) {
                        /* extension: B_phi = B0 r/R inside, B0 R/r outside, times s */
                        double bphi = rr < c->radius ? c->b0 * rr / c->radius
                                                     : c->b0 * c->radius / rr;
                        double f = rr > 0.0 ? s * bphi / rr : 0.0;
                        Bx = c->b_amb_x;
                        By = -f * (z - z0);
                        Bz = f * (y - y0);
                    }
                    P(5, gg, j, k) = Bx; P(6, gg, j, k) = By; P(7, gg, j, k) = Bz;
                    P(8, gg, j, k) = 0.0;
                }
            }
        }
    return used;
}

/* operator-split post-step sources (source_terms.py:5-55) */
void oracle_cooling(double* pr, int nv, int nx, int ny, int nz, int ng, double dt,
                    double cool, double heat, double pmax) {
    OGrid g0 = {nv, nx, ny, nz};
    const OGrid* g = &g0;
    if (cool == 0.0 && heat == 0.0) return;
    for (int i = ng; i < nx - ng; ++i)
        for (int j = ng; j < ny - ng; ++j)
            for (int k = ng; k < nz - ng; ++k) {
                double rho = P(0, i, j, k), p = P(4, i, j, k);
                double dp = dt * (heat - cool * rho * p);
                double pn = p + dp;
                if (pn < 1e-12) pn = 1e-12;
                if (pn > pmax) pn = pmax;
                P(4, i, j, k) = pn;
            }
}

void oracle_two_temperature(double* pr, int nv, int nx, int ny, int nz, int ng, double dt,
                            double tau, int off) {
    OGrid g0 = {nv, nx, ny, nz};
    const OGrid* g = &g0;
    if (nv < off + 2 || tau <= 0.0) return;
    for (int i = ng; i < nx - ng; ++i)
        for (int j = ng; j < ny - ng; ++j)
            for (int k = ng; k < nz - ng; ++k) {
                double rho = P(0, i, j, k), p = P(4, i, j, k);
                double T = p / dmax(rho, 1e-12);
                double Te = P(off, i, j, k), Ti = P(off + 1, i, j, k);
                Te += dt * (T - Te) / tau;
                Ti += dt * (T - Ti) / tau;
                P(off, i, j, k) = Te;
                P(off + 1, i, j, k) = Ti;
            }
}

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* H/He ionisation (chemistry.py:43-139), interior cells, in place      */
/* ------------------------------------------------------------------ */
static double ch_clamp(double x, double lo, double hi) {
    if (x < lo) return lo;
    if (x > hi) return hi;
    return x;
}
static double ch_ci(double a, double e, double T) {
    return a * sqrt(T) * exp(-e / dmax(T, 1.0)) / (1.0 + sqrt(T / 1.0e5));
}
void oracle_ion_chemistry(double* pr, int nv, int nx, int ny, int nz, int ng, int off, double dt,
                          double X, double Y, double tunit, double rate_scale,
                          double energy_scale, double tmin, double gamma) {
    OGrid g0 = {nv, nx, ny, nz};
    const OGrid* g = &g0;
    const double CSMALL = 1e-20; /* chemistry.py's SMALL */
    for (int i = ng; i < nx - ng; ++i)
        for (int j = ng; j < ny - ng; ++j)
            for (int k = ng; k < nz - ng; ++k) {
                double rho = P(0, i, j, k), p = P(4, i, j, k);
                if (rho <= 0.0 || p <= 0.0) continue;
                double T = (p / dmax(rho, CSMALL)) * tunit;
                if (T < tmin) T = tmin;
                double nH = X * rho, nHe = Y * rho / 4.0;
                double xHII = ch_clamp(P(off, i, j, k), 0.0, 1.0);
                double xHeII = ch_clamp(P(off + 1, i, j, k), 0.0, 1.0);
                double xHeIII = ch_clamp(P(off + 2, i, j, k), 0.0, 1.0);
                xHeII = xHeII < 1.0 - xHeIII ? xHeII : 1.0 - xHeIII;
                double xHeI = dmax(0.0, 1.0 - xHeII - xHeIII);
                double xHI = 1.0 - xHII;
                double ne = dmax(nH * xHII + nHe * (xHeII + 2.0 * xHeIII), CSMALL);
                double C_H = rate_scale * ch_ci(5.85e-11, 157809.1, T);
                double C_HeI = rate_scale * ch_ci(2.38e-11, 285335.4, T);
                double C_HeII = rate_scale * ch_ci(5.68e-12, 631515.0, T);
                double A_H = rate_scale * (2.59e-13 * pow(T / 1.0e4, -0.7));
                double A_HeII = rate_scale * (1.50e-10 * pow(T / 1.0e4, -0.6353));
                double A_HeIII = rate_scale * (3.36e-10 * pow(T / 1.0e4, -0.5));
                double xHII_n = (xHII + dt * ne * C_H * xHI) / (1.0 + dt * ne * A_H);
                double xHeIII_n = ch_clamp((xHeIII + dt * ne * C_HeII * xHeII) / (1.0 + dt * ne * A_HeIII),
                                           0.0, 1.0);
                double xHeII_n = (xHeII + dt * ne * (C_HeI * xHeI + A_HeIII * xHeIII_n)) /
                                 (1.0 + dt * ne * (A_HeII + C_HeII));
                xHII_n = ch_clamp(xHII_n, 0.0, 1.0);
                xHeII_n = ch_clamp(xHeII_n, 0.0, 1.0 - xHeIII_n);
                double dE = energy_scale * (nH * 157809.1 * (xHII_n - xHII) +
                                            nHe * 285335.4 * (xHeII_n - xHeII) +
                                            nHe * 631515.0 * (xHeIII_n - xHeIII));
                double pn = p + (-(gamma - 1.0) * dE / dmax(tunit, CSMALL));
                if (pn < CSMALL) pn = CSMALL;
                P(4, i, j, k) = pn;
                P(off, i, j, k) = xHII_n;
                P(off + 1, i, j, k) = xHeII_n;
                P(off + 2, i, j, k) = xHeIII_n;
            }
}

/* ------------------------------------------------------------------ */
/* causal dissipation (dissipation.py:5-215), interior cells, in place; */
/* work: 10 * nx*ny*nz doubles (the reference's advected copies)        */
/* ------------------------------------------------------------------ */
static double ocap(double x, double cap) {
    if (x > cap) return cap;
    if (x < -cap) return -cap;
    return x;
}
void oracle_causal_dissipation(double* pr, int nv, int nx, int ny, int nz, int ng, double dt,
                               double dx, double dy, double dz, double zeta, double eta,
                               double kappa, double tau_bulk, double tau_shear, double tau_heat,
                               double cap_frac, double pmax, int advect, double* work) {
    OGrid g0 = {nv, nx, ny, nz};
    const OGrid* g = &g0;
    const size_t nc = (size_t)nx * ny * nz;
    const double hx = dmax(dx, 1e-12), hy = dmax(dy, 1e-12), hz = dmax(dz, 1e-12);
    if (advect) {
        memcpy(work, pr + 5 * nc, 10 * nc * sizeof(double));
        for (int i = ng; i < nx - ng; ++i)
            for (int j = ng; j < ny - ng; ++j)
                for (int k = ng; k < nz - ng; ++k) {
                    double vx = P(1, i, j, k), vy = P(2, i, j, k), vz = P(3, i, j, k);
                    for (int v = 5; v < 15; ++v) {
                        double u0 = P(v, i, j, k), ddx, ddy, ddz;
                        if (vx > 0.0) ddx = (u0 - P(v, i - 1, j, k)) / hx;
                        else ddx = (P(v, i + 1, j, k) - u0) / hx;
                        if (vy > 0.0) ddy = (u0 - P(v, i, j - 1, k)) / hy;
                        else ddy = (P(v, i, j + 1, k) - u0) / hy;
                        if (vz > 0.0) ddz = (u0 - P(v, i, j, k - 1)) / hz;
                        else ddz = (P(v, i, j, k + 1) - u0) / hz;
                        work[(size_t)(v - 5) * nc + ((size_t)i * ny + j) * nz + k] =
                            u0 - dt * (vx * ddx + vy * ddy + vz * ddz);
                    }
                }
        memcpy(pr + 5 * nc, work, 10 * nc * sizeof(double));
    }
    const double i2x = 0.5 / hx, i2y = 0.5 / hy, i2z = 0.5 / hz, cap = cap_frac * pmax;
    for (int i = ng; i < nx - ng; ++i)
        for (int j = ng; j < ny - ng; ++j)
            for (int k = ng; k < nz - ng; ++k) {
                double dvx_dx = (P(1, i + 1, j, k) - P(1, i - 1, j, k)) * i2x;
                double dvx_dy = (P(1, i, j + 1, k) - P(1, i, j - 1, k)) * i2y;
                double dvx_dz = (P(1, i, j, k + 1) - P(1, i, j, k - 1)) * i2z;
                double dvy_dx = (P(2, i + 1, j, k) - P(2, i - 1, j, k)) * i2x;
                double dvy_dy = (P(2, i, j + 1, k) - P(2, i, j - 1, k)) * i2y;
                double dvy_dz = (P(2, i, j, k + 1) - P(2, i, j, k - 1)) * i2z;
                double dvz_dx = (P(3, i + 1, j, k) - P(3, i - 1, j, k)) * i2x;
                double dvz_dy = (P(3, i, j + 1, k) - P(3, i, j - 1, k)) * i2y;
                double dvz_dz = (P(3, i, j, k + 1) - P(3, i, j, k - 1)) * i2z;
                double divv = dvx_dx + dvy_dy + dvz_dz;
                if (zeta != 0.0) {
                    double pi_eq = -zeta * divv;
                    P(5, i, j, k) = ocap((P(5, i, j, k) + dt * pi_eq / tau_bulk) / (1.0 + dt / tau_bulk), cap);
                }
                if (eta != 0.0) {
                    double sxx = dvx_dx - (1.0 / 3.0) * divv, syy = dvy_dy - (1.0 / 3.0) * divv;
                    double szz = dvz_dz - (1.0 / 3.0) * divv;
                    double sxy = 0.5 * (dvx_dy + dvy_dx), sxz = 0.5 * (dvx_dz + dvz_dx);
                    double syz = 0.5 * (dvy_dz + dvz_dy);
                    double eq[6] = {-2.0 * eta * sxx, -2.0 * eta * syy, -2.0 * eta * szz,
                                    -2.0 * eta * sxy, -2.0 * eta * sxz, -2.0 * eta * syz};
                    double s6[6];
                    for (int m = 0; m < 6; ++m)
                        s6[m] = (P(6 + m, i, j, k) + dt * eq[m] / tau_shear) / (1.0 + dt / tau_shear);
                    s6[2] = -(s6[0] + s6[1]);
                    for (int m = 0; m < 6; ++m) P(6 + m, i, j, k) = ocap(s6[m], cap);
                }
                if (kappa != 0.0) {
#define OT(a, b, c) (P(4, a, b, c) / dmax(P(0, a, b, c), 1e-12))
                    double dTdx = (OT(i + 1, j, k) - OT(i - 1, j, k)) * i2x;
                    double dTdy = (OT(i, j + 1, k) - OT(i, j - 1, k)) * i2y;
                    double dTdz = (OT(i, j, k + 1) - OT(i, j, k - 1)) * i2z;
#undef OT
                    double eq[3] = {-kappa * dTdx, -kappa * dTdy, -kappa * dTdz};
                    for (int m = 0; m < 3; ++m)
                        P(12 + m, i, j, k) = ocap((P(12 + m, i, j, k) + dt * eq[m] / tau_heat) /
                                                  (1.0 + dt / tau_heat), cap);
                }
            }
}
