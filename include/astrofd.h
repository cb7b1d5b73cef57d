/*
 * astrofd.h -- C ABI of libastrofd_b200.so, the B200 (sm_100a) implementation
 * of AstroFD's per-step finite-volume right-hand side.
 *
 * Conventions
 *   - Every array pointer is DEVICE memory (CUDA global memory on the device
 *     that is current for the calling thread) unless a parameter name ends in
 *     _host.  Primitive blocks are float64, C-contiguous pr[v][i][j][k] with
 *     extents (nv, nx, ny, nz) INCLUDING ghost cells, k fastest -- the layout
 *     of the reference's numpy blocks (solvers/srhd3d_mpi_muscl.py:128).
 *   - `stream` is a cudaStream_t passed as void*; NULL means the legacy
 *     default stream.  All entry points are stream-ordered and asynchronous
 *     unless stated otherwise; none synchronises the device.
 *   - Scratch memory is caller-owned: query its size with the matching
 *     *_workspace_bytes() call and pass a device buffer of at least that size.
 *   - Return value: 0 on success, a negative ASTRO_E* code on failure
 *     (astro_error_string() describes it).  Numerical failures inside kernels
 *     (con2prim falling back, iteration caps) never trap: they are counted in
 *     AstroC2PStats.
 *   - Thread safety: calls on different streams are independent, with two
 *     exceptions that share process-wide state: astro_rhs_static, whose
 *     scratch is one array in the library's device memory shared by every
 *     call on a device, and the astro_prof_start/stop,
 *     astro_debug_set_mma_poll_limit, astro_debug_set_tile_poll_limit and
 *     astro_debug_set_step_polish settings.
 */
#ifndef ASTROFD_B200_H
#define ASTROFD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ASTRO_OK 0
#define ASTRO_E_INVALID (-1)      /* bad argument (null pointer, bad enum)        */
#define ASTRO_E_SHAPE (-2)        /* grid too small for the stencil / ghosts      */
#define ASTRO_E_WORKSPACE (-3)    /* workspace missing or smaller than required    */
#define ASTRO_E_UNSUPPORTED (-4)  /* configuration outside the supported path      */
#define ASTRO_E_CUDA (-5)         /* a CUDA launch or runtime call failed          */

/* physics */
#define ASTRO_SRHD 0
#define ASTRO_RMHD 1
/* reconstruction */
#define ASTRO_RECON_MUSCL 0
#define ASTRO_RECON_PPM 1
#define ASTRO_RECON_WENO 2
/* MUSCL limiter */
#define ASTRO_LIM_MC 0
#define ASTRO_LIM_MINMOD 1
#define ASTRO_LIM_VANLEER 2
/* Riemann solver: SRHD 0 = HLLE, 1 = HLLC; RMHD 0 = HLLE,
 * 1 = "hlld" (HLLC hydro + HLLE field), 2 = "hlld_full" (approximate HLLD) */
#define ASTRO_RIEMANN_HLLE 0
#define ASTRO_RIEMANN_HLLC 1
#define ASTRO_RIEMANN_HLLD 1
#define ASTRO_RIEMANN_HLLD_FULL 2
/* flux_mode */
#define ASTRO_FLUX_REFERENCE 0    /* reproduce the reference's x-face speeds     */
#define ASTRO_FLUX_CONSERVATIVE 1 /* every face evaluated once, from both sides  */
/* precision */
#define ASTRO_PREC_FP64 0         /* everything in float64                        */
#define ASTRO_PREC_MIXED 1        /* reconstruction + Riemann in float32; state,
                                     RK accumulation and con2prim in float64     */
/* con2prim initial guess */
#define ASTRO_GUESS_REFERENCE 0   /* hydro fixed point, as the reference          */
#define ASTRO_GUESS_LEARNED 1     /* MLP guess + <=2 Newton polish, full fallback */

/* Mirrors the keys read by srhd_core.configure (core/srhd_core.py:18-41) and
 * rmhd_core.configure (core/rmhd_core.py:21-50). */
typedef struct AstroParams {
    int32_t physics, recon, limiter, riemann;
    int32_t n_passive, passive_offset, resistive, flux_mode;
    int32_t precision, c2p_guess;
    int32_t fused_stage; /* 1: SSPRK stages of RMHD WENO5/PPM with HLLE or
                            "hlld", float32 faces and conservative fluxes run
                            as one fused kernel per stage (TMA-staged tiles,
                            faces and update together); 0: the per-direction
                            face passes + update (the default; the same
                            result to float32 rounding)                    */
    const void* mlp;     /* device pointer to the learned-guess network's
                            parameter block (astro_mlp_param_bytes() bytes),
                            used when c2p_guess == ASTRO_GUESS_LEARNED        */
    double gamma;        /* RMHD adiabatic index (GAMMA)                      */
    double srhd_gamma;   /* SRHD kernels: the reference freezes this at 5/3   */
    double p_max, v_max, glm_ch, glm_cp, resistivity;
} AstroParams;

typedef struct AstroGrid {
    int32_t nv, nx, ny, nz;   /* extents including ghosts */
    double dx, dy, dz;
} AstroGrid;

/* Nozzle inflow on the left x ghost layers (core/nozzle.py:27-91). */
typedef struct AstroNozzle {
    int32_t ng, profile;        /* profile 0 top_hat, 1 taper, 2 parabolic          */
    int32_t perturb, physics;   /* perturb != 0: draws supplied; physics 1 = rmhd   */
    int32_t b_init;             /* 0 none, 1 poloidal (Bx), 2 toroidal (By = B0 s),
                                   3 B_phi(r) = B0 r/R (r < R), B0 R/r (r >= R),
                                     times s, plus Bx = b_amb_x (no reference
                                     counterpart)                                 */
    int32_t n_tracers, tracer_offset, two_temperature, thermo_offset;
    int32_t ambient_bc;         /* cells with s = 0: 0 the fixed ambient state (the
                                   reference), 1 zero-gradient copy of the first
                                   interior x layer (no reference counterpart)    */
    double radius, shear_thick, gamma_jet, eta_rho, p_eq, rho_amb;
    double vx_amb, vy_amb, vz_amb, turb_vamp, turb_pamp, b0, te, ti;
    double dy, dz, y0, z0;
    double tracer_nozzle[8], tracer_amb[8];
    double b_amb_x;             /* axial ambient field carried through the inlet (b_init 3) */
    int32_t chemistry;          /* CHEMISTRY_ENABLED: the inflow carries the       */
    int32_t chem_offset;        /* ionisation fractions chem_x (xHII, xHeII,       */
    double chem_x[3];           /* xHeIII) at variables chem_offset.. +2            */
} AstroNozzle;

/* con2prim outcome counters accumulated by astro_step/astro_c2p */
typedef struct AstroC2PStats {
    unsigned long long cells;          /* con2prim calls                            */
    unsigned long long newton;         /* converged by Newton (any start)          */
    unsigned long long bisection;      /* reached the bisection fallback            */
    unsigned long long hydro_fallback; /* invalid result -> hydro guess kept        */
    unsigned long long learned_polish; /* learned guess converged within <=2 steps  */
    unsigned long long learned_fallback; /* learned guess failed -> full solve      */
    unsigned long long polish_steps;   /* total polish steps taken                  */
    unsigned long long wait_timeouts;  /* thread blocks whose bounded wait gave up:
                                          a learned-guess block whose tensor-core
                                          wait ran out finishes its cells from
                                          Z = D + tau + B^2 (the result is still the
                                          full solve's); a learned-guess or fused
                                          stage block whose bulk/tile load never
                                          landed leaves its cells unsolved (the
                                          call's result is invalid) */
} AstroC2PStats;

/* --- build / diagnostics ------------------------------------------------ */
int astro_version(void);
const char* astro_error_string(int code);

/* --- right-hand side ----------------------------------------------------
 * Replaces srhd_core.compute_rhs_{muscl,ppm,weno} (core/srhd_core.py:469,927,1167)
 * and rmhd_core.compute_rhs_{rmhd,ppm,weno} (core/rmhd_core.py:749,1280,1440).
 * rhs has extents (nm + n_passive, nx, ny, nz), nm = 5 (SRHD) or 9 (RMHD), and is
 * zero outside the reference's loop bounds. */
size_t astro_rhs_workspace_bytes(const AstroParams* p, const AstroGrid* g);
int astro_rhs(const AstroParams* p, const AstroGrid* g, const double* pr, double* rhs,
              void* work, size_t work_bytes, void* stream);

/* --- right-hand side without caller scratch --------------------------------
 * No counterpart in the reference.  Same result as astro_rhs, for callers
 * that cannot allocate device memory: a host code that binds this library
 * through an FFI (cgo, Fortran, ctypes) and owns only the primitive and rhs
 * arrays it passes, with no device allocator of its own to lend scratch from,
 * or a time-stepping loop that must not call cudaMalloc, which synchronises
 * the device.  The scratch is a fixed array of astro_rhs_static_max_bytes()
 * (32 MiB) in the library's device memory, held by every GPU that loads the
 * library until the process exits.  Grids whose scratch would exceed it are
 * rejected with ASTRO_E_WORKSPACE (e.g. up to ~48^3 cells including ghosts
 * for RMHD WENO in float64 reference mode).  The first call in each CUDA
 * context (each device's primary context, one re-created after
 * cudaDeviceReset, or a driver-API context the caller made current) looks up
 * the array's device address there (cudaGetSymbolAddress, which may load the
 * library's device code) and caches it under that context; make that first
 * call before any stream capture: made on a capturing stream it returns
 * ASTRO_E_INVALID.  All calls on a device share the one array, which keeps
 * the last call's contents: calls that overlap on the GPU (different streams
 * or host threads without ordering) race and must be serialised by the
 * caller.  It calls no cudaMalloc/cudaFree. */
size_t astro_rhs_static_max_bytes(void);
int astro_rhs_static(const AstroParams* p, const AstroGrid* g, const double* pr, double* rhs,
                     void* stream);

/* --- one SSPRK step -----------------------------------------------------
 * Replaces {srhd,rmhd}_core.step_ssprk2/3 (core/srhd_core.py:1286,1334;
 * core/rmhd_core.py:1559,1609): returns the new primitive block in pr_out
 * (pr_in is not modified; pr_out must not alias pr_in).  rk_order is 2 or 3.
 * If stats is non-NULL the step's con2prim counters are added to it (device
 * memory, one AstroC2PStats). */
size_t astro_step_workspace_bytes(const AstroParams* p, const AstroGrid* g);
int astro_step(const AstroParams* p, const AstroGrid* g, const double* pr_in,
               double* pr_out, double dt, int rk_order, void* work, size_t work_bytes,
               AstroC2PStats* stats, void* stream);
/* No reference counterpart: stage `stage` (0 .. rk_order-1) of the same
 * SSPRK step, for callers that refresh ghost layers between stages (an
 * x-slab halo exchange per stage makes a multi-rank run equal to the
 * one-block run; the reference's driver exchanges once per step).  pr_in:
 * the step's input; pr_stage: this stage's input (pr_in itself at stage 0,
 * else the previous stage's pr_out, ghosts possibly refreshed); pr_out
 * distinct from both.  The conserved state between stages lives in `work`
 * (astro_step_workspace_bytes): the stages of one step run in order on the
 * same workspace, with no other call on it in between.  Chained, the stages
 * give astro_step's result exactly. */
int astro_step_stage(const AstroParams* p, const AstroGrid* g, const double* pr_in,
                     const double* pr_stage, double* pr_out, double dt, int rk_order, int stage,
                     void* work, size_t work_bytes, AstroC2PStats* stats, void* stream);

/* Per-kernel-class device time of one step, from CUDA events recorded after
 * every launch.  Classes: 0 face-flux passes, 1 stage update (divergence, RK,
 * and con2prim unless learned), 2 other (ghost fills, reductions, sources),
 * 3 learned con2prim, 4 learned con2prim's fallback solves. */
typedef struct AstroKernelTimes {
    double ms[5];
    int32_t launches[5];
} AstroKernelTimes;

/* astro_step with per-launch event timing filled into *times.  Synchronises
 * the stream before returning (profiling use, e.g. a benchmark's roofline).
 * No counterpart in the reference (which has no device kernels to time). */
int astro_step_profiled(const AstroParams* p, const AstroGrid* g, const double* pr_in,
                        double* pr_out, double dt, int rk_order, void* work, size_t work_bytes,
                        AstroC2PStats* stats, void* stream, AstroKernelTimes* times);

/* Number of kernels this library has launched in the process so far
 * (a diagnostic counter; no counterpart in the reference). */
unsigned long long astro_launch_count(void);
/* Test hook, no counterpart in the reference: polls each tensor-core
 * completion wait of the learned con2prim makes before giving up, for the
 * launches that follow (0 restores the default of 2^26, about a second).
 * A small limit makes the waits give up while the MMAs are still running;
 * the kernels then finish without the network and wait for those MMAs
 * before freeing their tensor memory. */
int astro_debug_set_mma_poll_limit(long long polls);
/* Test hook, no counterpart in the reference: polls each tile-load wait of
 * the fused stage kernel (AstroParams.fused_stage) makes before giving up,
 * for the launches that follow (0 restores the default of 2^24).  A block
 * whose wait gives up stops, waits with the full budget for its loads still
 * in flight, and counts itself in AstroC2PStats.wait_timeouts; its cells are
 * not updated, so that step's result is invalid. */
int astro_debug_set_tile_poll_limit(long long polls);
/* Test hook, no counterpart in the reference: y[i] = the float64 reciprocal
 * of x[i] that the learned con2prim's polish uses in place of IEEE division
 * (a hardware approximation refined by two Newton-Raphson steps), so a test
 * can check its error bound against the IEEE quotient.  Device arrays. */
int astro_debug_rcp_f64(const double* x, double* y, int64_t n, void* stream);
/* Test hook, no counterpart in the reference: Newton polish steps the
 * learned con2prim of astro_step / astro_step_stage / astro_step_gr allows
 * before a cell goes to the reference's complete solve, for the calls that
 * follow (-1 restores the default of 2; 0 sends every cell whose start does
 * not already meet the tolerance to that solve). */
int astro_debug_set_step_polish(int steps);
/* No reference counterpart: kernel-class times over any sequence of this
 * library's calls, without host synchronisation in between.
 * astro_prof_start records an event on `stream`, then one after each of the
 * library's launches made from the calling thread (all on that stream, up to
 * max_launches); astro_prof_stop waits for the last event and charges each
 * gap to its launch's class (classes as in astro_step_profiled). */
int astro_prof_start(int max_launches, void* stream);
int astro_prof_stop(AstroKernelTimes* times);

/* --- CFL speed ----------------------------------------------------------
 * Replaces srhd_core.max_char_speed (core/srhd_core.py:1268): writes the max
 * characteristic speed over i,j,k in [1, n-1) to out (device double). */
size_t astro_max_char_speed_workspace_bytes(void);
int astro_max_char_speed(const AstroParams* p, const AstroGrid* g, const double* pr,
                         double* out, void* work, size_t work_bytes, void* stream);

/* --- ghost fills (in place) ----------------------------------------------
 * Replace boundary.apply_periodic_yz / apply_outflow_right_x
 * (core/boundary.py:4,10) and nozzle.apply_nozzle_left_x (core/nozzle.py:27).
 * draws: 3 uniforms per perturbed nozzle cell in the reference's draw order
 * (g, j, k), or NULL when unperturbed; rank_map: (ny-2ng)*(nz-2ng) int32 giving
 * each interior (j,k) its rank among cells with nozzle weight > 0 (or -1). */
int astro_periodic_yz(double* pr, const AstroGrid* g, int ng, void* stream);
int astro_outflow_right_x(double* pr, const AstroGrid* g, int ng, void* stream);
int astro_nozzle_left_x(double* pr, const AstroGrid* g, const AstroNozzle* nz,
                        const double* draws, const int32_t* rank_map, int32_t n_weighted,
                        void* stream);

/* Zero-gradient ("outflow") ghost fill of the four y and z faces over the
 * whole x extent: every ghost cell takes the value of the nearest interior
 * cell in y and z (the same as copying the y layers first, then the z layers).
 * No counterpart in the reference, whose driver fills y and z periodically
 * (astro_periodic_yz); jet set-ups with outflow on every face but the nozzle
 * use this instead. */
int astro_outflow_yz(double* pr, const AstroGrid* g, int ng, void* stream);

/* --- pointwise conversions ----------------------------------------------
 * Array forms of prim_to_cons / cons_to_prim (core/srhd_core.py:47,62) and
 * prim_to_cons_rmhd / cons_to_prim_rmhd (core/rmhd_core.py:138,249).
 * Arrays are (nm, count) float64.  For these and the batch calls below a
 * count of 0 does nothing and returns ASTRO_OK, with null arrays allowed. */
int astro_p2c(const AstroParams* p, const double* prim, double* cons, int64_t count,
              void* stream);
int astro_c2p(const AstroParams* p, const double* cons, double* prim, int64_t count,
              AstroC2PStats* stats, void* stream);

/* --- learned con2prim initial guess (no counterpart in the reference) ------
 * A 5-64-64-64-2 ReLU network on the invariants (log D, log1p|S|/D,
 * log1p tau/D, log1p B^2/D, log1p (S.B)^2/D^3) predicts log(Z / (D + tau +
 * B^2)) of the solution's Z = rho h W^2 (and log W, a training target only).
 * At most max_polish Newton steps of the reference's update
 * (core/rmhd_core.py:268-292) follow, from the network's Z or, where its
 * first step exceeds 1e-2 Z, from whichever of it and the reference's second
 * start D + tau + B^2 has the shorter first step.
 * Cells whose residual is then still >= 1e-10 max(1, tau) get the reference's
 * complete con2prim.  Evaluation and training use tcgen05 tensor cores (BF16
 * operands, FP32 accumulation).
 * The parameter block is float32: W1[64x5] b1[64] W2[64x64] b2[64] W3[64x64]
 * b3[64] W4[2x64] b4[2] (the astro_mlp_trainable() trainable floats), then
 * xmu[5] xsd[5] ymu[2] ysd[2] (feature / target normalisation).  `status`
 * (device int, may be NULL) is set to 1 if a tensor-core wait timed out. */
size_t astro_mlp_param_bytes(void);
int astro_mlp_trainable(void);
int astro_c2p_features(const double* cons, float* x, int64_t count, void* stream);
int astro_mlp_forward(const void* params, const float* x, float* y, int64_t n, int* status,
                      void* stream);
/* adds d(mean squared error)/d(params) over the n samples into grad
 * (astro_mlp_trainable() floats) and the mean squared error into *loss */
int astro_mlp_train_grad(const void* params, const float* x, const float* t, int64_t n,
                         float* grad, float* loss, int* status, void* stream);
/* one Adam step on the trainable prefix of params; zeroes grad */
int astro_mlp_adam(void* params, float* grad, float* m, float* v, float lr, float beta1,
                   float beta2, float eps, int step, void* stream);
/* con2prim of a (9, count) batch with the learned guess (p->mlp set); with
 * p->mlp == NULL the same polish/fallback runs from Z = D + tau + B^2 (the
 * reference's second Newton start), the no-network comparison.  States whose
 * polish fails get the reference's complete con2prim (cons_to_prim_rmhd,
 * core/rmhd_core.py:249): with a workspace of
 * astro_c2p_learned_workspace_bytes(count) bytes they are listed and solved
 * by a second kernel; with work == NULL inline, where one slow state holds up
 * its 128-state tile. */
size_t astro_c2p_learned_workspace_bytes(int64_t count);  /* 256 + 4 count */
int astro_c2p_learned(const AstroParams* p, const double* cons, double* prim, int64_t count,
                      int max_polish, void* work, size_t work_bytes, AstroC2PStats* stats,
                      int* status, void* stream);

/* --- operator-split post-step sources (core/source_terms.py:5,30) -------- */
int astro_cooling_heating(double* pr, const AstroGrid* g, int ng, double dt, double cool,
                          double heat, double p_max, void* stream);
int astro_two_temperature(double* pr, const AstroGrid* g, int ng, double dt, double tau,
                          int thermo_offset, void* stream);

/* H/He non-equilibrium ionisation on the interior cells, in place: replaces
 * chemistry.apply_ion_chemistry (core/chemistry.py:43).  Species xHII, xHeII,
 * xHeIII at variables chem_offset.. chem_offset+2; implicit recombination,
 * explicit ionisation, the ionisation energy taken from the pressure. */
typedef struct AstroChemistry {
    int32_t ng, chem_offset;
    double x, y;                 /* hydrogen / helium mass fractions         */
    double tunit_k, rate_scale, energy_scale, tmin_k, gamma;
} AstroChemistry;
int astro_ion_chemistry(double* pr, const AstroGrid* g, const AstroChemistry* c, double dt,
                        void* stream);

/* Israel-Stewart causal dissipation of the 15-variable SRHD block, in place:
 * replaces dissipation.apply_causal_dissipation (core/dissipation.py:5).  With
 * advect, first-order upwind advection of pi, pi_ij, q_i (variables 5..14) by
 * the velocity, then relaxation toward the Navier-Stokes targets of bulk
 * (zeta != 0), shear (eta != 0) and heat flux (kappa != 0) with the given
 * relaxation times, capped at cap_frac * p_max.  Scratch:
 * astro_causal_dissipation_workspace_bytes(g) bytes (10 float64 per cell). */
typedef struct AstroDissipation {
    int32_t ng, advect;
    double zeta, eta, kappa, tau_bulk, tau_shear, tau_heat, cap_frac, p_max;
} AstroDissipation;
size_t astro_causal_dissipation_workspace_bytes(const AstroGrid* g);

/* --- run diagnostics (utils/diagnostics.py:5,128) -------------------------
 * Device reductions over the interior of one block (ng ghost layers), into
 * out[6] (device memory, overwritten): max Lorentz factor (v^2 capped below 1
 * as the reference does), the sum of S_x = prim_to_cons(...)[1] over the first
 * interior x layer with adiabatic index `gamma` (multiply by dy dz for the
 * inlet flux; the reference passes no index there, so its module default 5/3
 * applies whatever GAMMA is configured), and for blocks of 8+ variables
 * max |div B|, the sum and the sum of squares of the central-difference div B
 * and the cell count.  Sums are accumulated with atomics: their rounding
 * depends on the order.  No reference counterpart for the MPI reductions. */
int astro_diagnostics(const AstroParams* p, const AstroGrid* g, int ng, const double* pr,
                      double gamma, double* out, void* stream);
int astro_causal_dissipation(double* pr, const AstroGrid* g, const AstroDissipation* c, double dt,
                             void* work, size_t work_bytes, void* stream);

/* --- fixed-metric GR wrappers (core/grhd_core.py, core/grmhd_core.py) -----
 * The SRHD / RMHD right-hand side of p (physics selects GRHD or GRMHD) with
 * the reference's approximate fixed-metric terms (metrics of
 * core/gr_metric.py:6-38, black hole of mass `mass` at the origin, cell
 * centres x = (offs_x + i - ng + 1/2) dx, y = (j - ng + 1/2) dy, ...):
 *  - SCHWARZSCHILD / KERR_SCHILD with orthonormal_flux: the fluxes see the
 *    interior velocities divided by the Kerr-Schild lapse (both metrics, as
 *    the reference; grhd_core.py:22-37);
 *  - every metric but MINKOWSKI: interior sources rhs[S_i] += w dln(alpha)/dx_i,
 *    rhs[tau] += S . grad ln(alpha), w = rho h W^2 + p (+ B^2 for GRMHD), h from
 *    the configured gamma, S from prim_to_cons (grhd_core.py:47-78); the
 *    isotropic Schwarzschild lapse for SCHWARZSCHILD, Kerr-Schild otherwise
 *    (OTHER: any other metric name, which the reference sends down the
 *    Kerr-Schild branch without the rescale).  spin is unused, as there. */
#define ASTRO_GR_MINKOWSKI 0
#define ASTRO_GR_SCHWARZSCHILD 1
#define ASTRO_GR_KERR_SCHILD 2
#define ASTRO_GR_OTHER 3
typedef struct AstroGR {
    int32_t metric, orthonormal_flux;  /* GR_METRIC, ORTHONORMAL_FLUX          */
    int32_t ng, offs_x;                /* ghost layers, first interior x index */
    double mass, spin;                 /* GR_MASS, GR_SPIN                     */
} AstroGR;
/* workspace of astro_rhs_gr (step = 0) or astro_step_gr (step = 1); 0 on a
 * bad configuration */
size_t astro_gr_workspace_bytes(const AstroParams* p, const AstroGrid* g, const AstroGR* gr,
                                int step);
/* compute_rhs_grhd (grhd_core.py:20) / compute_rhs_grmhd (grmhd_core.py:20) */
int astro_rhs_gr(const AstroParams* p, const AstroGrid* g, const AstroGR* gr, const double* pr,
                 double* rhs, void* work, size_t work_bytes, void* stream);
/* step_ssprk2/3 (grhd_core.py:76,124; grmhd_core.py:80,...): the core step
 * with the GR right-hand side; the learned con2prim guess works as in
 * astro_step */
int astro_step_gr(const AstroParams* p, const AstroGrid* g, const AstroGR* gr,
                  const double* pr_in, double* pr_out, double dt, int rk_order, void* work,
                  size_t work_bytes, AstroC2PStats* stats, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* ASTROFD_B200_H */
