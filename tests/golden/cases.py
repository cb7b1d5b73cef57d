"""Parity cases shared by the fixture generator and the tests.

Test infrastructure only.  Each case names one configuration of the
reference's hot path (physics x reconstruction x limiter x Riemann solver x
SSPRK order, plus passives / resistivity) on a small seeded state from
``states.make_state``.  Parameter keys are the reference's own config keys
(reference: utils/settings.py:13-258, core/srhd_core.py:18-41,
core/rmhd_core.py:21-50).
"""

BASE_SRHD = dict(GAMMA=5.0 / 3.0, P_MAX=2.0, V_MAX=0.9999)
BASE_RMHD = dict(GAMMA=4.0 / 3.0, P_MAX=2.0, V_MAX=0.9999, GLM_CH=1.0,
                 GLM_CP=0.1)


def _c(name, physics, recon, limiter, riemann, rk, ng, n_extra=0, seed=None,
       n=8, pad=0, state=None, **extra):
    base = BASE_SRHD if physics == "srhd" else BASE_RMHD
    params = dict(base)
    params.update(RECON=recon, LIMITER=limiter, RIEMANN=riemann, RK_ORDER=rk,
                  NG=ng, N_PASSIVE=n_extra,
                  PASSIVE_OFFSET=5 if physics == "srhd" else 9)
    params.update(extra)
    # pad: extra non-passive variables appended after the passives.  The
    # reference's MUSCL passive stencils read one row past the last variable
    # (undefined behaviour there); a padding variable makes that read defined.
    return dict(name=name, physics=physics, params=params, n=n, ng=ng,
                n_extra=n_extra, pad=pad, seed=seed, rk=rk, state=state or {})



# The reference's experimental HLLD (rmhd_core.py:602) is unstable on the
# roughest states (fields grow to 1e10 within a step and con2prim falls back
# to bisection), so its cases use milder, jet-like states.
MILD = dict(noise=0.05, bamp=0.05, vjet=0.9, stripes=False)

# seeds are fixed integers so fixture regeneration is reproducible
CASES = [
    # ---- SRHD --------------------------------------------------------
    _c("s_muscl_minmod_hlle_rk2", "srhd", "muscl", "minmod", "hlle", 2, 2, seed=101),
    _c("s_muscl_mc_hllc_rk3", "srhd", "muscl", "mc", "hllc", 3, 2, seed=102),
    _c("s_muscl_vanleer_hlle_rk2", "srhd", "muscl", "vanleer", "hlle", 2, 3, seed=103),
    _c("s_ppm_hllc_rk3", "srhd", "ppm", "mc", "hllc", 3, 3, seed=104),
    _c("s_ppm_hlle_rk2", "srhd", "ppm", "mc", "hlle", 2, 3, seed=105),
    _c("s_weno_hlle_rk3", "srhd", "weno", "mc", "hlle", 3, 3, seed=106),
    _c("s_weno_hllc_rk2", "srhd", "weno", "mc", "hllc", 2, 3, seed=107),
    _c("s_muscl_mc_hlle_pass2", "srhd", "muscl", "mc", "hlle", 2, 3, n_extra=2, seed=108),
    _c("s_muscl_vanleer_hllc_pass1", "srhd", "muscl", "vanleer", "hllc", 3, 2, n_extra=1, seed=109),
    _c("s_ppm_hllc_pass2", "srhd", "ppm", "minmod", "hllc", 3, 3, n_extra=2, seed=110),
    # configured Gamma=4/3 is ignored by the SRHD kernels (frozen default arg)
    _c("s_muscl_mc_hlle_gamma43", "srhd", "muscl", "mc", "hlle", 2, 2, seed=111,
       GAMMA=4.0 / 3.0),
    # Israel-Stewart blocks (15+ variables, passives from 15): bulk pressure
    # added to the MUSCL face pressures, dissipation fluxes once (MUSCL),
    # twice (PPM) or not at all (WENO), fields 5..14 carried by the step
    _c("s_muscl_mc_hlle_is", "srhd", "muscl", "mc", "hlle", 2, 2, seed=112,
       state=dict(n_is=10), PASSIVE_OFFSET=15),
    _c("s_muscl_minmod_hllc_is_pass1", "srhd", "muscl", "minmod", "hllc", 3, 3, n_extra=1,
       pad=1, seed=113, state=dict(n_is=10), PASSIVE_OFFSET=15),
    _c("s_ppm_hllc_is", "srhd", "ppm", "mc", "hllc", 3, 3, seed=114, state=dict(n_is=10),
       PASSIVE_OFFSET=15),
    _c("s_weno_hlle_is", "srhd", "weno", "mc", "hlle", 2, 3, seed=115, state=dict(n_is=10),
       PASSIVE_OFFSET=15),
    # ---- RMHD --------------------------------------------------------
    _c("r_muscl_mc_hlle_rk2", "rmhd", "muscl", "mc", "hlle", 2, 2, seed=201),
    _c("r_muscl_minmod_hlld_rk2", "rmhd", "muscl", "minmod", "hlld", 2, 2, seed=202),
    _c("r_muscl_vanleer_hlldfull_rk3", "rmhd", "muscl", "vanleer", "hlld_full", 3, 3, seed=203, state=MILD),
    _c("r_muscl_mc_hlld_resist_pass1", "rmhd", "muscl", "mc", "hlld", 3, 3, n_extra=1,
       seed=204, pad=1, RESISTIVE_ENABLED=True, RESISTIVITY=1e-3),
    _c("r_ppm_hlle_rk2", "rmhd", "ppm", "mc", "hlle", 2, 3, seed=205),
    _c("r_ppm_hlld_rk3", "rmhd", "ppm", "mc", "hlld", 3, 3, seed=206),
    _c("r_ppm_hlldfull_resist_rk3", "rmhd", "ppm", "mc", "hlld_full", 3, 3, seed=207, state=MILD,
       RESISTIVE_ENABLED=True, RESISTIVITY=1e-3),
    _c("r_weno_hlle_rk3", "rmhd", "weno", "mc", "hlle", 3, 3, seed=208),
    _c("r_weno_hlld_rk3", "rmhd", "weno", "mc", "hlld", 3, 3, seed=209),
    _c("r_weno_hlldfull_rk3", "rmhd", "weno", "mc", "hlld_full", 3, 3, seed=210, state=MILD),
    # C5-like: two passive thermo fields, resistivity on (a no-op in the
    # reference's WENO right-hand side)
    _c("r_weno_hlldfull_c5", "rmhd", "weno", "mc", "hlld_full", 3, 3, n_extra=2, seed=211,
       state=MILD,
       RESISTIVE_ENABLED=True, RESISTIVITY=1e-4),
    _c("r_muscl_mc_hlle_gamma53", "rmhd", "muscl", "mc", "hlle", 2, 2, seed=212,
       GAMMA=5.0 / 3.0),
]

# Non-cubic blocks (the x-slabs of the reference's MPI driver have unequal
# extents), with dx = 1/nx, dy = 1/ny, dz = 1/nz all different, and blocks
# with a single updated layer in one direction.
CASES += [
    _c("s_muscl_mc_hllc_ragged", "srhd", "muscl", "mc", "hllc", 3, 2, seed=121, n=(5, 9, 7)),
    _c("s_weno_hlle_ragged", "srhd", "weno", "mc", "hlle", 2, 3, seed=122, n=(9, 4, 6)),
    _c("s_ppm_hlle_ragged_pass1", "srhd", "ppm", "mc", "hlle", 3, 3, n_extra=1, seed=123,
       n=(6, 7, 5)),
    # SRHD MUSCL updates [2, n-3): of two interior x cells only the first
    _c("s_muscl_minmod_hlle_thin", "srhd", "muscl", "minmod", "hlle", 2, 2, seed=124,
       n=(2, 6, 5)),
    _c("r_weno_hlld_ragged", "rmhd", "weno", "mc", "hlld", 3, 3, seed=221, n=(6, 10, 5)),
    _c("r_muscl_mc_hlle_ragged_resist", "rmhd", "muscl", "mc", "hlle", 2, 2, seed=222,
       n=(11, 5, 8), RESISTIVE_ENABLED=True, RESISTIVITY=1e-3),
    _c("r_ppm_hlld_ragged", "rmhd", "ppm", "mc", "hlld", 2, 3, seed=223, n=(4, 6, 9)),
    _c("r_weno_hlle_thin", "rmhd", "weno", "mc", "hlle", 3, 3, seed=224, n=(5, 3, 1)),
]

CASE_BY_NAME = {c["name"]: c for c in CASES}


def sizes(c):
    """Interior cells (nx, ny, nz) of a case."""
    n = c["n"]
    return (n, n, n) if isinstance(n, int) else tuple(n)


def spacing(c):
    """(dx, dy, dz) of a case: the unit box over its interior cells."""
    return tuple(1.0 / m for m in sizes(c))


def step_dt(c):
    """dt of the single-step fixtures."""
    return DT_FRACTION * min(spacing(c))


def _gr(name, physics, recon, limiter, riemann, rk, ng, gr, offs_x, seed, **kw):
    c = _c(name, physics, recon, limiter, riemann, rk, ng, seed=seed, **kw)
    c.update(gr=gr, offs_x=offs_x)
    return c


# Fixed-metric GR wrappers (core/grhd_core.py, core/grmhd_core.py): black hole
# of mass 0.05 at the origin, the block's corner next to it (r >= 0.1, lapse
# >= 0.7), jets at v = 0.5 so that the lapse-rescaled velocities stay below 1
GR_STATE = dict(vjet=0.5)
GR_CASES = [
    _gr("gr_hd_schw_muscl", "srhd", "muscl", "mc", "hlle", 2, 2,
        dict(GR_METRIC="schwarzschild", GR_MASS=0.05, ORTHONORMAL_FLUX=True), 2, 301,
        state=GR_STATE, GAMMA=4.0 / 3.0),
    _gr("gr_hd_ks_ppm_plainflux", "srhd", "ppm", "mc", "hllc", 3, 3,
        dict(GR_METRIC="kerr-schild", GR_MASS=0.05, ORTHONORMAL_FLUX=False), 0, 302,
        state=GR_STATE),
    _gr("gr_hd_other_muscl_pass1", "srhd", "muscl", "vanleer", "hllc", 3, 2,
        dict(GR_METRIC="isotropic", GR_MASS=0.05, ORTHONORMAL_FLUX=True), 1, 303,
        n_extra=1, state=GR_STATE),
    _gr("gr_mhd_schw_weno", "rmhd", "weno", "mc", "hlld", 3, 3,
        dict(GR_METRIC="schwarzschild", GR_MASS=0.05, ORTHONORMAL_FLUX=True), 1, 304,
        state=dict(MILD, vjet=0.5)),
    _gr("gr_mhd_ks_muscl", "rmhd", "muscl", "mc", "hlle", 2, 2,
        dict(GR_METRIC="kerr-schild", GR_MASS=0.05, ORTHONORMAL_FLUX=True, GR_SPIN=0.5), 3, 305,
        state=dict(MILD, vjet=0.5)),
    _gr("gr_mhd_mink_ppm", "rmhd", "ppm", "mc", "hlld", 2, 3,
        dict(GR_METRIC="minkowski", GR_MASS=0.05), 0, 306, state=dict(MILD, vjet=0.5)),
]
GR_BY_NAME = {c["name"]: c for c in GR_CASES}

DT_FRACTION = 0.2  # dt = DT_FRACTION * dx for the single-step fixtures
