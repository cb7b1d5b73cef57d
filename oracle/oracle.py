"""ctypes front end of the C parity oracle (astro_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py as the checker / timed CPU baseline.  The
astrofd_b200 product never imports this module.

The functions mirror the reference's Python call surface
(core/srhd_core.py, core/rmhd_core.py, core/boundary.py, core/nozzle.py,
core/source_terms.py) on numpy float64 arrays.
"""
import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


class OParams(C.Structure):
    _fields_ = [("physics", C.c_int), ("recon", C.c_int), ("limiter", C.c_int),
                ("riemann", C.c_int), ("n_passive", C.c_int),
                ("passive_offset", C.c_int), ("resistive", C.c_int),
                ("flux_mode", C.c_int), ("gamma", C.c_double), ("p_max", C.c_double),
                ("v_max", C.c_double), ("glm_ch", C.c_double),
                ("glm_cp", C.c_double), ("resistivity", C.c_double)]


class OGR(C.Structure):
    _fields_ = [("metric", C.c_int), ("orthonormal", C.c_int), ("ng", C.c_int),
                ("offs_x", C.c_int), ("mass", C.c_double), ("spin", C.c_double)]


GR_METRICS = {"minkowski": 0, "schwarzschild": 1, "kerr-schild": 2}


def gr_struct(cfg, ng, offs_x):
    """GR_METRIC / GR_MASS / GR_SPIN / ORTHONORMAL_FLUX as grhd_core.configure
    reads them (grhd_core.py:13-18); any other metric name goes down the
    reference's Kerr-Schild source branch without the velocity rescale."""
    g = OGR()
    g.metric = GR_METRICS.get(str(cfg.get("GR_METRIC", "minkowski")).lower(), 3)
    g.orthonormal = 1 if bool(cfg.get("ORTHONORMAL_FLUX", True)) else 0
    g.ng, g.offs_x = int(ng), int(offs_x)
    g.mass, g.spin = float(cfg.get("GR_MASS", 1.0)), float(cfg.get("GR_SPIN", 0.0))
    return g


class ONozzle(C.Structure):
    _fields_ = [("ng", C.c_int), ("profile", C.c_int), ("perturb", C.c_int),
                ("physics", C.c_int), ("b_init", C.c_int), ("n_tracers", C.c_int),
                ("tracer_offset", C.c_int), ("two_temperature", C.c_int),
                ("thermo_offset", C.c_int), ("ambient_bc", C.c_int),
                ("radius", C.c_double), ("shear_thick", C.c_double),
                ("gamma_jet", C.c_double), ("eta_rho", C.c_double),
                ("p_eq", C.c_double), ("rho_amb", C.c_double),
                ("vx_amb", C.c_double), ("vy_amb", C.c_double),
                ("vz_amb", C.c_double), ("turb_vamp", C.c_double),
                ("turb_pamp", C.c_double), ("b0", C.c_double), ("te", C.c_double),
                ("ti", C.c_double), ("tracer_nozzle", C.c_double * 8),
                ("tracer_amb", C.c_double * 8), ("b_amb_x", C.c_double),
                ("chemistry", C.c_int), ("chem_offset", C.c_int),
                ("chem_x", C.c_double * 3)]


_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        L.oracle_rhs.argtypes = [C.POINTER(OParams), dp, C.c_int, C.c_int, C.c_int,
                                 C.c_int, C.c_double, C.c_double, C.c_double, dp]
        L.oracle_step.argtypes = [C.POINTER(OParams), dp, C.c_int, C.c_int, C.c_int,
                                  C.c_int, C.c_double, C.c_double, C.c_double,
                                  C.c_double, C.c_int, dp]
        L.oracle_rhs_gr.argtypes = [C.POINTER(OParams), C.POINTER(OGR), dp, C.c_int, C.c_int,
                                    C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, dp]
        L.oracle_step_gr.argtypes = [C.POINTER(OParams), C.POINTER(OGR), dp, C.c_int, C.c_int,
                                     C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                     C.c_double, C.c_int, dp]
        L.oracle_stage.argtypes = [C.POINTER(OParams), dp, dp, dp, C.c_int, C.c_int, C.c_int,
                                   C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                   C.c_int, C.c_int, dp]
        L.oracle_p2c.argtypes = [C.POINTER(OParams), dp, dp, C.c_long]
        L.oracle_c2p.argtypes = [C.POINTER(OParams), dp, dp, C.c_long]
        L.oracle_c2p_counters.argtypes = [C.POINTER(C.c_long), C.c_int]
        L.oracle_max_char_speed.argtypes = [dp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.oracle_max_char_speed.restype = C.c_double
        for f in (L.oracle_periodic_yz, L.oracle_outflow_right_x, L.oracle_outflow_yz):
            f.argtypes = [dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.oracle_nozzle_left_x.argtypes = [dp, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.c_double, C.c_double, C.c_int, C.c_int,
                                           C.c_double, C.c_double,
                                           C.POINTER(ONozzle), dp]
        L.oracle_nozzle_left_x.restype = C.c_long
        L.oracle_ion_chemistry.argtypes = [dp] + [C.c_int] * 6 + [C.c_double] * 8
        L.oracle_causal_dissipation.argtypes = ([dp] + [C.c_int] * 5 + [C.c_double] * 12 +
                                                [C.c_int, dp])
        L.oracle_cooling.argtypes = [dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                     C.c_double, C.c_double, C.c_double, C.c_double]
        L.oracle_two_temperature.argtypes = [dp, C.c_int, C.c_int, C.c_int, C.c_int,
                                             C.c_int, C.c_double, C.c_double, C.c_int]
        L.oracle_num_threads.restype = C.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


_RECON = {"muscl": 0, "ppm": 1, "weno": 2}
_LIMITER = {"mc": 0, "minmod": 1, "vanleer": 2}


def params_from_config(physics, cfg):
    """Restates configure() (srhd_core.py:18-41, rmhd_core.py:21-50)."""
    p = OParams()
    p.physics = 0 if physics == "srhd" else 1
    p.recon = _RECON.get(str(cfg.get("RECON", "muscl")).lower(), 0)
    p.limiter = _LIMITER.get(str(cfg.get("LIMITER", "mc")).lower(), 0)
    r = str(cfg.get("RIEMANN", "hlle")).lower()
    if physics == "srhd":
        p.riemann = 1 if r == "hllc" else 0
    else:
        p.riemann = 2 if r == "hlld_full" else (1 if r == "hlld" else 0)
    p.n_passive = int(cfg.get("N_PASSIVE", 0))
    p.passive_offset = int(cfg.get("PASSIVE_OFFSET", 5 if physics == "srhd" else 9))
    p.resistive = 1 if cfg.get("RESISTIVE_ENABLED", False) else 0
    p.gamma = float(cfg.get("GAMMA", 5.0 / 3.0))
    p.p_max = float(cfg.get("P_MAX", 1.0))
    p.v_max = float(cfg.get("V_MAX", 0.999))
    p.glm_ch = float(cfg.get("GLM_CH", 1.0))
    p.glm_cp = float(cfg.get("GLM_CP", 0.1))
    p.resistivity = float(cfg.get("RESISTIVITY", 0.0))
    p.flux_mode = 1 if str(cfg.get("FLUX_MODE", "reference")).lower() == "conservative" else 0
    return p


def rhs(params, pr, dx, dy, dz):
    pr = np.ascontiguousarray(pr, dtype=np.float64)
    nm = 5 if params.physics == 0 else 9
    out = np.zeros((nm + params.n_passive,) + pr.shape[1:])
    rc = lib().oracle_rhs(C.byref(params), _dp(pr), *pr.shape, dx, dy, dz, _dp(out))
    if rc != 0:
        raise RuntimeError(f"oracle_rhs failed ({rc})")
    return out


def step(params, pr, dx, dy, dz, dt, rk):
    pr = np.ascontiguousarray(pr, dtype=np.float64)
    out = np.zeros_like(pr)
    rc = lib().oracle_step(C.byref(params), _dp(pr), *pr.shape, dx, dy, dz, dt, rk, _dp(out))
    if rc != 0:
        raise RuntimeError(f"oracle_step failed ({rc})")
    return out


def stage(params, pr, prk, Uk, dx, dy, dz, dt, rk, st):
    """Stage st of the SSPRK step from pr; Uk (nm x cells, float64) carries the
    conserved state between the calls of one step (updated in place)."""
    pr = np.ascontiguousarray(pr, dtype=np.float64)
    prk = np.ascontiguousarray(prk, dtype=np.float64)
    assert Uk.flags.c_contiguous and Uk.dtype == np.float64
    out = np.zeros_like(pr)
    rc = lib().oracle_stage(C.byref(params), _dp(pr), _dp(prk), _dp(Uk), *pr.shape, dx, dy, dz,
                            dt, rk, st, _dp(out))
    if rc != 0:
        raise RuntimeError(f"oracle_stage failed ({rc})")
    return out


def rhs_gr(params, gr, pr, dx, dy, dz):
    pr = np.ascontiguousarray(pr, dtype=np.float64)
    nm = 5 if params.physics == 0 else 9
    out = np.zeros((nm + params.n_passive,) + pr.shape[1:])
    rc = lib().oracle_rhs_gr(C.byref(params), C.byref(gr), _dp(pr), *pr.shape, dx, dy, dz,
                             _dp(out))
    if rc != 0:
        raise RuntimeError(f"oracle_rhs_gr failed ({rc})")
    return out


def step_gr(params, gr, pr, dx, dy, dz, dt, rk):
    pr = np.ascontiguousarray(pr, dtype=np.float64)
    out = np.zeros_like(pr)
    rc = lib().oracle_step_gr(C.byref(params), C.byref(gr), _dp(pr), *pr.shape, dx, dy, dz, dt,
                              rk, _dp(out))
    if rc != 0:
        raise RuntimeError(f"oracle_step_gr failed ({rc})")
    return out


def p2c(params, q):
    q = np.ascontiguousarray(q, dtype=np.float64)
    out = np.zeros_like(q)
    lib().oracle_p2c(C.byref(params), _dp(q), _dp(out), q.shape[1])
    return out


def c2p(params, U):
    U = np.ascontiguousarray(U, dtype=np.float64)
    out = np.zeros_like(U)
    lib().oracle_c2p(C.byref(params), _dp(U), _dp(out), U.shape[1])
    return out


def c2p_counters(reset=True):
    a = (C.c_long * 3)()
    lib().oracle_c2p_counters(a, 1 if reset else 0)
    return dict(newton=a[0], bisect=a[1], hydro_fallback=a[2])


def max_char_speed(pr):
    pr = np.ascontiguousarray(pr, dtype=np.float64)
    return lib().oracle_max_char_speed(_dp(pr), *pr.shape)


def apply_periodic_yz(pr, ng):
    assert pr.flags.c_contiguous and pr.dtype == np.float64
    lib().oracle_periodic_yz(_dp(pr), *pr.shape, ng)


def apply_outflow_yz(pr, ng):
    """Zero-gradient y and z faces (an extension; the reference has none)."""
    assert pr.flags.c_contiguous and pr.dtype == np.float64
    lib().oracle_outflow_yz(_dp(pr), *pr.shape, ng)


def apply_outflow_right_x(pr, ng):
    assert pr.flags.c_contiguous and pr.dtype == np.float64
    lib().oracle_outflow_right_x(_dp(pr), *pr.shape, ng)


_PROFILE = {"taper": 1, "smooth": 1, "parabolic": 2, "parabola": 2}


def nozzle_struct(cfg):
    c = ONozzle()
    c.ng = int(cfg["NG"])
    c.profile = _PROFILE.get(cfg.get("NOZZLE_PROFILE", "top_hat"), 0)
    c.perturb = 0 if cfg.get("NOZZLE_PERTURB", "none") == "none" else 1
    c.physics = 1 if cfg.get("PHYSICS") in ("rmhd", "grmhd") else 0
    b = cfg.get("B_INIT")
    c.b_init = {"poloidal": 1, "toroidal": 2, "toroidal_phi": 3}.get(b, 0)
    c.ambient_bc = 1 if cfg.get("NOZZLE_AMBIENT", "fixed") == "outflow" else 0
    c.b_amb_x = float(cfg.get("B_AMB_X", 0.0))
    c.n_tracers = int(cfg.get("N_TRACERS", 0))
    c.tracer_offset = int(cfg.get("TRACER_OFFSET", 5))
    c.two_temperature = 1 if cfg.get("TWO_TEMPERATURE", False) else 0
    c.thermo_offset = int(cfg.get("THERMO_OFFSET", 0))
    c.radius = cfg["JET_RADIUS"]
    c.shear_thick = cfg["SHEAR_THICK"]
    c.gamma_jet = cfg["GAMMA_JET"]
    c.eta_rho = cfg["ETA_RHO"]
    c.p_eq = cfg["P_EQ"]
    c.rho_amb = cfg["RHO_AMB"]
    c.vx_amb, c.vy_amb, c.vz_amb = cfg["VX_AMB"], cfg["VY_AMB"], cfg["VZ_AMB"]
    c.turb_vamp = cfg.get("TURB_VAMP", 0.0)
    c.turb_pamp = cfg.get("TURB_PAMP", 0.0)
    c.b0 = cfg.get("B0", 0.0)
    c.te = float(cfg.get("TE_NOZZLE", cfg.get("TE_AMB", 0.0)) or 0.0)
    c.ti = float(cfg.get("TI_NOZZLE", cfg.get("TI_AMB", 0.0)) or 0.0)
    # the inflow's ionisation fractions, read only with chemistry on (the
    # reference's settings leave them None otherwise)
    c.chemistry = 1 if cfg.get("CHEMISTRY_ENABLED", False) else 0
    if c.chemistry:
        c.chem_offset = int(cfg.get("CHEM_OFFSET", 0))
        for m, key in enumerate(("CHEM_X_HII_NOZZLE", "CHEM_X_HEII_NOZZLE",
                                 "CHEM_X_HEIII_NOZZLE")):
            c.chem_x[m] = float(cfg.get(key, 0.0))
    nv = cfg.get("TRACER_NOZZLE_VALUES", []) or []
    av = cfg.get("TRACER_AMB_VALUES", []) or []
    for t in range(min(c.n_tracers, 8)):
        c.tracer_nozzle[t] = nv[t] if t < len(nv) else (1.0 if t == 0 else 0.0)
        c.tracer_amb[t] = av[t] if t < len(av) else 0.0
    return c


def nozzle_draw_count(cfg, dy, dz, ny_loc, nz_loc, y0, z0):
    """Number of rng.random() draws apply_nozzle_left_x makes (nozzle.py:50-53)."""
    if cfg.get("NOZZLE_PERTURB", "none") == "none":
        return 0
    from_weight = 0
    ng = cfg["NG"]
    prof = cfg.get("NOZZLE_PROFILE", "top_hat")
    for j in range(ng, ng + ny_loc):
        y = (j - ng + 0.5) * dy
        for k in range(ng, ng + nz_loc):
            z = (k - ng + 0.5) * dz
            rr = math.sqrt((y - y0) ** 2 + (z - z0) ** 2)
            if _weight(rr, cfg["JET_RADIUS"], cfg["SHEAR_THICK"], prof) > 0.0:
                from_weight += 1
    return 3 * ng * from_weight


def _weight(r, radius, shear, profile):
    if radius <= 0.0:
        return 0.0
    if profile in ("taper", "smooth"):
        return 0.0 if r >= radius else 0.5 * (1.0 + math.cos(math.pi * r / radius))
    if profile in ("parabolic", "parabola"):
        if r >= radius:
            return 0.0
        x = r / radius
        return max(0.0, 1.0 - x * x)
    if shear > 0.0:
        return 0.5 * (1.0 - math.tanh((r - radius) / shear))
    return 1.0 if r <= radius else 0.0


def apply_nozzle_left_x(pr, dx, dy, dz, ny_loc, nz_loc, y0, z0, rng, cfg):
    assert pr.flags.c_contiguous and pr.dtype == np.float64
    c = nozzle_struct(cfg)
    n = nozzle_draw_count(cfg, dy, dz, ny_loc, nz_loc, y0, z0)
    rnd = rng.random(n) if n > 0 else np.zeros(1)
    used = lib().oracle_nozzle_left_x(_dp(pr), *pr.shape, dy, dz, ny_loc, nz_loc, y0, z0,
                                      C.byref(c), _dp(rnd))
    assert used == n, (used, n)


def apply_ion_chemistry(pr, dt, cfg):
    """chemistry.apply_ion_chemistry (core/chemistry.py:43), with its gating."""
    if not cfg.get("CHEMISTRY_ENABLED", False) or int(cfg.get("N_CHEM", 0)) < 3:
        return pr
    off = int(cfg.get("CHEM_OFFSET", 0))
    if pr.shape[0] <= off + 2:
        return pr
    assert pr.flags.c_contiguous and pr.dtype == np.float64
    lib().oracle_ion_chemistry(_dp(pr), *pr.shape, int(cfg.get("NG", 2)), off, float(dt),
                               float(cfg.get("CHEM_X", 0.76)), float(cfg.get("CHEM_Y", 0.24)),
                               float(cfg.get("CHEM_TUNIT_K", 1.0e4)),
                               float(cfg.get("CHEM_RATE_SCALE", 1.0)),
                               float(cfg.get("CHEM_ENERGY_SCALE", 1.0)),
                               float(cfg.get("CHEM_TMIN_K", 1.0)),
                               float(cfg.get("GAMMA", 5.0 / 3.0)))
    return pr


def dissipation_taus(cfg):
    """The reference's relaxation times: a per-channel key, else RELAX_TAU
    (a zero per-channel value also falls back), core/dissipation.py:18-20."""
    base = cfg.get("RELAX_TAU", 0.1)
    return tuple(float(cfg.get(k, base) or base)
                 for k in ("RELAX_TAU_BULK", "RELAX_TAU_SHEAR", "RELAX_TAU_HEAT"))


def apply_causal_dissipation(pr, dt, dx, dy, dz, cfg):
    """dissipation.apply_causal_dissipation (core/dissipation.py:5)."""
    if not cfg.get("DISSIPATION_ENABLED", False) or cfg.get("PHYSICS") not in ("hydro", "grhd"):
        return pr
    zeta, eta, kappa = (float(cfg.get(k, 0.0)) for k in ("BULK_ZETA", "SHEAR_ETA", "HEAT_KAPPA"))
    tb, ts, th = dissipation_taus(cfg)
    if (zeta == 0.0 and eta == 0.0 and kappa == 0.0) or min(tb, ts, th) <= 0.0 or pr.shape[0] < 15:
        return pr
    assert pr.flags.c_contiguous and pr.dtype == np.float64
    work = np.empty((10,) + pr.shape[1:])
    lib().oracle_causal_dissipation(_dp(pr), *pr.shape, int(cfg.get("NG", 2)), float(dt),
                                    float(dx), float(dy), float(dz), zeta, eta, kappa, tb, ts, th,
                                    float(cfg.get("DISSIPATION_CAP_FRAC", 0.5)),
                                    float(cfg.get("P_MAX", 1.0)),
                                    1 if bool(cfg.get("DISSIPATION_ADVECT", True)) else 0,
                                    _dp(work))
    return pr


def apply_cooling_heating(pr, dt, cfg):
    if not cfg.get("COOLING_ENABLED", False):
        return pr
    lib().oracle_cooling(_dp(pr), *pr.shape, int(cfg.get("NG", 2)), dt,
                         float(cfg.get("COOLING_LAMBDA", 0.0)),
                         float(cfg.get("HEATING_RATE", 0.0)), float(cfg.get("P_MAX", 1.0)))
    return pr


def apply_two_temperature(pr, dt, cfg):
    if not cfg.get("TWO_TEMPERATURE", False):
        return pr
    lib().oracle_two_temperature(_dp(pr), *pr.shape, int(cfg.get("NG", 2)), dt,
                                 float(cfg.get("TEI_TAU", 0.5)),
                                 int(cfg.get("THERMO_OFFSET", 0)))
    return pr


def diagnostics(pr, dx, dy, dz, ng, is_rmhd, v_max=0.999, p_max=1.0):
    """One rank's diagnostics, restating utils/diagnostics.py: max Gamma
    (:14-25) and the inlet flux accumulated cell by cell in (j, k) order
    (:29-42) with prim_to_cons at its default adiabatic index 5/3; div B
    (:141-160) with the reference's numpy max / sum over the (i, j, k)-ordered
    values; the centreline (:72-99).  Dict of the values."""
    pr = np.ascontiguousarray(pr, dtype=np.float64)
    inner = (slice(ng, pr.shape[1] - ng), slice(ng, pr.shape[2] - ng), slice(ng, pr.shape[3] - ng))
    vx, vy, vz = (pr[v][inner] for v in (1, 2, 3))
    v2 = vx * vx + vy * vy + vz * vz
    v2 = np.where(v2 >= 1.0, 1.0 - 1e-14, v2)
    out = dict(max_gamma=float(np.max(1.0 / np.sqrt(1.0 - v2))) if v2.size else 0.0)
    nm = 9 if is_rmhd else 5
    q = pr[:nm, ng, inner[1], inner[2]].reshape(nm, -1)
    P = params_from_config("rmhd" if is_rmhd else "srhd",
                           dict(GAMMA=5.0 / 3.0, V_MAX=v_max, P_MAX=p_max))
    sx = p2c(P, q)[1]
    flux = 0.0
    for s in sx:
        flux += s * dy * dz
    out["inlet_flux"] = flux
    out["inlet_sx"] = float(math.fsum(sx))
    if pr.shape[0] >= 8:
        i, j, k = inner
        sh = lambda v, a, d: pr[v][tuple(slice(s.start + d, s.stop + d) if ax == a else s
                                          for ax, s in enumerate(inner))]
        d = ((sh(5, 0, 1) - sh(5, 0, -1)) / (2.0 * dx) + (sh(6, 1, 1) - sh(6, 1, -1)) / (2.0 * dy)
             + (sh(7, 2, 1) - sh(7, 2, -1)) / (2.0 * dz)).ravel()
        n = d.size
        out.update(divb_max=float(np.max(np.abs(d))) if n else 0.0, divb_sum=float(np.sum(d)),
                   divb_sumsq=float(np.sum(d * d)), divb_n=n)
        out["divb_mean"] = out["divb_sum"] / n if n else 0.0
        out["divb_rms"] = float(np.sqrt(out["divb_sumsq"] / n)) if n else 0.0
    return out


def centerline(pr, ng, v_max):
    """(Gamma, rho, p, vx) of utils/diagnostics.py:72-99 for one rank."""
    ny, nz = pr.shape[2] - 2 * ng, pr.shape[3] - 2 * ng
    j, k = ng + ny // 2, ng + nz // 2
    sl = slice(ng, pr.shape[1] - ng)
    rho, vx, vy, vz, p = (pr[v, sl, j, k].copy() for v in range(5))
    v2 = vx * vx + vy * vy + vz * vz
    vmax2 = v_max * v_max
    m = v2 >= vmax2
    if np.any(m):
        fac = v_max / np.sqrt(v2[m] + 1e-32)
        vx[m] *= fac
        vy[m] *= fac
        vz[m] *= fac
        v2[m] = vmax2 - 1e-14
    return 1.0 / np.sqrt(1.0 - np.clip(v2, 0, 1 - 1e-14)), rho, p, vx


def num_threads():
    return lib().oracle_num_threads()
