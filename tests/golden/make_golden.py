#!/usr/bin/env python3
"""Generate the golden parity fixtures by running the reference itself.

Test infrastructure only.  This script imports the reference's own Numba
hot path (core/srhd_core.py, core/rmhd_core.py, core/boundary.py,
core/nozzle.py, core/source_terms.py) read-only from a checkout of AstroFD
and records its outputs on seeded inputs as ``.npz`` files next to this
script.  The reference freezes its ``configure()`` globals at the first Numba
compile (core/srhd_core.py:18, core/rmhd_core.py:21), so every configuration
runs in a fresh subprocess.

Usage:
    python tests/golden/make_golden.py --ref <path-to-AstroFD> [--jobs 4] [names...]
"""
import argparse
import json
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402
from cases import CASES, CASE_BY_NAME, DT_FRACTION, GR_CASES, GR_BY_NAME, spacing, step_dt  # noqa: E402
import states  # noqa: E402

SPECIAL = ["bc_srhd", "bc_srhd_tracers", "bc_rmhd_pol", "bc_rmhd_tor", "bc_rmhd_chem",
           "c2p_rmhd", "c2p_srhd", "source_terms", "c1_run", "c5_run", "chemistry",
           "dissipation", "diagnostics", "gr_metric"]

NOZZLE_BASE = dict(JET_RADIUS=0.1, SHEAR_THICK=0.02, NOZZLE_PROFILE="top_hat",
                   GAMMA_JET=7.088812050083354, ETA_RHO=0.1, P_EQ=0.01,
                   RHO_AMB=1.0, VX_AMB=0.0, VY_AMB=0.0, VZ_AMB=0.0,
                   NOZZLE_PERTURB="none", TURB_VAMP=0.0, TURB_PAMP=0.0,
                   N_TRACERS=0, TWO_TEMPERATURE=False, PHYSICS="hydro",
                   B_INIT="none", B0=0.0)


def _import_ref(ref):
    sys.path.insert(0, ref)
    from core import srhd_core, rmhd_core, boundary, nozzle, source_terms
    return srhd_core, rmhd_core, boundary, nozzle, source_terms


def run_case(name, ref, out):
    S, R, B, N, ST = _import_ref(ref)
    c = CASE_BY_NAME[name]
    p = c["params"]
    mod = S if c["physics"] == "srhd" else R
    mod.configure(p)
    pr = states.make_state(c["seed"], c["n"], c["ng"], c["physics"],
                           c["n_extra"] + c["pad"], **c["state"])
    nx, ny, nz = pr.shape[1:]
    dx, dy, dz = spacing(c)
    if c["physics"] == "srhd":
        rhs_fn = {"muscl": S.compute_rhs_muscl, "ppm": S.compute_rhs_ppm,
                  "weno": S.compute_rhs_weno}[p["RECON"]]
    else:
        rhs_fn = {"muscl": R.compute_rhs_rmhd, "ppm": R.compute_rhs_ppm,
                  "weno": R.compute_rhs_weno}[p["RECON"]]
    rhs = rhs_fn(pr, nx, ny, nz, dx, dy, dz)
    dt = step_dt(c)
    step = mod.step_ssprk3 if c["rk"] == 3 else mod.step_ssprk2
    out_pr = step(pr.copy(), dx, dy, dz, dt)
    extra = {}
    if c["physics"] == "srhd":
        extra["max_char_speed"] = np.array(S.max_char_speed(pr, nx, ny, nz))
    np.savez_compressed(out, pr_in=pr, rhs=rhs, step_out=out_pr,
                        dt=np.array(dt), params=json.dumps(p), **extra)


def run_gr(name, ref, out):
    """core/grhd_core.py / core/grmhd_core.py: right-hand side and one step."""
    S, R, B, N, ST = _import_ref(ref)
    from core import grhd_core, grmhd_core
    c = GR_BY_NAME[name]
    p = c["params"]
    srhd = c["physics"] == "srhd"
    (S if srhd else R).configure(p)
    G = grhd_core if srhd else grmhd_core
    G.configure(c["gr"])
    pr = states.make_state(c["seed"], c["n"], c["ng"], c["physics"],
                           c["n_extra"] + c["pad"], **c["state"])
    dx = 1.0 / c["n"]
    rhs_fn = G.compute_rhs_grhd if srhd else G.compute_rhs_grmhd
    rhs = rhs_fn(pr, dx, dx, dx, c["offs_x"], c["ng"])
    dt = DT_FRACTION * dx
    step = G.step_ssprk3 if c["rk"] == 3 else G.step_ssprk2
    out_pr = step(pr.copy(), dx, dx, dx, dt, c["offs_x"], c["ng"])
    np.savez_compressed(out, pr_in=pr, rhs=rhs, step_out=out_pr, dt=np.array(dt),
                        params=json.dumps(p), gr=json.dumps(c["gr"]))


def _bc_setup(name):
    """State plus nozzle config for the ghost-fill fixtures."""
    cfg = dict(NOZZLE_BASE)
    if name == "bc_srhd":
        pr = states.make_state(301, 10, 2, "srhd")
        cfg.update(NG=2, NOZZLE_PERTURB="random", TURB_VAMP=0.02, TURB_PAMP=0.01,
                   SHEAR_THICK=0.02)
        seed = 1234
    elif name == "bc_srhd_tracers":
        pr = states.make_state(302, 10, 3, "srhd", n_extra=3)
        cfg.update(NG=3, N_TRACERS=1, TRACER_OFFSET=5, TRACER_NOZZLE_VALUES=[1.0],
                   TRACER_AMB_VALUES=[0.0], TWO_TEMPERATURE=True, THERMO_OFFSET=6,
                   TE_NOZZLE=0.5, TI_NOZZLE=0.25, SHEAR_THICK=0.0,
                   NOZZLE_PROFILE="parabolic", NOZZLE_PERTURB="random",
                   TURB_VAMP=0.05, TURB_PAMP=0.0)
        seed = 77
    elif name == "bc_rmhd_pol":
        pr = states.make_state(303, 10, 3, "rmhd")
        cfg.update(NG=3, PHYSICS="rmhd", B_INIT="poloidal", B0=0.05,
                   NOZZLE_PROFILE="taper")
        seed = 5
    elif name == "bc_rmhd_chem":
        # ion chemistry on: the inflow carries the nozzle's ionisation
        # fractions (nozzle.py:77-82) at CHEM_OFFSET, after Te/Ti
        pr = states.make_state(305, 10, 3, "rmhd", n_extra=5)
        cfg.update(NG=3, PHYSICS="rmhd", B_INIT="toroidal", B0=0.2, TWO_TEMPERATURE=True,
                   THERMO_OFFSET=9, TE_NOZZLE=0.1, TI_NOZZLE=0.08, CHEMISTRY_ENABLED=True,
                   CHEM_OFFSET=11, CHEM_X_HII_NOZZLE=0.9, CHEM_X_HEII_NOZZLE=0.05,
                   CHEM_X_HEIII_NOZZLE=0.01, SHEAR_THICK=0.03, NOZZLE_PERTURB="random",
                   TURB_VAMP=0.01, TURB_PAMP=0.01)
        seed = 11
    else:  # bc_rmhd_tor
        pr = states.make_state(304, 10, 2, "rmhd", n_extra=2)
        cfg.update(NG=2, PHYSICS="rmhd", B_INIT="toroidal", B0=0.3,
                   TWO_TEMPERATURE=True, THERMO_OFFSET=9, TE_NOZZLE=0.02,
                   TI_NOZZLE=0.03, NOZZLE_PERTURB="random", TURB_VAMP=0.01,
                   TURB_PAMP=0.02, SHEAR_THICK=0.05)
        seed = 9
    return pr, cfg, seed


def run_bc(name, ref, out):
    S, R, B, N, ST = _import_ref(ref)
    pr, cfg, seed = _bc_setup(name)
    ng = cfg["NG"]
    nint = pr.shape[2] - 2 * ng
    d = 1.0 / nint
    rng = np.random.default_rng(seed)
    after = pr.copy()
    B.apply_periodic_yz(after, ng)
    periodic = after.copy()
    B.apply_outflow_right_x(after, ng)
    N.apply_nozzle_left_x(after, d, d, d, nint, nint, 0.5, 0.5, rng, cfg)
    np.savez_compressed(out, pr_in=pr, periodic=periodic, filled=after,
                        rng_seed=np.array(seed), cfg=json.dumps(cfg))


def run_c2p(name, ref, out):
    S, R, B, N, ST = _import_ref(ref)
    if name == "c2p_rmhd":
        R.configure(dict(GAMMA=4.0 / 3.0, P_MAX=1e3, V_MAX=0.9999))
        pr = states.make_c2p_batch(401, 3000)
        # also some states with B perpendicular to v (p2c/c2p consistent)
        pr2 = states.make_c2p_batch(402, 1000)
        v = pr2[1:4]
        b = pr2[5:8]
        b -= v * (np.sum(v * b, axis=0) / np.maximum(np.sum(v * v, axis=0), 1e-300))
        pr = np.concatenate([pr, pr2], axis=1)
        m = pr.shape[1]
        U = np.zeros_like(pr)
        out_pr = np.zeros_like(pr)
        for c in range(m):
            U[:, c] = R.prim_to_cons_rmhd(*pr[:, c], 4.0 / 3.0)
        for c in range(m):
            out_pr[:, c] = R.cons_to_prim_rmhd(*U[:, c])
        np.savez_compressed(out, pr_in=pr, cons=U, pr_out=out_pr,
                            params=json.dumps(dict(GAMMA=4.0 / 3.0, P_MAX=1e3,
                                                   V_MAX=0.9999)))
    else:
        S.configure(dict(GAMMA=5.0 / 3.0, P_MAX=2.0, V_MAX=0.9999))
        rng = np.random.default_rng(403)
        m = 3000
        pr = np.zeros((5, m))
        pr[0] = 10.0 ** rng.uniform(-4, 1, m)
        W = 10.0 ** rng.uniform(0, np.log10(20.0), m)
        v = np.sqrt(1 - 1 / W ** 2)
        d = rng.normal(size=(3, m))
        d /= np.linalg.norm(d, axis=0)
        pr[1:4] = v * d
        pr[4] = 10.0 ** rng.uniform(-6, np.log10(2.0), m)
        U = np.zeros_like(pr)
        out_pr = np.zeros_like(pr)
        for c in range(m):
            U[:, c] = S.prim_to_cons(*pr[:, c])
        for c in range(m):
            out_pr[:, c] = S.cons_to_prim(*U[:, c])
        np.savez_compressed(out, pr_in=pr, cons=U, pr_out=out_pr,
                            params=json.dumps(dict(GAMMA=5.0 / 3.0, P_MAX=2.0,
                                                   V_MAX=0.9999)))


def run_source(name, ref, out):
    S, R, B, N, ST = _import_ref(ref)
    pr = states.make_state(501, 8, 3, "rmhd", n_extra=2)
    pr[9] = np.abs(pr[9]) * 0.02
    pr[10] = np.abs(pr[10]) * 0.03
    cfg = dict(COOLING_ENABLED=True, COOLING_LAMBDA=0.01, HEATING_RATE=1e-4,
               NG=3, P_MAX=2.0, TWO_TEMPERATURE=True, TEI_TAU=0.1,
               THERMO_OFFSET=9, N_TRACERS=0)
    dt = 0.01
    a = pr.copy()
    ST.apply_cooling_heating(a, dt, cfg)
    b = a.copy()
    ST.apply_two_temperature(b, dt, cfg)
    np.savez_compressed(out, pr_in=pr, cooled=a, two_temp=b, dt=np.array(dt),
                        cfg=json.dumps(cfg))


def _run_loop(ref, physics, n, ng, params, cfg, steps, seed, sources=None):
    """Reference driver loop (solvers/srhd3d_mpi_muscl.py:276-326) on one rank."""
    S, R, B, N, ST = _import_ref(ref)
    mod = S if physics == "srhd" else R
    mod.configure(params)
    rng = np.random.default_rng(seed)
    Nn = n + 2 * ng
    nm = 5 if physics == "srhd" else 9
    nv = nm + params.get("N_PASSIVE", 0)
    pr = np.zeros((nv, Nn, Nn, Nn))
    pr[0] = 1.0 * (1.0 + 0.01 * (2.0 * rng.random((Nn, Nn, Nn)) - 1.0))
    pr[4] = 0.01
    if physics == "rmhd":
        pr[5] = cfg.get("BX_AMB", 0.0)
        pr[1:4] += 0.01 * (2.0 * rng.random((3, Nn, Nn, Nn)) - 1.0)
    if params.get("N_PASSIVE", 0) == 2:
        pr[nm] = 0.01
        pr[nm + 1] = 0.01
    pr0 = pr.copy()
    d = 1.0 / n
    brng = np.random.default_rng(1234)
    B.apply_periodic_yz(pr, ng)
    B.apply_outflow_right_x(pr, ng)
    N.apply_nozzle_left_x(pr, d, d, d, n, n, 0.5, 0.5, brng, cfg)
    dts = []
    for _ in range(steps):
        if physics == "srhd":
            amax = S.max_char_speed(pr, Nn, Nn, Nn)
        else:
            amax = 1.0
        dt = params["CFL"] * d / max(amax, 1e-12)
        dts.append(dt)
        B.apply_periodic_yz(pr, ng)
        B.apply_outflow_right_x(pr, ng)
        N.apply_nozzle_left_x(pr, d, d, d, n, n, 0.5, 0.5, brng, cfg)
        step = mod.step_ssprk3 if params["RK_ORDER"] == 3 else mod.step_ssprk2
        pr = step(pr, d, d, d, dt)
        B.apply_periodic_yz(pr, ng)
        B.apply_outflow_right_x(pr, ng)
        N.apply_nozzle_left_x(pr, d, d, d, n, n, 0.5, 0.5, brng, cfg)
        if sources is not None:
            pr = ST.apply_cooling_heating(pr, dt, sources)
            pr = ST.apply_two_temperature(pr, dt, sources)
    return pr0, pr, np.array(dts)


def run_loop(name, ref, out):
    if name == "c1_run":
        params = dict(GAMMA=5.0 / 3.0, P_MAX=2.0, V_MAX=0.9999, RECON="muscl",
                      LIMITER="minmod", RIEMANN="hlle", RK_ORDER=2, CFL=0.4,
                      N_PASSIVE=0, PASSIVE_OFFSET=5)
        cfg = dict(NOZZLE_BASE, NG=2, SHEAR_THICK=0.0)
        pr0, pr, dts = _run_loop(ref, "srhd", 16, 2, params, cfg, 10, 601)
        np.savez_compressed(out, pr_init=pr0, pr_final=pr, dts=dts,
                            params=json.dumps(params), cfg=json.dumps(cfg),
                            steps=np.array(10), n=np.array(16), ng=np.array(2))
    else:  # c5_run: magnetised WENO/HLLD jet with thermo passives + sources
        params = dict(GAMMA=4.0 / 3.0, P_MAX=2.0, V_MAX=0.9999, RECON="weno",
                      LIMITER="mc", RIEMANN="hlld_full", RK_ORDER=3, CFL=0.35,
                      GLM_CH=1.0, GLM_CP=0.1, N_PASSIVE=2, PASSIVE_OFFSET=9,
                      RESISTIVE_ENABLED=True, RESISTIVITY=1e-4)
        cfg = dict(NOZZLE_BASE, NG=3, PHYSICS="rmhd", B_INIT="toroidal", B0=0.2,
                   GAMMA_JET=10.0, TWO_TEMPERATURE=True, THERMO_OFFSET=9,
                   TE_NOZZLE=0.1, TI_NOZZLE=0.1, BX_AMB=0.1)
        sources = dict(COOLING_ENABLED=True, COOLING_LAMBDA=0.01, HEATING_RATE=0.0,
                       NG=3, P_MAX=2.0, TWO_TEMPERATURE=True, TEI_TAU=0.1,
                       THERMO_OFFSET=9, N_TRACERS=0)
        pr0, pr, dts = _run_loop(ref, "rmhd", 10, 3, params, cfg, 3, 602, sources)
        np.savez_compressed(out, pr_init=pr0, pr_final=pr, dts=dts,
                            params=json.dumps(params), cfg=json.dumps(cfg),
                            sources=json.dumps(sources), steps=np.array(3),
                            n=np.array(10), ng=np.array(3))


def run_chem_dissip(name, ref, out):
    """core/chemistry.py apply_ion_chemistry and core/dissipation.py
    apply_causal_dissipation (plain Python in the reference) on seeded blocks."""
    sys.path.insert(0, ref)
    rng = np.random.default_rng(701 if name == "chemistry" else 702)
    n, ng = 12, 2
    N = n + 2 * ng
    dt, d = 0.01, 1.0 / n
    if name == "chemistry":
        from core import chemistry as CH
        pr = np.zeros((8, N, N, N))
        pr[0] = 10.0 ** rng.uniform(-1, 1, (N, N, N))
        pr[4] = pr[0] * 10.0 ** rng.uniform(-3, 2, (N, N, N))  # T = 10 K .. 1e6 K
        pr[1:4] = 0.1 * rng.standard_normal((3, N, N, N))
        pr[5:8] = rng.uniform(-0.1, 1.1, (3, N, N, N))          # clamps exercised
        pr[0, 3, 3, 3] = -1.0                                    # skipped cell
        outs = {}
        for tag, scale in (("nominal", 1.0), ("fast", 1e9)):
            cfg = dict(CHEMISTRY_ENABLED=True, N_CHEM=3, CHEM_OFFSET=5, NG=ng,
                       CHEM_RATE_SCALE=scale, CHEM_ENERGY_SCALE=1e-6, GAMMA=5.0 / 3.0)
            outs[tag] = CH.apply_ion_chemistry(pr.copy(), dt, cfg)
            outs["cfg_" + tag] = np.array(json.dumps(cfg))
        np.savez_compressed(out, pr_in=pr, dt=np.array(dt), **outs)
    else:
        from core import dissipation as DI
        pr = np.zeros((15, N, N, N))
        pr[0] = 1.0 + 0.5 * rng.random((N, N, N))
        pr[4] = 0.1 + 0.5 * rng.random((N, N, N))
        pr[1:4] = 0.3 * rng.standard_normal((3, N, N, N))
        pr[5:15] = 0.2 * rng.standard_normal((10, N, N, N))
        outs = {}
        cases = {"full": dict(BULK_ZETA=0.1, SHEAR_ETA=0.05, HEAT_KAPPA=0.02, RELAX_TAU=0.1,
                              RELAX_TAU_SHEAR=0.2, DISSIPATION_CAP_FRAC=0.5, P_MAX=0.5,
                              DISSIPATION_ADVECT=True),
                 "noadvect": dict(BULK_ZETA=0.0, SHEAR_ETA=0.3, HEAT_KAPPA=0.0, RELAX_TAU=0.05,
                                  DISSIPATION_CAP_FRAC=0.5, P_MAX=1.0, DISSIPATION_ADVECT=False)}
        for tag, extra in cases.items():
            cfg = dict(DISSIPATION_ENABLED=True, PHYSICS="hydro", NG=ng, **extra)
            outs[tag] = DI.apply_causal_dissipation(pr.copy(), dt, d, d, d, cfg)
            outs["cfg_" + tag] = np.array(json.dumps(cfg))
        np.savez_compressed(out, pr_in=pr, dt=np.array(dt), dx=np.array(d), **outs)


class _OneRank:
    """The mpi4py surface utils/diagnostics.py uses, for one rank (mpi4py
    is not installed where the fixtures are made)."""
    MAX, SUM = "max", "sum"

    def allreduce(self, v, op=None):
        return v

    def gather(self, v, root=0):
        return [v]

    def Gatherv(self, sendbuf, recvbuf, root=0):
        recvbuf[0][:] = sendbuf


def diagnostics_blocks():
    """Seeded SRHD (5-variable) and RMHD (9-variable) blocks with cells at
    v >= 1 (Gamma capping), above V_MAX on the centreline and at the inlet
    (velocity cap of prim_to_cons_rmhd) and p above P_MAX."""
    rng = np.random.default_rng(703)
    n, ng = 10, 2
    N = n + 2 * ng
    out = {}
    for name, nv in (("srhd", 5), ("rmhd", 9)):
        pr = np.zeros((nv, N, N, N))
        pr[0] = 0.5 + rng.random((N, N, N))
        pr[4] = 10.0 ** rng.uniform(-3, 0.5, (N, N, N))
        v = rng.standard_normal((3, N, N, N))
        v *= rng.uniform(0.0, 0.995, (N, N, N)) / np.linalg.norm(v, axis=0)
        pr[1:4] = v
        pr[1:4, 4, 5, 6] *= 1.2 / np.linalg.norm(pr[1:4, 4, 5, 6])   # v > 1
        pr[1:4, 5, 7, 7] *= 0.9995 / np.linalg.norm(pr[1:4, 5, 7, 7])  # centreline, > V_MAX
        pr[1:4, ng, 3, 4] *= 0.9992 / np.linalg.norm(pr[1:4, ng, 3, 4])  # inlet, > V_MAX
        if nv == 9:
            pr[5:8] = 0.3 * rng.standard_normal((3, N, N, N))
            pr[8] = 0.01 * rng.standard_normal((N, N, N))
        out[name] = pr
    return out, ng


def run_diagnostics(name, ref, out):
    """utils/diagnostics.py on one rank, with a stub communicator; the RMHD
    block under GAMMA 4/3 (the diagnostics' prim_to_cons keeps 5/3)."""
    import tempfile
    import types
    stub = types.ModuleType("mpi4py")
    stub.MPI = _OneRank
    sys.modules["mpi4py"] = stub
    sys.path.insert(0, ref)
    from core import srhd_core, rmhd_core
    from utils import diagnostics as DG
    cfg = dict(GAMMA=4.0 / 3.0, V_MAX=0.999, P_MAX=1.0)
    rmhd_core.configure(cfg)
    blocks, ng = diagnostics_blocks()
    d = 0.1
    rec = {}
    for phys, pr in blocks.items():
        with tempfile.TemporaryDirectory() as run:
            comm = _OneRank()
            rmhd = phys == "rmhd"
            res = DG.compute_diagnostics_and_write(
                pr, d, 0.7 * d, 1.3 * d, 0, None, comm, 0, 7, 0.25, 1e-3, 0.9, run,
                rmhd_core.prim_to_cons_rmhd if rmhd else srhd_core.prim_to_cons, ng, rmhd)
            DG.compute_centerline_and_write(pr, d, 0.7 * d, 1.3 * d, 0, None, comm, 0, 7, 0.25,
                                            run, cfg["V_MAX"], ng)
            dv = DG.compute_divb_and_write(pr, d, 0.7 * d, 1.3 * d, 0, None, comm, 0, 7, 0.25,
                                           run, ng)
            rec[phys + "_diag"] = np.array(res, dtype=np.float64)
            rec[phys + "_divb"] = np.array([np.nan if x is None else x for x in dv])
            for f in ("diagnostics.csv", "centerline.csv", "divb.csv"):
                path = os.path.join(run, f)
                text = open(path).read() if os.path.exists(path) else ""
                rec[phys + "_" + f.split(".")[0] + "_csv"] = np.array(text)
        rec[phys + "_pr"] = pr
    np.savez_compressed(out, ng=np.array(ng), d=np.array(d), cfg=np.array(json.dumps(cfg)), **rec)


def run_driver_case(name, ref, out):
    """The reference's driver script, unchanged, on its own core modules (one
    rank, through tests/driver_harness.py's mpi4py and json5 stand-ins)."""
    import tempfile
    sys.path.insert(0, os.path.dirname(HERE))
    import driver_harness as DH
    with tempfile.TemporaryDirectory() as tmp:
        res = DH.run_driver(ref, name[len("driver_"):], tmp, dropin=False)
    np.savez_compressed(out, t_end=np.array(DH.T_END), **res)


def one(name, ref):
    out = os.path.join(HERE, name + ".npz")
    if name.startswith("driver_"):
        run_driver_case(name, ref, out)
    elif name in CASE_BY_NAME:
        run_case(name, ref, out)
    elif name.startswith("bc_"):
        run_bc(name, ref, out)
    elif name.startswith("c2p_"):
        run_c2p(name, ref, out)
    elif name == "source_terms":
        run_source(name, ref, out)
    elif name in ("chemistry", "dissipation"):
        run_chem_dissip(name, ref, out)
    elif name == "diagnostics":
        run_diagnostics(name, ref, out)
    elif name in GR_BY_NAME:
        run_gr(name, ref, out)
    elif name == "gr_metric":
        sys.path.insert(0, ref)
        from core import gr_metric as GM
        pts = np.random.default_rng(707).uniform(-2.0, 2.0, (64, 3))
        pts[0] = 0.0  # the 1e-12 offset of r
        pts[1] = (0.025, 0.0, 0.0)  # r = M/2 for M = 0.05: 1 - a^2 = 0 branch
        iso = [GM.schwarzschild_iso_lapse_and_grad(*p, 0.05) for p in pts]
        ks = [GM.schwarzschild_ks_lapse_shift_and_grad(*p, 0.05) for p in pts]
        kerr = [GM.kerr_schild_lapse_shift_and_grad(*p, 0.05, 0.7) for p in pts]
        np.savez_compressed(out, pts=pts, iso=np.array(iso), ks=np.array(ks),
                            kerr=np.array(kerr))
    else:
        run_loop(name, ref, out)
    print("wrote", out, flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True)
    ap.add_argument("--jobs", type=int, default=4)
    ap.add_argument("--one", default=None)
    ap.add_argument("names", nargs="*")
    a = ap.parse_args()
    if a.one:
        one(a.one, a.ref)
        return
    sys.path.insert(0, os.path.dirname(HERE))
    import driver_harness as DH
    names = a.names or ([c["name"] for c in CASES] + SPECIAL + [c["name"] for c in GR_CASES] +
                        ["driver_" + c for c in DH.CONFIGS])
    env = dict(os.environ, PYTHONDONTWRITEBYTECODE="1", NUMBA_NUM_THREADS="1")

    def launch(nm):
        r = subprocess.run([sys.executable, __file__, "--ref", a.ref, "--one", nm],
                           env=env, capture_output=True, text=True)
        if r.returncode != 0:
            return f"FAIL {nm}\n{r.stdout}\n{r.stderr}"
        return r.stdout.strip()

    with ThreadPoolExecutor(a.jobs) as ex:
        for msg in ex.map(launch, names):
            print(msg, flush=True)


if __name__ == "__main__":
    main()
