"""Drop-in replacement of AstroFD's core/nozzle.py (left-x jet inflow).

``nozzle_weight`` (core/nozzle.py:5) is the reference's host-side profile
function; ``apply_nozzle_left_x`` (core/nozzle.py:27) fills the left x ghost
layers on the device.  For perturbed nozzles the random numbers are drawn on
the host from the caller's ``numpy.random.Generator`` in the reference's order
(3 per cell with weight > 0, loop order g, j, k) and uploaded, so the stream
advances exactly as the reference's does.
"""
import math

import numpy as np
import torch

from .. import _lib, runtime as rt

_PROFILE = {"taper": 1, "smooth": 1, "parabolic": 2, "parabola": 2}
_rank_cache = {}


def nozzle_weight(r, radius, shear_thick, profile):
    if radius <= 0.0:
        return 0.0
    if profile in ("taper", "smooth"):
        if r >= radius:
            return 0.0
        return 0.5 * (1.0 + math.cos(math.pi * r / radius))
    if profile in ("parabolic", "parabola"):
        if r >= radius:
            return 0.0
        x = r / radius
        return max(0.0, 1.0 - x * x)
    if shear_thick > 0.0:
        return 0.5 * (1.0 - math.tanh((r - radius) / shear_thick))
    return 1.0 if r <= radius else 0.0


def _rank_map(ng, ny_loc, nz_loc, dy, dz, y0, z0, radius, shear, profile):
    key = (ng, ny_loc, nz_loc, dy, dz, y0, z0, radius, shear, profile)
    hit = _rank_cache.get(key)
    if hit is not None:
        return hit
    rank = np.full((ny_loc, nz_loc), -1, dtype=np.int32)
    n = 0
    for jj in range(ny_loc):
        y = (jj + 0.5) * dy
        for kk in range(nz_loc):
            z = (kk + 0.5) * dz
            rr = math.sqrt((y - y0) ** 2 + (z - z0) ** 2)
            if nozzle_weight(rr, radius, shear, profile) > 0.0:
                rank[jj, kk] = n
                n += 1
    _rank_cache[key] = (rank, n)
    return rank, n


def nozzle_struct(cfg, dy, dz, y0, z0):
    c = _lib.AstroNozzle()
    c.ng = int(cfg["NG"])
    prof = cfg.get("NOZZLE_PROFILE", "top_hat")
    c.profile = _PROFILE.get(prof, 0)
    c.perturb = 0 if cfg.get("NOZZLE_PERTURB", "none") == "none" else 1
    c.physics = 1 if cfg.get("PHYSICS") in ("rmhd", "grmhd") else 0
    b = cfg.get("B_INIT")
    c.b_init = {"poloidal": 1, "toroidal": 2, "toroidal_phi": 3}.get(b, 0)
    c.ambient_bc = 1 if cfg.get("NOZZLE_AMBIENT", "fixed") == "outflow" else 0
    c.b_amb_x = float(cfg.get("B_AMB_X", 0.0))
    c.n_tracers = int(cfg.get("N_TRACERS", 0))
    if c.n_tracers > 8:
        raise _lib.AstroError("at most 8 tracers are supported")
    c.tracer_offset = int(cfg.get("TRACER_OFFSET", 5))
    c.two_temperature = 1 if cfg.get("TWO_TEMPERATURE", False) else 0
    c.thermo_offset = int(cfg.get("THERMO_OFFSET", 0))
    c.radius = float(cfg["JET_RADIUS"])
    c.shear_thick = float(cfg["SHEAR_THICK"])
    c.gamma_jet = float(cfg["GAMMA_JET"])
    c.eta_rho = float(cfg["ETA_RHO"])
    c.p_eq = float(cfg["P_EQ"])
    c.rho_amb = float(cfg["RHO_AMB"])
    c.vx_amb, c.vy_amb, c.vz_amb = (float(cfg[k]) for k in ("VX_AMB", "VY_AMB", "VZ_AMB"))
    c.turb_vamp = float(cfg.get("TURB_VAMP", 0.0))
    c.turb_pamp = float(cfg.get("TURB_PAMP", 0.0))
    c.b0 = float(cfg.get("B0", 0.0))
    c.te = float(cfg.get("TE_NOZZLE", cfg.get("TE_AMB", 0.0)) or 0.0)
    c.ti = float(cfg.get("TI_NOZZLE", cfg.get("TI_AMB", 0.0)) or 0.0)
    c.dy, c.dz, c.y0, c.z0 = float(dy), float(dz), float(y0), float(z0)
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
    for t in range(c.n_tracers):
        c.tracer_nozzle[t] = nv[t] if t < len(nv) else (1.0 if t == 0 else 0.0)
        c.tracer_amb[t] = av[t] if t < len(av) else 0.0
    return c


def apply_nozzle_left_x(pr, dx, dy, dz, ny_loc, nz_loc, y0, z0, rng, cfg):
    L = _lib.load()
    c = nozzle_struct(cfg, dy, dz, y0, z0)
    draws_t = rank_t = None
    nw = 0
    if c.perturb:
        rank, nw = _rank_map(c.ng, int(ny_loc), int(nz_loc), float(dy), float(dz), float(y0),
                             float(z0), c.radius, c.shear_thick,
                             cfg.get("NOZZLE_PROFILE", "top_hat"))
        draws = rng.random(3 * c.ng * nw) if nw > 0 else np.zeros(1)

    def f(t):
        nonlocal draws_t, rank_t
        if c.perturb:
            draws_t = torch.from_numpy(np.ascontiguousarray(draws)).to(t.device)
            rank_t = torch.from_numpy(np.ascontiguousarray(rank)).to(t.device)
        g = rt.grid_of(t)
        if g.ny - 2 * c.ng != int(ny_loc) or g.nz - 2 * c.ng != int(nz_loc):
            raise _lib.AstroError("ny_loc/nz_loc must match the block's interior extents")
        _lib.check(L.astro_nozzle_left_x(
            rt.ptr(t), g, c, rt.ptr(draws_t) if draws_t is not None else None,
            rt.ptr(rank_t) if rank_t is not None else None, int(nw),
            rt.stream_handle(t.device)), "astro_nozzle_left_x")

    if isinstance(pr, torch.Tensor):
        f(pr)
    else:
        t, _ = rt.to_device(pr)
        f(t)
        np.copyto(pr, t.cpu().numpy())
