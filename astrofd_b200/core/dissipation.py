"""Drop-in replacement of AstroFD's core/dissipation.py.

``apply_causal_dissipation(pr, dt, dx, dy, dz, cfg)`` (core/dissipation.py:5):
Israel-Stewart bulk/shear/heat-flux fields (variables 5..14 of a 15-variable
SRHD block) advected first-order upwind by the velocity, then relaxed toward
their Navier-Stokes targets with the given relaxation times and capped, on the
interior cells.  Same configuration keys and gating as the reference (hydro
physics only, 15+ variables, a non-zero coefficient and positive relaxation
times); updates ``pr`` in place and returns it.  The dissipation fluxes that
the reference's RHS adds for 15+-variable blocks are not part of this library.
"""
import numpy as np
import torch

from .. import _lib, runtime as rt


def relaxation_times(cfg):
    """Per-channel RELAX_TAU_BULK / _SHEAR / _HEAT, falling back to RELAX_TAU
    (also when the per-channel value is 0), as core/dissipation.py:18-20."""
    base = cfg.get("RELAX_TAU", 0.1)
    return tuple(float(cfg.get(k, base) or base)
                 for k in ("RELAX_TAU_BULK", "RELAX_TAU_SHEAR", "RELAX_TAU_HEAT"))


def apply_causal_dissipation(pr, dt, dx, dy, dz, cfg):
    if not cfg.get("DISSIPATION_ENABLED", False):
        return pr
    if cfg.get("PHYSICS") not in ("hydro", "grhd"):
        return pr
    zeta, eta, kappa = (float(cfg.get(k, 0.0)) for k in ("BULK_ZETA", "SHEAR_ETA", "HEAT_KAPPA"))
    tb, ts, th = relaxation_times(cfg)
    if (zeta == 0.0 and eta == 0.0 and kappa == 0.0) or min(tb, ts, th) <= 0.0:
        return pr
    if pr.shape[0] < 15:
        return pr
    L = _lib.load()
    c = _lib.AstroDissipation()
    c.ng = int(cfg.get("NG", 2))
    c.advect = 1 if bool(cfg.get("DISSIPATION_ADVECT", True)) else 0
    c.zeta, c.eta, c.kappa = zeta, eta, kappa
    c.tau_bulk, c.tau_shear, c.tau_heat = tb, ts, th
    c.cap_frac = float(cfg.get("DISSIPATION_CAP_FRAC", 0.5))
    c.p_max = float(cfg.get("P_MAX", 1.0))

    def f(t):
        g = rt.grid_of(t, dx, dy, dz)
        nb = L.astro_causal_dissipation_workspace_bytes(g)
        w = rt.workspace(nb, t.device)
        _lib.check(L.astro_causal_dissipation(rt.ptr(t), g, c, float(dt), rt.ptr(w), nb,
                                              rt.stream_handle(t.device)),
                   "astro_causal_dissipation")

    if isinstance(pr, torch.Tensor):
        f(pr)
    else:
        t, _ = rt.to_device(pr)
        f(t)
        np.copyto(pr, t.cpu().numpy())
    return pr
