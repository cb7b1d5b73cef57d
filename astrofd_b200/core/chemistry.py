"""Drop-in replacement of AstroFD's core/chemistry.py.

``apply_ion_chemistry(pr, dt, cfg)`` (core/chemistry.py:43): H/He
non-equilibrium ionisation of the interior cells with the reference's rate
fits, an implicit-recombination / explicit-ionisation step and the ionisation
energy taken from the pressure, on the device.  Same configuration keys and
gating as the reference; updates ``pr`` in place and returns it (numpy blocks
go through the device and are copied back).
"""
import numpy as np
import torch

from .. import _lib, runtime as rt


def apply_ion_chemistry(pr, dt, cfg):
    if not cfg.get("CHEMISTRY_ENABLED", False):
        return pr
    if int(cfg.get("N_CHEM", 0)) < 3:
        return pr
    off = int(cfg.get("CHEM_OFFSET", 0))
    if pr.shape[0] <= off + 2:
        return pr
    L = _lib.load()
    c = _lib.AstroChemistry()
    c.ng, c.chem_offset = int(cfg.get("NG", 2)), off
    c.x, c.y = float(cfg.get("CHEM_X", 0.76)), float(cfg.get("CHEM_Y", 0.24))
    c.tunit_k = float(cfg.get("CHEM_TUNIT_K", 1.0e4))
    c.rate_scale = float(cfg.get("CHEM_RATE_SCALE", 1.0))
    c.energy_scale = float(cfg.get("CHEM_ENERGY_SCALE", 1.0))
    c.tmin_k = float(cfg.get("CHEM_TMIN_K", 1.0))
    c.gamma = float(cfg.get("GAMMA", 5.0 / 3.0))

    def f(t):
        g = rt.grid_of(t)
        _lib.check(L.astro_ion_chemistry(rt.ptr(t), g, c, float(dt), rt.stream_handle(t.device)),
                   "astro_ion_chemistry")

    if isinstance(pr, torch.Tensor):
        f(pr)
    else:
        t, _ = rt.to_device(pr)
        f(t)
        np.copyto(pr, t.cpu().numpy())
    return pr
