"""Drop-in replacement of AstroFD's core/source_terms.py (operator-split
post-step sources): ``apply_cooling_heating`` (core/source_terms.py:5) and
``apply_two_temperature`` (core/source_terms.py:30), in place on the device.
"""
import numpy as np
import torch

from .. import _lib, runtime as rt


def _run(pr, fn):
    if isinstance(pr, torch.Tensor):
        fn(pr)
        return pr
    t, _ = rt.to_device(pr)
    fn(t)
    np.copyto(pr, t.cpu().numpy())
    return pr


def apply_cooling_heating(pr, dt, cfg):
    if not cfg.get("COOLING_ENABLED", False):
        return pr
    cool = float(cfg.get("COOLING_LAMBDA", 0.0))
    heat = float(cfg.get("HEATING_RATE", 0.0))
    if cool == 0.0 and heat == 0.0:
        return pr
    L = _lib.load()
    ng = int(cfg.get("NG", 2))
    pmax = float(cfg.get("P_MAX", 1.0))

    def f(t):
        _lib.check(L.astro_cooling_heating(rt.ptr(t), rt.grid_of(t), ng, float(dt), cool, heat,
                                           pmax, rt.stream_handle(t.device)),
                   "astro_cooling_heating")
    return _run(pr, f)


def apply_two_temperature(pr, dt, cfg):
    if not cfg.get("TWO_TEMPERATURE", False):
        return pr
    off = int(cfg.get("THERMO_OFFSET", 0))
    if pr.shape[0] < off + 2:
        return pr
    tau = float(cfg.get("TEI_TAU", 0.5))
    if tau <= 0.0:
        return pr
    L = _lib.load()
    ng = int(cfg.get("NG", 2))

    def f(t):
        _lib.check(L.astro_two_temperature(rt.ptr(t), rt.grid_of(t), ng, float(dt), tau, off,
                                           rt.stream_handle(t.device)),
                   "astro_two_temperature")
    return _run(pr, f)
