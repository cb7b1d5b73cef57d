"""Drop-in replacement of AstroFD's core/boundary.py (in-place ghost fills).

``apply_periodic_yz`` (core/boundary.py:4) and ``apply_outflow_right_x``
(core/boundary.py:10).  numpy blocks are filled through the device and copied
back in place; CUDA tensors are filled in place on the current stream.

``apply_outflow_yz`` has no counterpart in the reference: zero-gradient y and
z faces, for jet set-ups with outflow on every face but the nozzle (the
reference's driver fills y and z periodically).
"""
import numpy as np
import torch

from .. import _lib, runtime as rt


def _inplace(pr, fn):
    if isinstance(pr, torch.Tensor):
        if not pr.is_contiguous():
            raise _lib.AstroError("primitive tensor must be contiguous")
        fn(pr)
        return
    t, _ = rt.to_device(pr)
    fn(t)
    np.copyto(pr, t.cpu().numpy())


def apply_periodic_yz(pr, ng):
    L = _lib.load()

    def f(t):
        g = rt.grid_of(t)
        _lib.check(L.astro_periodic_yz(rt.ptr(t), g, int(ng), rt.stream_handle(t.device)),
                   "astro_periodic_yz")
    _inplace(pr, f)


def apply_outflow_right_x(pr, ng):
    L = _lib.load()

    def f(t):
        g = rt.grid_of(t)
        _lib.check(L.astro_outflow_right_x(rt.ptr(t), g, int(ng), rt.stream_handle(t.device)),
                   "astro_outflow_right_x")
    _inplace(pr, f)


def apply_outflow_yz(pr, ng):
    L = _lib.load()

    def f(t):
        g = rt.grid_of(t)
        _lib.check(L.astro_outflow_yz(rt.ptr(t), g, int(ng), rt.stream_handle(t.device)),
                   "astro_outflow_yz")
    _inplace(pr, f)
