"""Drop-in replacement of AstroFD's core/srhd_core.py on the B200.

Same names, arguments and return conventions as the reference module
(core/srhd_core.py): ``configure`` :18, ``prim_to_cons`` :47, ``cons_to_prim``
:62, ``compute_rhs_muscl`` :469, ``compute_rhs_ppm`` :927,
``compute_rhs_weno`` :1167, ``max_char_speed`` :1268, ``step_ssprk2`` :1286,
``step_ssprk3`` :1334.  Arrays may be numpy float64 blocks (uploaded, computed
on the GPU, returned as numpy) or float64 CUDA tensors (stay on the device).

Extra configure keys (not in the reference): ``FLUX_MODE`` ("reference" |
"conservative"), ``PRECISION`` ("fp64" | "mixed"), ``SRHD_HONOUR_GAMMA``.
"""
import numpy as np

from .. import _lib
from ._engine import Engine

GAMMA = 5.0 / 3.0
P_MAX = 1.0
V_MAX = 0.999
LIMITER_ID = 0
RECON_ID = 0
RIEMANN_ID = 0
SMALL = 1e-12
N_PASSIVE = 0
PASSIVE_OFFSET = 5

_E = Engine(_lib.SRHD)


def configure(params):
    """Set the parameters used by every following call (re-callable)."""
    global GAMMA, P_MAX, V_MAX, LIMITER_ID, RECON_ID, RIEMANN_ID, N_PASSIVE, PASSIVE_OFFSET
    _E.configure(params)
    p = _E.p
    GAMMA, P_MAX, V_MAX = p.gamma, p.p_max, p.v_max
    LIMITER_ID, RECON_ID, RIEMANN_ID = p.limiter, p.recon, p.riemann
    N_PASSIVE, PASSIVE_OFFSET = p.n_passive, p.passive_offset


def compute_rhs_muscl(pr, nx, ny, nz, dx, dy, dz):
    return _rhs_with(0, pr, nx, ny, nz, dx, dy, dz)


def compute_rhs_ppm(pr, nx, ny, nz, dx, dy, dz):
    return _rhs_with(1, pr, nx, ny, nz, dx, dy, dz)


def compute_rhs_weno(pr, nx, ny, nz, dx, dy, dz):
    return _rhs_with(2, pr, nx, ny, nz, dx, dy, dz)


def _rhs_with(recon, pr, nx, ny, nz, dx, dy, dz):
    saved = _E.p.recon
    _E.p.recon = recon
    try:
        return _E.rhs(pr, nx, ny, nz, dx, dy, dz)
    finally:
        _E.p.recon = saved


def max_char_speed(pr, nx, ny, nz):
    """Host float, like the reference (one device->host read)."""
    return float(_E.max_char_speed(pr, nx, ny, nz).item())


def max_char_speed_device(pr):
    """The same reduction left on the device (1-element float64 tensor)."""
    return _E.max_char_speed(pr, *pr.shape[1:])


def step_ssprk2(pr, dx, dy, dz, dt, out=None):
    return _E.step(pr, dx, dy, dz, dt, 2, out)


def step_ssprk3(pr, dx, dy, dz, dt, out=None):
    return _E.step(pr, dx, dy, dz, dt, 3, out)


def step_stage(pr, pr_stage, out, dx, dy, dz, dt, rk_order, stage):
    """No reference counterpart: stage `stage` of step_ssprk2/3 from the step
    input pr, this stage's input pr_stage (pr itself at stage 0) into out, for
    callers that refresh ghost layers between stages (astrofd_b200.slabs).
    CUDA tensors; the stages of one step run in order, nothing else stepping
    on the device in between."""
    return _E.step_stage(pr, pr_stage, out, dx, dy, dz, dt, rk_order, stage)


def prim_to_cons(rho, vx, vy, vz, p, gamma=None):
    """Scalars (as the reference) or equal-shaped arrays/tensors.  Without
    ``gamma`` the reference's default applies: 5/3, bound when the module was
    imported (core/srhd_core.py:47), whatever GAMMA is configured; an explicit
    ``gamma`` is used for this call, as the reference honours it."""
    return _pointwise(_E.p2c_array, (rho, vx, vy, vz, p), gamma)


def cons_to_prim(D, Sx, Sy, Sz, tau, gamma=None):
    """Inverse of prim_to_cons, with the same ``gamma`` rule
    (core/srhd_core.py:62)."""
    return _pointwise(_E.c2p_array, (D, Sx, Sy, Sz, tau), gamma)


def _pointwise(fn, comps, gamma=None):
    if gamma is None:
        return _pointwise_call(fn, comps)
    saved = _E.p.srhd_gamma
    _E.p.srhd_gamma = float(gamma)
    try:
        return _pointwise_call(fn, comps)
    finally:
        _E.p.srhd_gamma = saved


def _pointwise_call(fn, comps):
    import torch
    if isinstance(comps[0], torch.Tensor):
        shape = comps[0].shape
        out = fn(torch.stack([c.reshape(-1) for c in comps]))
        return tuple(out[v].reshape(shape) for v in range(out.shape[0]))
    if np.ndim(comps[0]) == 0:
        return _E.scalar_convert(fn, [[float(c)] for c in comps])
    shape = np.shape(comps[0])
    out = fn(np.stack([np.asarray(c, dtype=np.float64).reshape(-1) for c in comps]))
    return tuple(out[v].reshape(shape) for v in range(out.shape[0]))


def c2p_stats(reset=False):
    return _E.c2p_stats(reset)


def engine():
    return _E
