"""Drop-in replacement of AstroFD's core/rmhd_core.py on the B200.

Same names, arguments and return conventions as the reference module
(core/rmhd_core.py): ``configure`` :21, ``prim_to_cons_rmhd`` :138,
``cons_to_prim_rmhd`` :249, ``compute_rhs_rmhd`` (MUSCL) :749,
``compute_rhs_ppm`` :1280, ``compute_rhs_weno`` :1440, ``step_ssprk2`` :1559,
``step_ssprk3`` :1609.  Arrays may be numpy float64 blocks (uploaded, computed
on the GPU, returned as numpy) or float64 CUDA tensors (stay on the device).

Extra configure keys (not in the reference): ``FLUX_MODE`` ("reference" keeps
the reference's loop-carried x-face wave speeds in PPM/WENO; "conservative"
evaluates every face once with its own speeds and applies the resistive term
once for every reconstruction), ``PRECISION`` ("fp64" | "mixed"),
``C2P_GUESS`` ("reference" | "learned").
"""
import numpy as np

from .. import _lib
from ._engine import Engine
from .srhd_core import _pointwise

GAMMA = 5.0 / 3.0
P_MAX = 1.0
V_MAX = 0.999
GLM_CH = 1.0
GLM_CP = 0.1
LIMITER_ID = 0
RECON_ID = 0
RIEMANN_ID = 0
SMALL = 1e-12
RESISTIVE_ENABLED = False
RESISTIVITY = 0.0
N_PASSIVE = 0
PASSIVE_OFFSET = 9

_E = Engine(_lib.RMHD)


def configure(params):
    global GAMMA, P_MAX, V_MAX, GLM_CH, GLM_CP, LIMITER_ID, RECON_ID, RIEMANN_ID
    global N_PASSIVE, PASSIVE_OFFSET, RESISTIVE_ENABLED, RESISTIVITY
    _E.configure(params)
    p = _E.p
    GAMMA, P_MAX, V_MAX, GLM_CH, GLM_CP = p.gamma, p.p_max, p.v_max, p.glm_ch, p.glm_cp
    LIMITER_ID, RECON_ID, RIEMANN_ID = p.limiter, p.recon, p.riemann
    RESISTIVE_ENABLED, RESISTIVITY = bool(p.resistive), p.resistivity
    N_PASSIVE, PASSIVE_OFFSET = p.n_passive, p.passive_offset


def _rhs_with(recon, pr, nx, ny, nz, dx, dy, dz):
    saved = _E.p.recon
    _E.p.recon = recon
    try:
        return _E.rhs(pr, nx, ny, nz, dx, dy, dz)
    finally:
        _E.p.recon = saved


def compute_rhs_rmhd(pr, nx, ny, nz, dx, dy, dz):
    return _rhs_with(0, pr, nx, ny, nz, dx, dy, dz)


def compute_rhs_ppm(pr, nx, ny, nz, dx, dy, dz):
    return _rhs_with(1, pr, nx, ny, nz, dx, dy, dz)


def compute_rhs_weno(pr, nx, ny, nz, dx, dy, dz):
    return _rhs_with(2, pr, nx, ny, nz, dx, dy, dz)


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


def prim_to_cons_rmhd(rho, vx, vy, vz, p, Bx, By, Bz, psi, gamma=None):
    """Scalars (as the reference) or equal-shaped arrays/tensors.  As in the
    reference, an omitted gamma means the import-time default 5/3
    (core/rmhd_core.py:138); hot-path callers pass GAMMA explicitly."""
    g = 5.0 / 3.0 if gamma is None else float(gamma)
    saved = _E.p.gamma
    _E.p.gamma = g
    try:
        return _pointwise(_E.p2c_array, (rho, vx, vy, vz, p, Bx, By, Bz, psi))
    finally:
        _E.p.gamma = saved


def cons_to_prim_rmhd(D, Sx, Sy, Sz, tau, Bx, By, Bz, psi):
    return _pointwise(_E.c2p_array, (D, Sx, Sy, Sz, tau, Bx, By, Bz, psi))


def set_c2p_network(params):
    """Parameter block of the learned con2prim guess used when
    C2P_GUESS='learned' (defaults to the packaged trained network)."""
    _E.set_network(params)


def c2p_stats(reset=False):
    return _E.c2p_stats(reset)


def engine():
    return _E
