"""Recovery paths of the float32 faces and of the learned con2prim, through
the C ABI on the device.

* More non-finite float32 faces than the float64 fix-up list holds (its
  capacity is nc/16 + 1024 faces per pass): every face of the pass is then
  checked and the failed ones recomputed in float64, so the mixed right-hand
  side still matches the float64 one instead of keeping NaN fluxes.
* A tensor-core wait of the learned con2prim that gives up (made to give up
  here by a poll limit of one poll, while the MMAs are still running): the
  thread block finishes its cells from the analytic start, waits for the MMAs
  still in flight before freeing its tensor memory, and the step counts the
  event in AstroC2PStats.wait_timeouts; the primitives are the full solve's.
* A tile-load wait of the fused stage kernel that gives up: the block waits
  for its loads still in flight, stops and is counted in wait_timeouts.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import parity as PT
from astrofd_b200 import _lib, learned_c2p as LC
from astrofd_b200.core import boundary, nozzle, rmhd_core
from astrofd_b200.workloads import rmhd_jet, rmhd_jet_config
from states import make_state

pytestmark = pytest.mark.gpu


def _rmhd_params(precision):
    p = _lib.AstroParams()
    p.physics, p.recon, p.riemann, p.limiter = _lib.RMHD, 2, 1, 0
    p.passive_offset = 9
    p.gamma = p.srhd_gamma = 4.0 / 3.0
    p.p_max, p.v_max, p.glm_ch, p.glm_cp = 1e60, 0.9999, 1.0, 0.1
    p.flux_mode = _lib.FLUX_CONSERVATIVE
    p.precision = precision
    return p


def _rhs(L, p, pr):
    nv, nx, ny, nz = pr.shape
    g = _lib.AstroGrid(nv, nx, ny, nz, 1 / 20, 1 / 20, 1 / 20)
    nb = L.astro_rhs_workspace_bytes(C.byref(p), C.byref(g))
    w = torch.empty(nb, dtype=torch.uint8, device="cuda")
    out = torch.full((9, nx, ny, nz), float("nan"), dtype=torch.float64, device="cuda")
    rc = L.astro_rhs(C.byref(p), C.byref(g), C.c_void_p(pr.data_ptr()),
                     C.c_void_p(out.data_ptr()), C.c_void_p(w.data_ptr()), nb, None)
    assert rc == 0, L.astro_error_string(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_float32_fixup_list_overflow_recomputes_every_failed_face():
    """Fields of ~1e12 with O(1) relative jumps: the squared WENO smoothness
    indicators (~1e24, squared again in the weights) overflow float32 on every
    face while the fluxes (~B^2) still fit, so all ~3 x 20^3 faces fail, far
    more than the list's 1024 + 26^3/16 slots."""
    L = _lib.load()
    pr = make_state(41, 20, 3, "rmhd", noise=0.1, bamp=0.1, vjet=0.5, stripes=False)
    rng = np.random.default_rng(3)
    pr[5:8] = 1e12 * (1.0 + 0.5 * rng.random(pr[5:8].shape))
    pr[4] = 1e20
    t = torch.from_numpy(pr).cuda()
    ref = _rhs(L, _rmhd_params(_lib.PREC_FP64), t)
    got = _rhs(L, _rmhd_params(_lib.PREC_MIXED), t)
    assert np.isfinite(ref).all()
    assert np.isfinite(got).all()
    # the recomputed fluxes are stored as float32: relative rounding ~1e-7
    assert PT.normwise(got, ref) < 1e-5


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_learned_con2prim_recovers_from_a_wait_that_gives_up(precision):
    L = _lib.load()
    N, NG = 32, 3
    core, noz, _ = rmhd_jet_config(N, NG)
    d = 1.0 / N
    # the magnetised jet's block with its ghost fills (nozzle inflow), as in
    # the learned-guess step test
    base = torch.from_numpy(rmhd_jet(N, NG)).cuda()
    boundary.apply_periodic_yz(base, NG)
    boundary.apply_outflow_right_x(base, NG)
    nozzle.apply_nozzle_left_x(base, d, d, d, N, N, 0.5, 0.5, np.random.default_rng(7), noz)

    def step(guess):
        rmhd_core.configure(dict(core, PRECISION=precision, FLUX_MODE="conservative",
                                 C2P_GUESS=guess))
        rmhd_core.set_c2p_network(LC.load())
        rmhd_core.c2p_stats(reset=True)
        out = rmhd_core.step_ssprk3(base.clone(), d, d, d, core["CFL"] * d)
        torch.cuda.synchronize()
        return out.cpu().numpy(), rmhd_core.c2p_stats(reset=True)

    ref, st_ref = step("reference")
    normal, st_normal = step("learned")
    assert st_normal["wait_timeouts"] == 0
    assert L.astro_debug_set_mma_poll_limit(1) == 0
    try:
        got, st = step("learned")
    finally:
        assert L.astro_debug_set_mma_poll_limit(0) == 0
    assert st["wait_timeouts"] > 0, st
    assert st["cells"] == st_normal["cells"]
    assert np.isfinite(got).all()
    tol = 1e-8 if precision == "fp64" else 1e-6
    assert PT.normwise(got, ref) < tol
    assert PT.normwise(got, normal) < tol
    # the device still runs the network normally afterwards
    again, st_again = step("learned")
    assert st_again["wait_timeouts"] == 0
    assert PT.normwise(again, normal) == 0.0


def test_fused_stage_reports_a_tile_wait_that_gives_up():
    """The fused stage kernel's tile-load waits are bounded.  With a budget of
    one non-blocking poll (astro_debug_set_tile_poll_limit(1)) they give up
    while the TMA loads are still in flight: every block then waits for its
    loads with the full budget before its shared memory goes away, stops, and
    counts itself in AstroC2PStats.wait_timeouts, so the caller learns that
    the step's result is invalid.  The device stays usable: the next step,
    with the default budget, equals a normal fused step bit for bit."""
    L = _lib.load()
    N, NG = 32, 3
    core, noz, _ = rmhd_jet_config(N, NG)
    d = 1.0 / N
    base = torch.from_numpy(rmhd_jet(N, NG)).cuda()
    boundary.apply_periodic_yz(base, NG)
    boundary.apply_outflow_right_x(base, NG)
    nozzle.apply_nozzle_left_x(base, d, d, d, N, N, 0.5, 0.5, np.random.default_rng(7), noz)
    rmhd_core.configure(dict(core, PRECISION="mixed", FLUX_MODE="conservative",
                             C2P_GUESS="reference", STAGE_KERNEL="fused"))

    def step():
        rmhd_core.c2p_stats(reset=True)
        out = rmhd_core.step_ssprk3(base.clone(), d, d, d, core["CFL"] * d)
        torch.cuda.synchronize()
        return out.cpu().numpy(), rmhd_core.c2p_stats(reset=True)

    try:
        normal, st_normal = step()
        assert st_normal["wait_timeouts"] == 0
        assert np.isfinite(normal).all()
        assert L.astro_debug_set_tile_poll_limit(1) == 0
        try:
            _, st = step()
        finally:
            assert L.astro_debug_set_tile_poll_limit(0) == 0
        assert st["wait_timeouts"] > 0, st
        again, st_again = step()
        assert st_again["wait_timeouts"] == 0
        assert np.array_equal(again, normal)
    finally:
        rmhd_core.configure(dict(core, STAGE_KERNEL="split"))


def test_polish_reciprocal_within_two_ulp_of_the_ieee_quotient():
    """The learned polish replaces float64 division by the hardware reciprocal
    approximation refined by two Newton-Raphson steps (rcp_nr): over normal
    values of both signs from 1e-300 to 1e300 (and exact powers of two) it is
    within 2 ulp of the IEEE quotient 1/x."""
    L = _lib.load()
    rng = np.random.default_rng(5)
    x = 10.0 ** rng.uniform(-300, 300, 1 << 20)
    x *= np.where(rng.random(x.size) < 0.5, -1.0, 1.0)
    x = np.concatenate([x, 2.0 ** np.arange(-1000, 1001, 7), [1.0, -1.0, 3.0, 1e-24, 1e300]])
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    assert L.astro_debug_rcp_f64(C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()), x.size,
                                 None) == 0
    torch.cuda.synchronize()
    y = yd.cpu().numpy()
    ref = 1.0 / x
    ulp = np.spacing(np.abs(ref))
    assert np.all(np.abs(y - ref) <= 2 * ulp), np.max(np.abs(y - ref) / ulp)
