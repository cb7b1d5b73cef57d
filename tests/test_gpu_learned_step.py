"""Stage updates with the learned con2prim guess (C2P_GUESS="learned") against
the same step with the reference's guess, through astro_step.

Both solve the reference's con2prim equation (rmhd_f_of_Z, core/rmhd_core.py:229)
to the same tolerance |f| < 1e-10 max(1, tau) from different starting points,
so the primitives agree to that tolerance, not bit for bit.  One driver step
(three stages) of a 32^3 magnetised jet is compared: at this resolution the
jet inlet sits on the pressure floor and the hydro fallback, discontinuous
branches that amplify 1e-10 differences to O(1) within a few steps in either
run.  Float64: 1e-8 of each variable's scale; mixed precision: 1e-6 (the
float32 fluxes of the later stages round the slightly different primitives
differently).

With no polish step allowed (astro_debug_set_step_polish(0)) nearly every
cell goes to the fallback list (a slot for every cell), and all of them are
solved by the fallback kernel.
"""
import numpy as np
import pytest
import torch

import parity as PT
from astrofd_b200 import learned_c2p as LC
from astrofd_b200.core import boundary, nozzle, rmhd_core
from astrofd_b200.workloads import rmhd_jet, rmhd_jet_config

pytestmark = pytest.mark.gpu

N, NG, STEPS = 32, 3, 1
TOL = {"fp64": 1e-8, "mixed": 1e-6}


def _run(precision, guess, params):
    core, noz, _ = rmhd_jet_config(N, NG)
    rmhd_core.configure(dict(core, PRECISION=precision, FLUX_MODE="conservative", C2P_GUESS=guess))
    if params is not None:
        rmhd_core.set_c2p_network(params)
    d = 1.0 / N
    dt = core["CFL"] * d
    rng = np.random.default_rng(7)
    a = torch.from_numpy(rmhd_jet(N, NG)).cuda()
    b = torch.empty_like(a)
    rmhd_core.c2p_stats(reset=True)
    for _ in range(STEPS):
        boundary.apply_periodic_yz(a, NG)
        boundary.apply_outflow_right_x(a, NG)
        nozzle.apply_nozzle_left_x(a, d, d, d, N, N, 0.5, 0.5, rng, noz)
        rmhd_core.step_ssprk3(a, d, d, d, dt, out=b)
        a, b = b, a
    stats = rmhd_core.c2p_stats(reset=True)
    if params is not None:
        rmhd_core.set_c2p_network(LC.load())
    return a.cpu().numpy(), stats


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_learned_guess_matches_reference_guess(precision):
    ref, _ = _run(precision, "reference", None)
    got, st = _run(precision, "learned", LC.load())
    assert np.isfinite(got).all()
    err = PT.normwise(got, ref)
    assert err < TOL[precision], err
    ncells = (N + 2 * NG) ** 3
    assert st["cells"] == 3 * STEPS * ncells
    assert st["learned_polish"] > 0.98 * st["cells"], st


def test_fallback_list_solves():
    from astrofd_b200 import _lib
    L = _lib.load()
    ref, _ = _run("fp64", "reference", None)
    assert L.astro_debug_set_step_polish(0) == 0
    try:
        got, st = _run("fp64", "learned", LC.load())
    finally:
        assert L.astro_debug_set_step_polish(-1) == 0
    nc = (N + 2 * NG) ** 3
    # most cells fell back and were listed
    assert st["learned_fallback"] > 0.5 * 3 * STEPS * nc, st
    assert np.isfinite(got).all()
    err = PT.normwise(got, ref)
    assert err < TOL["fp64"], err
