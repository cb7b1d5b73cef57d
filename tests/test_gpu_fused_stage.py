"""The fused SSPRK stage kernel (stage.cu) against the per-direction face
passes + update (the split path, STAGE_KERNEL="split"), through the C ABI.

Both evaluate the same float32 faces from the same float32 primitive copy and
the same float64 update.  They are not bit-identical: the compiler contracts
and orders the two kernels' float32 arithmetic differently, which moves some
HLLC hydro fluxes by a float32 rounding (measured on B200: after one stage,
the induction and psi rows agree bit for bit and the hydro rows to 1e-7 of
their scale, in a few hundred of ~40 000 cells).  So the bars are: one stage
within 1e-6 of the split stage, and no less accurate against the float64
stage than the split stage is (per variable, within 10 %); a whole SSPRK step
no further from the float64 step than twice the split step's distance (con2prim
amplifies float32 rounding near its branches on these rough states).  Covered: WENO5 and PPM, HLLE and "hlld", SSPRK2 and SSPRK3, the
reference's and the learned con2prim start, passive rows, resistivity, block
extents that are not multiples of the 4 x 32 tile or of the 32-plane chunk,
and a float32 overflow that the fused kernel recomputes in float64 in place.
"""
import numpy as np
import pytest
import torch

import parity as PT
from astrofd_b200 import learned_c2p as LC
from astrofd_b200.core import rmhd_core
from astrofd_b200.workloads import rmhd_jet, rmhd_jet_config
from states import make_state

pytestmark = pytest.mark.gpu


def _step(pr, kernel, recon="weno", riemann="hlld", rk=3, guess="reference", prec="mixed",
          resist=True, steps=1, stage_only=False):
    n = pr.shape[2] - 6
    core, _, _ = rmhd_jet_config(n, 3)
    rmhd_core.configure(dict(core, RECON=recon, RIEMANN=riemann, PRECISION=prec,
                             FLUX_MODE="conservative", C2P_GUESS=guess, STAGE_KERNEL=kernel,
                             RESISTIVE_ENABLED=resist, RK_ORDER=rk))
    if guess == "learned":
        rmhd_core.set_c2p_network(LC.load())
    d = 1.0 / n
    a = torch.from_numpy(pr.copy()).cuda()
    rmhd_core.c2p_stats(reset=True)
    if stage_only:
        out = torch.empty_like(a)
        rmhd_core.step_stage(a, a, out, d, d, d, 0.3 * d, rk, 0)
        a = out
    else:
        for _ in range(steps):
            a = (rmhd_core.step_ssprk3 if rk == 3 else rmhd_core.step_ssprk2)(a, d, d, d, 0.3 * d)
    torch.cuda.synchronize()
    st = rmhd_core.c2p_stats(reset=True)
    assert st["wait_timeouts"] == 0
    return a.cpu().numpy()


def _per_var(a, b):
    return [np.abs(a[v] - b[v]).max() / max(np.abs(b[v]).max(), 1e-300) for v in range(b.shape[0])]


def _jet(shape, seed=3):
    pr = make_state(seed, shape, 3, "rmhd", n_extra=2, noise=0.1, bamp=0.1, vjet=0.9,
                    stripes=False)
    pr[9:] = 0.01 + 0.001 * np.random.default_rng(seed).random(pr[9:].shape)
    return pr


@pytest.mark.parametrize("recon,riemann,rk,guess", [
    ("weno", "hlld", 3, "reference"), ("weno", "hlld", 3, "learned"),
    ("weno", "hlle", 2, "reference"), ("ppm", "hlld", 3, "reference"),
    ("ppm", "hlle", 3, "learned")])
def test_fused_step_matches_split_step(recon, riemann, rk, guess):
    # 37 x 26 x 41 interior cells: partial tiles in y and z, two x chunks
    pr = _jet((37, 26, 41))
    fs = _step(pr, "fused", recon, riemann, rk, guess, stage_only=True)
    ss = _step(pr, "split", recon, riemann, rk, guess, stage_only=True)
    ds = _step(pr, "split", recon, riemann, rk, guess, prec="fp64", stage_only=True)
    assert np.isfinite(fs).all()
    assert PT.normwise(fs, ss) < 1e-6
    for ef, es in zip(_per_var(fs, ds), _per_var(ss, ds)):
        assert ef <= 1.1 * es + 1e-12, (ef, es)
    # a whole step: both mixed paths at the same distance from float64 (the
    # rough state's con2prim branches amplify float32 rounding either way)
    a = _step(pr, "fused", recon, riemann, rk, guess)
    b = _step(pr, "split", recon, riemann, rk, guess)
    d = _step(pr, "split", recon, riemann, rk, guess, prec="fp64")
    assert np.isfinite(a).all()
    ef, es = PT.normwise(a, d), PT.normwise(b, d)
    assert ef < 2.0 * es + 1e-6, (ef, es)


def _driver_run(kernel, prec, n=48, steps=8):
    """Driver-loop steps (ghost fills, SSPRK3 step, ghost fills, sources) of
    the unmagnetised W = 2.29 jet whose float64 runs stay 1e-12 apart."""
    from astrofd_b200.core import boundary, nozzle, source_terms
    core, noz, src = rmhd_jet_config(n, 3, vjet=0.9, sigma_amb=0.0, sigma_jet=0.0,
                                     boundaries="baseline")
    rmhd_core.configure(dict(core, PRECISION=prec, FLUX_MODE="conservative",
                             C2P_GUESS="reference", STAGE_KERNEL=kernel))
    d = 1.0 / n
    dt = core["CFL"] * d
    rng = np.random.default_rng(1234)
    a = torch.from_numpy(rmhd_jet(n, 3, sigma_amb=0.0)).cuda()

    def bcs(t):
        boundary.apply_outflow_yz(t, 3)
        boundary.apply_outflow_right_x(t, 3)
        nozzle.apply_nozzle_left_x(t, d, d, d, n, n, 0.5, 0.5, rng, noz)

    for _ in range(steps):
        bcs(a)
        a = rmhd_core.step_ssprk3(a, d, d, d, dt)
        bcs(a)
        source_terms.apply_cooling_heating(a, dt, src)
        source_terms.apply_two_temperature(a, dt, src)
    torch.cuda.synchronize()
    return a.cpu().numpy()


def test_fused_jet_run_matches_split_and_float64():
    fused, split = _driver_run("fused", "mixed"), _driver_run("split", "mixed")
    f64 = _driver_run("split", "fp64")
    ef, es = PT.normwise(fused, f64), PT.normwise(split, f64)
    assert ef < 1e-5 and es < 1e-5, (ef, es)
    assert ef < 1.5 * es + 1e-9, (ef, es)
    assert PT.normwise(fused, split) < 1e-5


def test_fused_recomputes_float32_overflows_in_float64():
    """Fields of ~1e12: every float32 face overflows and is recomputed in
    float64 inside the fused kernel; the step then matches the split path,
    whose fix-up kernel does the same recomputation."""
    pr = _jet((20, 20, 20), seed=9)
    rng = np.random.default_rng(4)
    pr[5:8] = 1e12 * (1.0 + 0.5 * rng.random(pr[5:8].shape))
    pr[4] = 1e20
    a = _step(pr, "fused", resist=False, stage_only=True)
    b = _step(pr, "split", resist=False, stage_only=True)
    assert np.isfinite(a).all() and np.isfinite(b).all()
    assert PT.normwise(a, b) < 1e-6
