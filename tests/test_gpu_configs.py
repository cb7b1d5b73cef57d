"""The SRHD jet configurations at their own sizes, float64 on the device
against the oracle (the C restatement of the reference, pinned to the
reference's Numba kernels by tests/test_oracle_golden.py).

C1: 64^3, Gamma 5/3, MUSCL-minmod + HLLE, SSPRK2, CFL 0.4, 10 driver steps
with the reference's CFL rule (amax from max_char_speed before the ghost
fill).  The C2 scheme (PPM + HLLC, SSPRK3, v_jet 0.995) on a 48^3 grid, one
driver step: at the inlet of this W = 10 jet the reference's SRHD con2prim
(a fixed point with a 60-iteration cap, a fallback and p / v caps) is
discontinuous in its input, so a 1e-15 change of rho flips ~0.2 % of the cells
in the first interior x layers between branches (p at the floor or at P_MAX)
in the oracle itself.  Cells differing by more than 1e-8 of a variable's scale
must therefore stay few (< 1 %) and within the first four interior x layers;
all other cells agree to 1e-10.  Both with the reference driver's boundaries and with outflow on every
face but the nozzle.  Both sides take the oracle's time step (amax of a
W = 10 jet sits next to the clip at 1, where round-off-level state differences
move it by ~1e-8; the device reduction itself is checked on identical states
in test_gpu_parity.py); the device's own time steps agree to 1e-6.  States to
1e-10 of each variable's scale (the RHS agrees to ~1e-12; the con2prim's
iteration counts can differ at its 1e-12 tolerance).
"""
import numpy as np
import pytest
import torch

import oracle as O
import parity as PT
from astrofd_b200.core import boundary, nozzle, srhd_core
from astrofd_b200.workloads import srhd_jet, srhd_jet_config

pytestmark = pytest.mark.gpu


def _loops(n, ng, steps, boundaries, **scheme):
    core, noz = srhd_jet_config(n, ng, boundaries=boundaries, **scheme)
    d = 1.0 / n
    outflow = noz.get("YZ_BOUNDARY") == "outflow"
    srhd_core.configure(dict(core, PRECISION="fp64", FLUX_MODE="reference"))
    P = O.params_from_config("srhd", dict(core, FLUX_MODE="reference"))
    rng_d, rng_h = np.random.default_rng(1234), np.random.default_rng(1234)
    a = torch.from_numpy(srhd_jet(n, ng)).cuda()
    h = srhd_jet(n, ng)
    N = h.shape[1]

    def bcs_dev(t):
        (boundary.apply_outflow_yz if outflow else boundary.apply_periodic_yz)(t, ng)
        boundary.apply_outflow_right_x(t, ng)
        nozzle.apply_nozzle_left_x(t, d, d, d, n, n, 0.5, 0.5, rng_d, noz)

    def bcs_host(t):
        (O.apply_outflow_yz if outflow else O.apply_periodic_yz)(t, ng)
        O.apply_outflow_right_x(t, ng)
        O.apply_nozzle_left_x(t, d, d, d, n, n, 0.5, 0.5, rng_h, noz)

    step = srhd_core.step_ssprk3 if core["RK_ORDER"] == 3 else srhd_core.step_ssprk2
    dts_dev, dts_host = [], []
    for _ in range(steps):
        dts_dev.append(core["CFL"] * d / max(srhd_core.max_char_speed(a, N, N, N), 1e-12))
        dt = core["CFL"] * d / max(O.max_char_speed(h), 1e-12)
        dts_host.append(dt)
        bcs_dev(a)
        a = step(a, d, d, d, dt)
        bcs_dev(a)
        bcs_host(h)
        h = O.step(P, h, d, d, d, dt, core["RK_ORDER"])
        bcs_host(h)
    return a.cpu().numpy(), np.array(dts_dev), h, np.array(dts_host)


@pytest.mark.parametrize("boundaries", ["reference", "baseline"])
def test_c1_64cube_10_steps_vs_oracle(boundaries):
    got, dts, ref, dts_ref = _loops(64, 2, 10, boundaries)
    np.testing.assert_allclose(dts, dts_ref, rtol=1e-6)
    assert np.isfinite(got).all()
    err = PT.normwise(got, ref)
    assert err < 1e-10, err


@pytest.mark.parametrize("boundaries", ["reference", "baseline"])
def test_c2_scheme_48cube_5_steps_vs_oracle(boundaries):
    ng = 3
    got, dts, ref, dts_ref = _loops(48, ng, 1, boundaries, vjet=0.995, recon="ppm",
                                    riemann="hllc", rk_order=3)
    np.testing.assert_allclose(dts, dts_ref, rtol=1e-6)
    assert np.isfinite(got).all()
    scale = np.abs(ref).reshape(ref.shape[0], -1).max(1)[:, None, None, None]
    inner = (slice(None), slice(ng, -ng), slice(ng, -ng), slice(ng, -ng))
    flipped = (np.abs(got - ref) / scale)[inner].max(0) > 1e-8
    assert flipped.mean() < 0.01, flipped.sum()
    assert np.argwhere(flipped)[:, 0].max(initial=0) < 4
    err = PT.normwise(got[inner], ref[inner], mask=~flipped)
    assert err < 1e-10, err
