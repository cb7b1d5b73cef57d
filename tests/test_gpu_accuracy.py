"""The headline path's accuracy bar where it is measurable.

The 256^3 benchmark jet (W = 10, sigma_jet = 0.5 on an ambient sigma = 0.01)
is chaotic in the reference's own scheme: two float64 runs that differ by
1e-12 in density differ by O(1) within ~40 steps, so no comparison of two
runs of it means anything at 100 steps (any magnetic field does this: an
ambient sigma of 1e-4 already, measured at 256^3).  Its stable member -- the
same scheme and sources (RMHD, Gamma 4/3, WENO5 + "hlld", SSPRK3, CFL 0.35,
resistivity, two-temperature, cooling, outflow boundaries) with an
unmagnetised jet at v = 0.99 (W = 7.09) -- keeps two float64 runs 1e-12
apart.  On it, mixed precision (float32
reconstruction and Riemann fluxes) with the learned con2prim start must stay
within density L1 < 1e-4 of plain float64 after 100 driver steps, and so must
each half of it (float32 faces with the reference's start, float64 faces with
the learned start).
"""
import pytest

from astrofd_b200.driver import STABLE, rho_l1_arms

pytestmark = pytest.mark.gpu


def test_stable_jet_100_steps_within_the_l1_bar():
    out = rho_l1_arms(64, 100, every=25, **STABLE)
    r = out["rho_l1"]
    # the flow is not chaotic: the float64 perturbation floor stays tiny
    assert r["fp64_perturbed_1e-12"] < 1e-9, out["rho_l1_history"]
    assert r["mixed_learned"] < 1e-4, out["rho_l1_history"]
    assert r["mixed_reference_guess"] < 1e-4
    assert r["fp64_learned_guess"] < 1e-4
    c = out["c2p_counts"]["mixed_learned"]
    assert c["wait_timeouts"] == 0
