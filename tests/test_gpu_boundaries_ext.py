"""Device ghost fills that the reference lacks (zero-gradient y/z faces; the
nozzle's zero-gradient ambient part of the x = 0 face and its B_phi(r)
profile) against the oracle's restatement, through the C ABI.  Copies are
exact; the nozzle's jet state to 1e-14 relative (contraction of a*b + c on the
device)."""
import numpy as np
import pytest
import torch

import oracle as O
from astrofd_b200.core import boundary, nozzle

pytestmark = pytest.mark.gpu


def _block(nv, n, ng, seed):
    return np.random.default_rng(seed).standard_normal((nv, n + 2 * ng, n + 2 * ng, n + 2 * ng))


@pytest.mark.parametrize("ng", [2, 3])
def test_outflow_yz_matches_oracle(ng):
    host = _block(11, 14, ng, 3)
    dev = torch.from_numpy(host.copy()).cuda()
    boundary.apply_outflow_yz(dev, ng)
    O.apply_outflow_yz(host, ng)
    assert np.array_equal(dev.cpu().numpy(), host)


@pytest.mark.parametrize("shear", [0.0, 0.03])
@pytest.mark.parametrize("perturb", ["none", "random"])
def test_nozzle_outflow_ambient_and_toroidal_phi_match_oracle(shear, perturb):
    n, ng = 16, 3
    d = 1.0 / n
    cfg = dict(NG=ng, JET_RADIUS=0.2, SHEAR_THICK=shear, NOZZLE_PROFILE="top_hat",
               GAMMA_JET=10.0, ETA_RHO=0.1, P_EQ=0.01, RHO_AMB=1.0, VX_AMB=0.0, VY_AMB=0.0,
               VZ_AMB=0.0, NOZZLE_PERTURB=perturb, TURB_VAMP=0.01, TURB_PAMP=0.01,
               PHYSICS="rmhd", B_INIT="toroidal_phi", B0=2.5, B_AMB_X=0.1,
               NOZZLE_AMBIENT="outflow", N_TRACERS=0, TWO_TEMPERATURE=True, THERMO_OFFSET=9,
               TE_NOZZLE=0.1, TI_NOZZLE=0.1)
    host = _block(11, n, ng, 4)
    dev = torch.from_numpy(host.copy()).cuda()
    nozzle.apply_nozzle_left_x(dev, d, d, d, n, n, 0.5, 0.5, np.random.default_rng(9), cfg)
    O.apply_nozzle_left_x(host, d, d, d, n, n, 0.5, 0.5, np.random.default_rng(9), cfg)
    got = dev.cpu().numpy()
    assert np.allclose(got, host, rtol=1e-14, atol=1e-300)
