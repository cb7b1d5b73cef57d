"""Chemistry (core/chemistry.py:43) and causal dissipation
(core/dissipation.py:5) on the device, through the drop-in modules and the C
ABI, against fixtures from the reference's own code.  1e-13 relative: CUDA's
exp and pow differ from the host libm's by an ulp or two, and the device may
contract a*b + c into one rounding."""
import json

import numpy as np
import pytest
import torch

import parity as PT
from astrofd_b200.core import chemistry, dissipation

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", ["nominal", "fast"])
def test_chemistry_on_device(tag):
    d = PT.load("chemistry")
    cfg = json.loads(str(d["cfg_" + tag]))
    t = torch.from_numpy(d["pr_in"].copy()).cuda()
    out = chemistry.apply_ion_chemistry(t, float(d["dt"]), cfg)
    assert out is t
    np.testing.assert_allclose(t.cpu().numpy(), d[tag], rtol=1e-13, atol=1e-300)
    # numpy blocks: filled in place through the device
    h = d["pr_in"].copy()
    chemistry.apply_ion_chemistry(h, float(d["dt"]), cfg)
    np.testing.assert_allclose(h, d[tag], rtol=1e-13, atol=1e-300)


@pytest.mark.parametrize("tag", ["full", "noadvect"])
def test_dissipation_on_device(tag):
    d = PT.load("dissipation")
    cfg = json.loads(str(d["cfg_" + tag]))
    h = float(d["dx"])
    t = torch.from_numpy(d["pr_in"].copy()).cuda()
    out = dissipation.apply_causal_dissipation(t, float(d["dt"]), h, h, h, cfg)
    assert out is t
    got = t.cpu().numpy()
    assert PT.normwise(got, d[tag]) < 1e-13
    np.testing.assert_array_equal(got[:5], d[tag][:5])


def test_gating_leaves_block_untouched():
    d = PT.load("dissipation")
    cfg = json.loads(str(d["cfg_full"]))
    t = torch.from_numpy(d["pr_in"].copy()).cuda()
    dissipation.apply_causal_dissipation(t, 0.01, 0.1, 0.1, 0.1, dict(cfg, PHYSICS="rmhd"))
    chemistry.apply_ion_chemistry(t, 0.01, dict(CHEMISTRY_ENABLED=True, N_CHEM=2))
    assert np.array_equal(t.cpu().numpy(), d["pr_in"])
