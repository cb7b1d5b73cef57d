"""The oracle's chemistry (core/chemistry.py:43) and causal dissipation
(core/dissipation.py:5) against fixtures from the reference's own code
(tests/golden/make_golden.py): bit-exact."""
import json

import numpy as np
import pytest

import oracle as O
import parity as PT


@pytest.mark.parametrize("tag", ["nominal", "fast"])
def test_chemistry_matches_reference(tag):
    d = PT.load("chemistry")
    pr = d["pr_in"].copy()
    O.apply_ion_chemistry(pr, float(d["dt"]), json.loads(str(d["cfg_" + tag])))
    assert np.array_equal(pr, d[tag])
    assert (d[tag] != d["pr_in"]).any()


@pytest.mark.parametrize("tag", ["full", "noadvect"])
def test_dissipation_matches_reference(tag):
    d = PT.load("dissipation")
    pr = d["pr_in"].copy()
    h = float(d["dx"])
    O.apply_causal_dissipation(pr, float(d["dt"]), h, h, h, json.loads(str(d["cfg_" + tag])))
    assert np.array_equal(pr, d[tag])
    assert (d[tag] != d["pr_in"]).any()
