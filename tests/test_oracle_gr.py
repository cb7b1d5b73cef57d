"""Fixed-metric GR wrappers (core/grhd_core.py, core/grmhd_core.py,
core/gr_metric.py): the oracle and the drop-in metric helpers against
fixtures made by the reference's own code (tests/golden/make_golden.py).

Tolerances as for the core schemes: right-hand sides 1e-10 normwise, steps
1e-7 (con2prim stops at |f| < 1e-10 max(1, tau)); the scalar metric helpers
bit-exact (the same floating-point operations).
"""
import json
import os

import numpy as np
import pytest

import oracle as O
import parity as PT
from cases import GR_CASES
from astrofd_b200.core import gr_metric

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    d = np.load(os.path.join(HERE, name + ".npz"))
    return d, json.loads(str(d["params"])), json.loads(str(d["gr"]))


@pytest.mark.parametrize("case", GR_CASES, ids=[c["name"] for c in GR_CASES])
def test_oracle_rhs_and_step_match_reference(case):
    d, params, gcfg = load(case["name"])
    P = O.params_from_config(case["physics"], params)
    gr = O.gr_struct(gcfg, case["ng"], case["offs_x"])
    dx = 1.0 / case["n"]
    r = O.rhs_gr(P, gr, d["pr_in"], dx, dx, dx)
    assert r.shape == d["rhs"].shape
    assert PT.normwise(r, d["rhs"]) < 1e-10
    s = O.step_gr(P, gr, d["pr_in"], dx, dx, dx, float(d["dt"]), case["rk"])
    assert PT.normwise(s, d["step_out"]) < 1e-7
    if gcfg["GR_METRIC"] != "minkowski":
        # the metric terms are far above the tolerance on these states
        assert PT.normwise(O.rhs(P, d["pr_in"], dx, dx, dx), d["rhs"]) > 1e-2


def test_metric_helpers_match_reference():
    d = np.load(os.path.join(HERE, "gr_metric.npz"))
    for p, iso, ks, kerr in zip(d["pts"], d["iso"], d["ks"], d["kerr"]):
        assert gr_metric.schwarzschild_iso_lapse_and_grad(*p, 0.05) == tuple(iso)
        assert gr_metric.schwarzschild_ks_lapse_shift_and_grad(*p, 0.05) == tuple(ks)
        assert gr_metric.kerr_schild_lapse_shift_and_grad(*p, 0.05, 0.7) == tuple(kerr)
