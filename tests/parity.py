"""Shared parity metrics and golden-fixture helpers (test infrastructure)."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def params_of(d, key="params"):
    return json.loads(str(d[key]))


def normwise(a, b, mask=None):
    """max over variables of max|a_v - b_v| / max|b_v| (per-variable scale)."""
    worst = 0.0
    for v in range(b.shape[0]):
        av, bv = a[v], b[v]
        if mask is not None:
            av, bv = av[mask], bv[mask]
        if bv.size == 0:
            continue
        s = np.abs(bv).max()
        e = np.abs(av - bv).max()
        worst = max(worst, e / s if s > 0 else e)
    return worst


def sane_mask(pr, physics):
    """Cells whose reference state has not blown up (the reference's
    experimental HLLD drives fields to 1e10+ on rough states, where
    con2prim is ill-conditioned)."""
    m = np.all(np.isfinite(pr), axis=0) & (pr[0] < 1e3)
    if physics == "rmhd":
        m &= np.sqrt((pr[5:8] ** 2).sum(axis=0)) < 1e2
    return m

