"""astro_step_stage (the drop-in cores' step_stage): the stages of one SSPRK
step run one call at a time give astro_step's result bit for bit, in float64
and in mixed precision with the learned con2prim; and a ghost refresh
between the stages is seen by the next stage."""
import numpy as np
import pytest
import torch

import parity as PT
from cases import CASE_BY_NAME
from astrofd_b200.core import rmhd_core, srhd_core

pytestmark = pytest.mark.gpu


def _configure(case, **extra):
    m = srhd_core if case["physics"] == "srhd" else rmhd_core
    p = dict(RESISTIVE_ENABLED=False, RESISTIVITY=0.0, FLUX_MODE="reference",
             PRECISION="fp64", C2P_GUESS="reference")
    p.update(case["params"])
    p.update(extra)
    m.configure(p)
    return m


def _chain(m, pr, d, dt, rk):
    bufs = [torch.empty_like(pr) for _ in range(2)]
    out = torch.empty_like(pr)
    cur = pr
    for st in range(rk):
        dst = out if st == rk - 1 else bufs[st % 2]
        m.step_stage(pr, cur, dst, d, d, d, dt, rk, st)
        cur = dst
    return out


@pytest.mark.parametrize("name,extra", [
    ("s_ppm_hllc_rk3", {}),
    ("s_muscl_minmod_hllc_is_pass1", {}),
    ("r_weno_hlld_rk3", {}),
    ("r_weno_hlld_rk3", dict(PRECISION="mixed", FLUX_MODE="conservative")),
    ("r_weno_hlldfull_c5", dict(PRECISION="mixed", FLUX_MODE="conservative",
                                C2P_GUESS="learned")),
])
def test_stage_chain_equals_step(name, extra):
    case = CASE_BY_NAME[name]
    m = _configure(case, **extra)
    if extra.get("C2P_GUESS") == "learned":
        from astrofd_b200 import learned_c2p
        rmhd_core.set_c2p_network(learned_c2p.load())
    d = PT.load(name)
    pr = torch.from_numpy(d["pr_in"]).cuda()
    dx, dt, rk = 1.0 / case["n"], float(d["dt"]), case["rk"]
    step = m.step_ssprk3 if rk == 3 else m.step_ssprk2
    ref = step(pr, dx, dx, dx, dt)
    got = _chain(m, pr, dx, dt, rk)
    assert torch.isfinite(got).all()
    assert torch.equal(got, ref)


def test_ghost_refresh_between_stages_is_used():
    case = CASE_BY_NAME["r_weno_hlld_rk3"]
    m = _configure(case)
    d = PT.load("r_weno_hlld_rk3")
    pr = torch.from_numpy(d["pr_in"]).cuda()
    dx, dt, ng = 1.0 / case["n"], float(d["dt"]), case["ng"]
    s1, s2, out = (torch.empty_like(pr) for _ in range(3))
    m.step_stage(pr, pr, s1, dx, dx, dx, dt, 3, 0)
    a = s1.clone()
    a[:, :ng] *= 1.01   # a stand-in for the x ghosts a neighbour would send
    m.step_stage(pr, a, s2, dx, dx, dx, dt, 3, 1)
    m.step_stage(pr, pr, s1, dx, dx, dx, dt, 3, 0)   # redo stage 0: U back to stage 0
    m.step_stage(pr, s1, out, dx, dx, dx, dt, 3, 1)
    inner = out[:, ng:ng + 2, ng:-ng, ng:-ng]
    assert not torch.equal(s2[:, ng:ng + 2, ng:-ng, ng:-ng], inner)
    assert torch.equal(s2[:, -ng - 3:-ng, ng:-ng, ng:-ng], out[:, -ng - 3:-ng, ng:-ng, ng:-ng])
