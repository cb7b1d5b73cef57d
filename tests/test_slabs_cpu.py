"""x-slab decomposition (astrofd_b200/slabs.py) on the CPU over gloo.

decompose_x against solvers/srhd3d_mpi_muscl.py:92-97; the ghost exchange
against the one-block array; and the reference driver's multi-rank loop
(exchange, boundary fills with the nozzle on the first rank and the +x
outflow on the last, step, fills; solvers/srhd3d_mpi_muscl.py:286-324) run on
2 and 3 gloo ranks with the oracle's step, bit-exact against the same loop
emulated in one process with the exchange done by array copies.
"""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
from astrofd_b200.slabs import decompose_x
from astrofd_b200.workloads import srhd_jet_config

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N, NG, STEPS = 12, 2, 3


def test_decompose_x():
    assert decompose_x(10, 3, 0) == (4, 0, [4, 3, 3], [0, 4, 7])
    assert decompose_x(10, 3, 2) == (3, 7, [4, 3, 3], [0, 4, 7])
    assert decompose_x(256, 8, 5)[:2] == (32, 160)
    for nx, size in ((13, 2), (13, 3), (7, 7), (100, 6)):
        c = decompose_x(nx, size, 0)[2]
        assert sum(c) == nx and max(c) - min(c) <= 1


def global_block(nx_glob):
    rng = np.random.default_rng(77)
    pr = np.zeros((5, nx_glob + 2 * NG, N + 2 * NG, N + 2 * NG))
    pr[0] = 1.0 + 0.01 * (2.0 * rng.random(pr.shape[1:]) - 1.0)
    pr[1:4] = 0.05 * rng.standard_normal((3,) + pr.shape[1:])
    pr[4] = 0.01
    return pr


def bcs(a, first, last, rng, noz):
    d = 1.0 / N
    O.apply_periodic_yz(a, NG)
    if last:
        O.apply_outflow_right_x(a, NG)
    if first:
        O.apply_nozzle_left_x(a, d, d, d, N, N, 0.5, 0.5, rng, noz)


def params():
    core, noz = srhd_jet_config(N, NG)
    return O.params_from_config("srhd", dict(core, FLUX_MODE="reference")), noz, core


CHILD = r"""
import sys
for p in ({root!r}, {oracle!r}, {tests!r}):
    sys.path.insert(0, p)
import numpy as np, torch, torch.distributed as dist
import oracle as O
import test_slabs_cpu as T
from astrofd_b200.slabs import SlabDomain
dist.init_process_group("gloo", init_method="env://")
rank = dist.get_rank()
G = T.global_block({nx})
dom = SlabDomain({nx}, T.NG)
lo, hi = dom.offset, dom.offset + dom.nx + 2 * T.NG
pr = torch.from_numpy(G[:, lo:hi].copy())
# the exchange alone: spoiled ghosts come back as the one-block array's cells
pr[:, :T.NG] = float("nan")
pr[:, -T.NG:] = float("nan")
dom.exchange(pr)
a = pr.numpy()
inner = slice(0 if not dom.first else T.NG, a.shape[1] - (0 if not dom.last else T.NG))
assert np.array_equal(a[:, inner], G[:, lo:hi][:, inner]), "exchange"
P, noz, core = T.params()
dt = core["CFL"] / T.N
rng = np.random.default_rng(1234 + rank * 777)
for s in range(T.STEPS):
    dom.exchange(pr)
    a = pr.numpy()
    T.bcs(a, dom.first, dom.last, rng, noz)
    a = O.step(P, a, 1.0 / T.N, 1.0 / T.N, 1.0 / T.N, dt, 2)
    T.bcs(a, dom.first, dom.last, rng, noz)
    pr = torch.from_numpy(a)
np.save({out!r} + f"/rank{{rank}}.npy", pr.numpy())
dist.destroy_process_group()
"""


def _emulate(nx, size):
    """The same loop with the exchange as array copies between the slabs."""
    G = global_block(nx)
    P, noz, core = params()
    dt = core["CFL"] / N
    doms = [decompose_x(nx, size, r) for r in range(size)]
    slabs = [G[:, o:o + c + 2 * NG].copy() for c, o, _, _ in doms]
    rngs = [np.random.default_rng(1234 + r * 777) for r in range(size)]
    for _ in range(STEPS):
        send = [(s[:, NG:2 * NG].copy(), s[:, -2 * NG:-NG].copy()) for s in slabs]
        for r, s in enumerate(slabs):
            if r > 0:
                s[:, :NG] = send[r - 1][1]
            if r + 1 < size:
                s[:, -NG:] = send[r + 1][0]
        for r in range(size):
            a = slabs[r]
            bcs(a, r == 0, r == size - 1, rngs[r], noz)
            a = O.step(P, a, 1.0 / N, 1.0 / N, 1.0 / N, dt, 2)
            bcs(a, r == 0, r == size - 1, rngs[r], noz)
            slabs[r] = a
    return slabs


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("size,nx", [(2, 13), (3, 14)])
def test_driver_loop_on_gloo_ranks_matches_emulation(size, nx, tmp_path):
    port = _free_port()
    code = CHILD.format(root=ROOT, oracle=os.path.join(ROOT, "oracle"),
                        tests=os.path.join(ROOT, "tests"), nx=nx, out=str(tmp_path))
    procs = []
    for r in range(size):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(size), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, text=True,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE))
    try:
        for p in procs:
            _, err = p.communicate(timeout=240)
            assert p.returncode == 0, err[-3000:]
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    want = _emulate(nx, size)
    for r in range(size):
        got = np.load(tmp_path / f"rank{r}.npy")
        assert np.isfinite(got).all()
        assert np.array_equal(got, want[r]), r


# ---- per-stage exchange: the ranks compute exactly what one block would ----

def stage_case(phys):
    """(G, params, rk, dt, d, ng): a seeded block whose right-hand-side bounds
    cover its whole interior (PPM with NG = 3; RMHD MUSCL with NG = 2), ghosts
    filled once as the driver does before a step."""
    import states
    if phys == "srhd":
        ng, rk = 3, 3
        cfg = dict(GAMMA=5 / 3, P_MAX=2.0, V_MAX=0.9999, RECON="ppm", LIMITER="mc",
                   RIEMANN="hllc", N_PASSIVE=0, PASSIVE_OFFSET=5)
    else:
        ng, rk = 2, 2
        cfg = dict(GAMMA=4 / 3, P_MAX=2.0, V_MAX=0.9999, GLM_CH=1.0, GLM_CP=0.1, RECON="muscl",
                   LIMITER="mc", RIEMANN="hlle", N_PASSIVE=0, PASSIVE_OFFSET=9)
    pr = states.make_state(31 if phys == "srhd" else 32, 8, ng, phys, 0, noise=0.2, bamp=0.1,
                           vjet=0.6)
    G = np.concatenate([pr, pr[:, ng:-ng][:, ::-1]], axis=1)[:, :14 + 2 * ng].copy()
    O.apply_periodic_yz(G, ng)
    O.apply_outflow_right_x(G, ng)
    P = O.params_from_config(phys, cfg)
    d = 1.0 / 8
    return G, P, rk, 0.1 * d, d, ng


@pytest.mark.parametrize("phys", ["srhd", "rmhd"])
def test_oracle_stages_chain_to_the_step(phys):
    G, P, rk, dt, d, ng = stage_case(phys)
    nm = 5 if phys == "srhd" else 9
    Uk = np.zeros((nm,) + G.shape[1:])
    cur = G
    for st in range(rk):
        cur = O.stage(P, G, cur, Uk, d, d, d, dt, rk, st)
    assert np.array_equal(cur, O.step(P, G, d, d, d, dt, rk))


CHILD_STAGES = r"""
import sys
for p in ({root!r}, {oracle!r}, {tests!r}, {golden!r}):
    sys.path.insert(0, p)
import numpy as np, torch, torch.distributed as dist
import oracle as O
import test_slabs_cpu as T
from astrofd_b200.slabs import SlabDomain
dist.init_process_group("gloo", init_method="env://")
rank = dist.get_rank()
G, P, rk, dt, d, ng = T.stage_case({phys!r})
dom = SlabDomain(G.shape[1] - 2 * ng, ng)
lo, hi = dom.offset, dom.offset + dom.nx + 2 * ng
pr = torch.from_numpy(G[:, lo:hi].copy())
Uk = np.zeros(({nm},) + tuple(pr.shape[1:]))

def stage_fn(p0, pk, dst, st):
    dst.copy_(torch.from_numpy(O.stage(P, p0.numpy(), pk.numpy(), Uk, d, d, d, dt, rk, st)))

out = torch.empty_like(pr)
dom.step_stagewise(stage_fn, pr, out, [torch.empty_like(pr), torch.empty_like(pr)], rk)
np.save({out!r} + f"/rank{{rank}}.npy", out.numpy())
dist.destroy_process_group()
"""


@pytest.mark.parametrize("phys,size", [("srhd", 2), ("srhd", 3), ("rmhd", 2)])
def test_stagewise_exchange_reproduces_one_block(phys, size, tmp_path):
    """x-slabs exchanging every RK stage's output give, cell for cell, the
    one-block step of the same block; exchanging once per step (the
    reference driver) does not."""
    G, P, rk, dt, d, ng = stage_case(phys)
    port = _free_port()
    code = CHILD_STAGES.format(root=ROOT, oracle=os.path.join(ROOT, "oracle"),
                               tests=os.path.join(ROOT, "tests"),
                               golden=os.path.join(ROOT, "tests", "golden"), phys=phys,
                               nm=5 if phys == "srhd" else 9, out=str(tmp_path))
    procs = []
    for r in range(size):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(size), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, text=True,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE))
    try:
        for p in procs:
            _, err = p.communicate(timeout=240)
            assert p.returncode == 0, err[-3000:]
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    ref = O.step(P, G, d, d, d, dt, rk)
    nx = G.shape[1] - 2 * ng
    for r in range(size):
        cnt, off = decompose_x(nx, size, r)[:2]
        got = np.load(tmp_path / f"rank{r}.npy")
        assert np.array_equal(got[:, ng:ng + cnt], ref[:, ng + off:ng + off + cnt]), r
    # without the stage exchanges (a step on the first slab alone) the cells
    # next to the slab face differ
    cnt = decompose_x(nx, size, 0)[0]
    alone = O.step(P, G[:, :cnt + 2 * ng].copy(), d, d, d, dt, rk)
    assert not np.array_equal(alone[:, ng:ng + cnt], ref[:, ng:ng + cnt])
