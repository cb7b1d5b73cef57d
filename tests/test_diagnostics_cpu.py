"""Run diagnostics (utils/diagnostics.py): the oracle against fixtures made by
the reference's own code (tests/golden/make_golden.py, one rank), and the
host side of astrofd_b200.utils.diagnostics -- CSV rows, rank 0 inlet, the
reductions and gathers over ranks -- with the device reductions replaced by
the oracle (the device kernel itself is checked in test_gpu_diagnostics.py).

Tolerances: max Gamma and div B bit-exact (same operations, numpy's
reductions in the reference's order); the inlet flux to 1e-13 relative (the
C prim_to_cons of the oracle may round differently from Numba's); CSV text
exact.
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
from astrofd_b200.utils import diagnostics as D

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
G = np.load(os.path.join(ROOT, "tests", "golden", "diagnostics.npz"))
NG, DX = int(G["ng"]), float(G["d"])
DY, DZ = 0.7 * DX, 1.3 * DX
VMAX = json.loads(str(G["cfg"]))["V_MAX"]


@pytest.mark.parametrize("phys", ["srhd", "rmhd"])
def test_oracle_matches_reference_fixture(phys):
    pr = G[phys + "_pr"]
    r = O.diagnostics(pr, DX, DY, DZ, NG, phys == "rmhd", v_max=VMAX)
    maxg, flux, aflux = G[phys + "_diag"]
    assert r["max_gamma"] == maxg
    assert r["max_gamma"] > 1e6  # a cell at v >= 1 was capped
    assert abs(r["inlet_flux"] - flux) <= 1e-13 * abs(flux)
    if phys == "rmhd":
        assert [r["divb_max"], r["divb_rms"], r["divb_mean"]] == list(G["rmhd_divb"])
    else:
        assert "divb_max" not in r and np.isnan(G["srhd_divb"]).all()
    Gm, rho, p, vx = O.centerline(pr, NG, VMAX)
    rows = str(G[phys + "_centerline_csv"]).splitlines()[1:]
    assert len(rows) == Gm.size
    for ii, row in enumerate(rows):
        got = [float(x) for x in row.split(",")[4:]]
        ref = [Gm[ii], rho[ii], p[ii], vx[ii]]
        np.testing.assert_allclose(got, ref, rtol=6e-9)


def _fake_reductions(pr, dx, dy, dz, NG, is_rmhd, gamma=D.INLET_GAMMA):
    r = O.diagnostics(np.asarray(pr), dx, dy, dz, NG, is_rmhd, v_max=VMAX)
    return dict(max_gamma=r["max_gamma"], inlet_sx=r["inlet_sx"],
                divb_max=r.get("divb_max", 0.0), divb_sum=r.get("divb_sum", 0.0),
                divb_sumsq=r.get("divb_sumsq", 0.0), divb_n=r.get("divb_n", 0))


def _fake_centerline(pr, V_MAX, NG):
    return O.centerline(np.asarray(pr), NG, V_MAX)


@pytest.fixture
def host_only(monkeypatch):
    monkeypatch.setattr(D, "device_reductions", _fake_reductions)
    monkeypatch.setattr(D, "centerline", _fake_centerline)


def _run_all(pr, run, comm=None, rank=0, rmhd=True):
    res = D.compute_diagnostics_and_write(pr, DX, DY, DZ, 0, None, comm, rank, 7, 0.25, 1e-3, 0.9,
                                          str(run), None, NG, rmhd)
    D.compute_centerline_and_write(pr, DX, DY, DZ, 0, None, comm, rank, 7, 0.25, str(run), VMAX,
                                   NG)
    dv = D.compute_divb_and_write(pr, DX, DY, DZ, 0, None, comm, rank, 7, 0.25, str(run), NG)
    return res, dv


def _read(run, name):
    p = os.path.join(str(run), name + ".csv")
    return open(p).read() if os.path.exists(p) else ""


@pytest.mark.parametrize("phys", ["srhd", "rmhd"])
def test_host_side_writes_the_reference_csv(phys, tmp_path, host_only):
    res, dv = _run_all(G[phys + "_pr"], tmp_path, rmhd=phys == "rmhd")
    np.testing.assert_allclose(res, G[phys + "_diag"], rtol=1e-13)
    for f in ("diagnostics", "centerline", "divb"):
        assert _read(tmp_path, f) == str(G[phys + "_" + f + "_csv"]), f
    if phys == "srhd":
        assert dv == (None, None, None)
    # appending: one more row, no second header
    _run_all(G[phys + "_pr"], tmp_path, rmhd=phys == "rmhd")
    txt = _read(tmp_path, "diagnostics").splitlines()
    assert len(txt) == 3 and txt[1] == txt[2] and txt[0].startswith("step,")


def test_empty_interior(tmp_path, host_only):
    pr = np.zeros((9, 2 * NG, 8, 8))
    res, dv = _run_all(pr, tmp_path)
    assert res == (0.0, 0.0, 0.0) and dv == (0.0, 0.0, 0.0)


CHILD = r"""
import json, os, sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {oracle!r}); sys.path.insert(0, {tests!r})
import numpy as np
import torch.distributed as dist
import test_diagnostics_cpu as T
from astrofd_b200.utils import diagnostics as D
D.device_reductions, D.centerline = T._fake_reductions, T._fake_centerline
dist.init_process_group("gloo", init_method="env://")
rank = dist.get_rank()
pr = T.G["rmhd_pr"]
n, ng = pr.shape[1] - 2 * T.NG, T.NG
lo, hi = (0, n // 2) if rank == 0 else (n // 2, n)
slab = np.ascontiguousarray(pr[:, lo:hi + 2 * ng])   # interior x [lo, hi) with its ghost layers
run = {run!r}
res, dv = T._run_all(slab, run, D.TorchComm(), rank)
print(json.dumps(dict(rank=rank, res=res, dv=dv)))
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_x_slabs_over_gloo_equal_one_block(tmp_path):
    """World size 2: each rank holds half of the x interior (with ghost
    layers from its neighbour), as the reference's x-slab decomposition; max
    Gamma, inlet flux (rank 0 only), div B and the gathered centreline equal
    the one-block values."""
    port = _free_port()
    run1 = tmp_path / "ranks"
    run1.mkdir()
    code = CHILD.format(root=ROOT, oracle=os.path.join(ROOT, "oracle"),
                        tests=os.path.join(ROOT, "tests"), run=str(run1))
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, text=True,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE))
    outs = []
    try:
        for p in procs:
            out, err = p.communicate(timeout=180)
            assert p.returncode == 0, err[-3000:]
            outs.append(json.loads(out.strip().splitlines()[-1]))
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    r0 = [o for o in outs if o["rank"] == 0][0]
    maxg, flux, _ = G["rmhd_diag"]
    assert r0["res"][0] == maxg
    assert abs(r0["res"][1] - flux) <= 1e-13 * abs(flux)
    np.testing.assert_allclose(r0["dv"], G["rmhd_divb"], rtol=1e-12)
    assert _read(run1, "centerline") == str(G["rmhd_centerline_csv"])
    assert len(_read(run1, "diagnostics").splitlines()) == 2
    assert [o["res"] for o in outs][0] == [o["res"] for o in outs][1]


def test_mpi4py_communicator_gets_mpi_ops(monkeypatch):
    """The reference's driver passes MPI.COMM_WORLD (utils/diagnostics.py:28,44
    reduce with MPI.MAX / MPI.SUM): an mpi4py communicator receives mpi4py's
    op objects, other communicators this module's MAX / SUM."""
    import types
    mpi = types.ModuleType("mpi4py.MPI")
    mpi.MAX, mpi.SUM = object(), object()
    seen = []

    class Comm:
        def allreduce(self, value, op=None):
            seen.append(op)
            return value

    Comm.__module__ = "mpi4py.MPI"
    pkg = types.ModuleType("mpi4py")
    pkg.MPI = mpi
    monkeypatch.setitem(sys.modules, "mpi4py", pkg)
    monkeypatch.setitem(sys.modules, "mpi4py.MPI", mpi)
    assert D._allreduce(Comm(), 2.0, D.MAX) == 2.0
    assert D._allreduce(Comm(), 3.0, D.SUM) == 3.0
    assert seen[0] is mpi.MAX and seen[1] is mpi.SUM

    class Other:
        def allreduce(self, value, op=None):
            seen.append(op)
            return value

    D._allreduce(Other(), 1.0, D.MAX)
    assert seen[-1] == D.MAX
