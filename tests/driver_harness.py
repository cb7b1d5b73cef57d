"""Test harness: run the reference's own driver script, unchanged, from a
checkout of AstroFD (solvers/srhd3d_mpi_muscl.py with its utils/settings.py and
utils/io_utils.py), either on the reference's core modules or on this
package's drop-ins (astrofd_b200.core.* registered as ``core.*`` and
astrofd_b200.utils.diagnostics as ``utils.diagnostics``).

The driver imports mpi4py and its settings loader imports json5; neither is
installed here, so the harness registers two stand-ins: a one-rank mpi4py
(COMM_WORLD of size 1: allreduce returns its value, Barrier does nothing; a
single rank has no halo neighbours, so Sendrecv is never called) and a json5
that parses the configs' plain JSON with the standard json module.

Test infrastructure only: used by tests/golden/make_golden.py (the reference's
core, to record the golden outputs) and by the GPU test of the drop-in.
"""
import contextlib
import glob
import importlib
import json
import os
import runpy
import sys
import types

import numpy as np

CORE_MODULES = ("srhd_core", "rmhd_core", "grhd_core", "grmhd_core", "dissipation",
                "source_terms", "chemistry", "boundary", "nozzle")
# the smoke configurations the reference's own runner uses
# (tools/run_smoke_suite.py), run for a few steps
CONFIGS = ("config_hllc_small", "config_minmod", "config_vanleer", "config_two_temp",
           "config_chemistry", "config_dissipation", "config_resist", "config_grmhd")
T_END = "0.12"


def _mpi_stub():
    mpi = types.ModuleType("mpi4py.MPI")

    class Op:
        def __init__(self, name):
            self.name = name

        def __repr__(self):
            return "MPI." + self.name

    mpi.MAX, mpi.MIN, mpi.SUM = Op("MAX"), Op("MIN"), Op("SUM")

    class Comm:
        def Get_rank(self):
            return 0

        def Get_size(self):
            return 1

        def allreduce(self, value, op=None):
            return value

        def Barrier(self):
            pass

        def gather(self, obj, root=0):
            return [obj]

        def Gatherv(self, sendbuf, recvbuf, root=0):
            # one rank: its piece is the whole receive buffer
            recvbuf[0][...] = sendbuf

        def bcast(self, obj, root=0):
            return obj

        def Sendrecv(self, *args, **kw):
            raise RuntimeError("one rank has no halo neighbours")

    Comm.__module__ = "mpi4py.MPI"
    mpi.Comm = Comm
    mpi.COMM_WORLD = Comm()
    pkg = types.ModuleType("mpi4py")
    pkg.MPI = mpi
    return pkg, mpi


@contextlib.contextmanager
def _isolated():
    modules, path, argv, cwd = dict(sys.modules), list(sys.path), list(sys.argv), os.getcwd()
    try:
        yield
    finally:
        sys.modules.clear()
        sys.modules.update(modules)
        sys.path[:] = path
        sys.argv[:] = argv
        os.chdir(cwd)


def run_driver(ref_root, config, workdir, dropin, t_end=T_END):
    """Run solvers/srhd3d_mpi_muscl.py --config config/<config>.json --t-end
    t_end in workdir; returns the outputs of its last step: the snapshot's
    arrays and the diagnostics CSV texts."""
    with _isolated():
        pkg, mpi = _mpi_stub()
        sys.modules["mpi4py"], sys.modules["mpi4py.MPI"] = pkg, mpi
        j5 = types.ModuleType("json5")
        j5.load, j5.loads = json.load, json.loads
        sys.modules["json5"] = j5
        for name in [m for m in sys.modules if m.split(".")[0] in ("core", "utils")]:
            del sys.modules[name]
        if dropin:
            core = importlib.import_module("astrofd_b200.core")
            sys.modules["core"] = core
            for name in CORE_MODULES:
                mod = importlib.import_module("astrofd_b200.core." + name)
                sys.modules["core." + name] = mod
                setattr(core, name, mod)
            from astrofd_b200.utils import diagnostics
            utils = types.ModuleType("utils")
            utils.__path__ = [os.path.join(ref_root, "utils")]
            utils.diagnostics = diagnostics
            sys.modules["utils"] = utils
            sys.modules["utils.diagnostics"] = diagnostics
        driver = os.path.join(ref_root, "solvers", "srhd3d_mpi_muscl.py")
        cfg = os.path.join(ref_root, "config", config + ".json")
        sys.argv = [driver, "--config", cfg, "--t-end", t_end, "--out-every", "1"]
        os.chdir(workdir)
        runpy.run_path(driver, run_name="__main__")
        snaps = sorted(glob.glob(os.path.join(workdir, "results", "*", "jet3d_rank0000_step*.npz")))
        out = {}
        with np.load(snaps[-1], allow_pickle=True) as d:
            for k in d.files:
                if d[k].dtype != object:
                    out["snap_" + k] = np.array(d[k])
        out["steps"] = np.array(len(snaps))
        for f in ("diagnostics.csv", "centerline.csv", "divb.csv"):
            hits = glob.glob(os.path.join(workdir, "results", "*", f))
            out[f.split(".")[0] + "_csv"] = np.array(open(hits[0]).read() if hits else "")
        return out


def csv_numbers(text):
    """The numeric fields of a CSV text (header skipped), row by row."""
    rows = [r for r in str(text).strip().splitlines()[1:] if r]
    return np.array([[float(x) for x in r.split(",")] for r in rows]) if rows else np.zeros((0, 0))
