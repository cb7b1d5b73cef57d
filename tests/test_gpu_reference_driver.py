"""The reference's driver script, unchanged, on the drop-in modules.

solvers/srhd3d_mpi_muscl.py of an AstroFD checkout runs with
astrofd_b200.core.* registered as its ``core.*`` modules and
astrofd_b200.utils.diagnostics as ``utils.diagnostics`` (its own
utils/settings.py and utils/io_utils.py load its config files), on the smoke
configurations of the reference's runner (tools/run_smoke_suite.py: SRHD
MUSCL with HLLC, minmod, van Leer, two-temperature, ion chemistry, causal
dissipation; RMHD with resistivity; GRMHD Kerr-Schild), for the steps up to
t = 0.12.  Its snapshot of the last step and its diagnostics / centreline /
div B CSV files must match those the same driver wrote on the reference's own
Numba core (tests/golden/driver_*.npz, made by tests/golden/make_golden.py):
the fields to 1e-10 of each field's scale (5e-8 for the magnetised runs,
whose con2prim stops at its tolerance), the CSV numbers to their printed
precision of each column's scale.

The reference checkout is read at run time, so the test runs only where one
is given: ASTROFD_REFERENCE=<path to the checkout>.  The one-rank mpi4py and
the json5 the driver imports are stand-ins (tests/driver_harness.py).
"""
import os

import numpy as np
import pytest

import driver_harness as DH
import parity as PT

pytestmark = pytest.mark.gpu

REF = os.environ.get("ASTROFD_REFERENCE", "")
needs_ref = pytest.mark.skipif(
    not os.path.isfile(os.path.join(REF, "solvers", "srhd3d_mpi_muscl.py")),
    reason="set ASTROFD_REFERENCE to an AstroFD checkout to run its driver")


@needs_ref
@pytest.mark.parametrize("config", DH.CONFIGS)
def test_reference_driver_runs_unchanged_on_the_dropin(config, tmp_path):
    gold = PT.load("driver_" + config)
    got = DH.run_driver(REF, config, str(tmp_path), dropin=True)
    assert int(got["steps"]) == int(gold["steps"])
    fields = [k for k in gold.files if k.startswith("snap_") and gold[k].dtype.kind == "f"]
    assert "snap_rho" in fields
    # SRHD to 1e-10; the magnetised runs to 5e-8: their con2prim stops at
    # |f| < 1e-10 max(1, tau) after iteration counts that Numba's fastmath
    # shifts (the same bar as the device's single steps against the
    # reference's fixtures, over three steps)
    bar = 5e-8 if "snap_Bx" in fields else 1e-10
    for k in fields:
        a, b = got[k], gold[k]
        assert a.shape == b.shape, k
        scale = max(np.abs(b).max(), 1e-300)
        assert np.abs(a - b).max() / scale < bar, (k, np.abs(a - b).max() / scale)
    for f in ("diagnostics_csv", "centerline_csv", "divb_csv"):
        a, b = DH.csv_numbers(got[f]), DH.csv_numbers(gold[f])
        assert a.shape == b.shape, f
        if b.size:
            # to the printed precision (7-9 significant digits) of each
            # column's scale: entries that are zero up to round-off (a
            # transverse velocity of 1e-18) carry no digits of their own
            scale = np.abs(b).max(axis=0)
            assert (np.abs(a - b) <= 2e-6 * scale + 1e-300).all(), (f, np.abs(a - b).max(0))
