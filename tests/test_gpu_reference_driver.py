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
the fields to 1e-10 of each field's scale, the CSV numbers to their printed
precision.

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
    for k in fields:
        a, b = got[k], gold[k]
        assert a.shape == b.shape, k
        scale = max(np.abs(b).max(), 1e-300)
        assert np.abs(a - b).max() / scale < 1e-10, (k, np.abs(a - b).max() / scale)
    for f in ("diagnostics_csv", "centerline_csv", "divb_csv"):
        a, b = DH.csv_numbers(got[f]), DH.csv_numbers(gold[f])
        assert a.shape == b.shape, f
        np.testing.assert_allclose(a, b, rtol=2e-6, atol=1e-300, err_msg=f)
