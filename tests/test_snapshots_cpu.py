"""NPZ snapshots and checkpoints in the reference driver's format
(solvers/srhd3d_mpi_muscl.py:332-389 snapshot keys, :420-428 checkpoint,
:192-200 load_checkpoint), numpy blocks on the CPU; the device writer is
checked in test_gpu_snapshots.py."""
import numpy as np
import pytest

from astrofd_b200.utils import snapshots as S


def _block(nv, n=6, seed=0):
    return np.random.default_rng(seed).random((nv, n, n + 1, n + 2))


CASES = {
    # settings, number of variables, the driver's key list
    "hydro": (dict(PHYSICS="hydro"), 5, ["rho", "vx", "vy", "vz", "p"]),
    "hydro_is_tracers": (dict(PHYSICS="hydro", N_TRACERS=2, TRACER_OFFSET=15,
                              TRACER_NAMES=["jet", "amb"]), 17,
                         ["rho", "vx", "vy", "vz", "p", "pi", "pixx", "piyy", "pizz", "pixy",
                          "pixz", "piyz", "qx", "qy", "qz", "jet", "amb", "tracer_names"]),
    "rmhd_c5": (dict(PHYSICS="rmhd", N_THERMO=2, TRACER_OFFSET=9, THERMO_OFFSET=9), 11,
                ["rho", "vx", "vy", "vz", "p", "Bx", "By", "Bz", "psi", "Te", "Ti"]),
    "grmhd_all": (dict(PHYSICS="grmhd", N_TRACERS=1, TRACER_OFFSET=9, N_THERMO=2,
                       THERMO_OFFSET=10, N_CHEM=3, CHEM_OFFSET=12), 15,
                  ["rho", "vx", "vy", "vz", "p", "Bx", "By", "Bz", "psi", "tracer0",
                   "tracer_names", "Te", "Ti", "xHII", "xHeII", "xHeIII"]),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_snapshot_keys_and_fields(case, tmp_path):
    settings, nv, keys = CASES[case]
    pr = _block(nv)
    path = S.write_snapshot(pr, str(tmp_path), 3, 120, 0.1, 0.2, 0.3, 1.25, settings)
    assert path.endswith("jet3d_rank0003_step000120.npz")
    z = np.load(path, allow_pickle=True)
    assert z.files == keys + ["meta", "comment"]
    hydro = settings["PHYSICS"] in ("hydro", "grhd")
    assert str(z["comment"]) == ("3D SRHD/GRHD block (with ghosts)." if hydro
                                 else "3D RMHD/GRMHD block (with ghosts).")
    np.testing.assert_array_equal(z["meta"], [0.1, 0.2, 0.3, 1.25])
    offsets = {k: i for i, k in enumerate(k for k in keys if k != "tracer_names")}
    for k, v in offsets.items():
        assert np.array_equal(z[k], pr[v]), k
    if "tracer_names" in keys:
        assert list(z["tracer_names"]) == list(settings.get("TRACER_NAMES", []))


def test_checkpoint_round_trip(tmp_path):
    pr = _block(9, seed=4)
    path = S.write_checkpoint(pr, str(tmp_path), 0, 7, 0.1, 0.1, 0.1, 0.5)
    assert path.endswith("checkpoint_rank0000_step000007.npz")
    z = np.load(path)
    assert z.files == ["prim", "meta", "comment"]
    np.testing.assert_array_equal(z["meta"], [0.1, 0.1, 0.1, 0.5, 7])
    got, t, step = S.load_checkpoint(path)
    assert np.array_equal(got, pr) and (t, step) == (0.5, 7)


def test_load_checkpoint_without_meta(tmp_path):
    p = tmp_path / "c.npz"
    np.savez(p, prim=np.ones((5, 2, 2, 2)), meta=np.array([0.1, 0.1, 0.1, 2.0]))
    got, t, step = S.load_checkpoint(str(p))
    assert (t, step) == (0.0, 0) and got.shape == (5, 2, 2, 2)
