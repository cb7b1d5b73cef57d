"""SnapshotWriter on CUDA blocks: the files hold the block as it was when
the snapshot was requested, although the caller's stream overwrites it right
after (the staging copy is ordered on that stream; the host copy and the
file write run behind it), and equal the synchronous numpy writer's files."""
import numpy as np
import pytest
import torch

from astrofd_b200.utils import snapshots as S

pytestmark = pytest.mark.gpu


def test_async_snapshot_and_checkpoint_hold_the_requested_state(tmp_path):
    settings = dict(PHYSICS="rmhd", N_THERMO=2, TRACER_OFFSET=9, THERMO_OFFSET=9)
    g = torch.Generator(device="cuda").manual_seed(5)
    pr = torch.rand((11, 70, 64, 64), dtype=torch.float64, device="cuda", generator=g)
    want = pr.cpu().numpy()
    w = S.SnapshotWriter()
    (tmp_path / "a").mkdir()
    (tmp_path / "b").mkdir()
    p1 = w.snapshot(pr, str(tmp_path / "a"), 0, 5, 0.1, 0.1, 0.1, 0.75, settings)
    pr.mul_(-1.0)                        # the next 'step' overwrites the block
    p2 = w.checkpoint(pr, str(tmp_path / "a"), 0, 5, 0.1, 0.1, 0.1, 0.75)
    pr.add_(3.0)
    w.wait()
    ref = S.write_snapshot(want, str(tmp_path / "b"), 0, 5, 0.1, 0.1, 0.1, 0.75, settings)
    a, b = np.load(p1), np.load(ref)
    assert a.files == b.files
    for k in a.files:
        assert np.array_equal(a[k], b[k]), k
    got, t, step = S.load_checkpoint(p2, device="cuda")
    assert got.is_cuda and (t, step) == (0.75, 5)
    assert torch.equal(got, torch.from_numpy(-want).cuda())
