"""Empty inputs through the drop-in: the reference's array loops return empty
arrays for empty batches, and so do the device paths."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("physics", ["srhd", "rmhd"])
def test_empty_conversion_batches(physics):
    from astrofd_b200.core import rmhd_core, srhd_core
    m = srhd_core if physics == "srhd" else rmhd_core
    m.configure({})
    nm = 5 if physics == "srhd" else 9
    for a in (np.zeros((nm, 0)), torch.zeros((nm, 0), dtype=torch.float64, device="cuda")):
        for fn in (m.engine().p2c_array, m.engine().c2p_array):
            out = fn(a)
            assert tuple(out.shape) == (nm, 0)
            assert isinstance(out, type(a))


def test_empty_learned_batch_and_forward():
    from astrofd_b200 import learned_c2p as LC
    from astrofd_b200.core import rmhd_core
    rmhd_core.configure({})
    params = torch.from_numpy(LC.init_params(0)).cuda()
    U = torch.zeros((9, 0), dtype=torch.float64, device="cuda")
    for listed in (True, False):
        q, st = LC.c2p_learned(rmhd_core.engine(), U, params, listed=listed)
        assert tuple(q.shape) == (9, 0)
        assert st["cells"] == 0 and st["status"] == 0
    net = LC.Trainer(LC.init_params(0))
    Y = net.forward(torch.zeros((0, 5), dtype=torch.float32, device="cuda"))
    assert tuple(Y.shape) == (0, 2)
