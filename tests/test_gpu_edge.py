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


# Blocks too small for a scheme's cell range: the reference's loops update
# nothing there (rhs = 0) and a step is the p2c -> c2p round trip of every
# cell; ranges of one layer in some directions and none in others.
TINY = [("srhd", "muscl", "minmod", "hlle", 2, (1, 1, 1)),
        ("srhd", "weno", "mc", "hllc", 3, (1, 2, 1)),
        ("srhd", "ppm", "mc", "hlle", 3, (2, 1, 1)),
        ("rmhd", "muscl", "mc", "hlld", 2, (2, 1, 3)),
        ("rmhd", "ppm", "mc", "hlle", 3, (1, 1, 2)),
        ("rmhd", "weno", "mc", "hlld", 3, (3, 1, 1))]


@pytest.mark.parametrize("physics,recon,lim,riemann,ng,n", TINY,
                         ids=[f"{t[0]}_{t[1]}_{'x'.join(map(str, t[5]))}" for t in TINY])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tiny_blocks_vs_oracle(physics, recon, lim, riemann, ng, n, precision):
    import oracle as O
    import parity as PT
    from states import make_state
    from astrofd_b200.core import rmhd_core, srhd_core
    m = srhd_core if physics == "srhd" else rmhd_core
    base = dict(GAMMA=5.0 / 3.0 if physics == "srhd" else 4.0 / 3.0, P_MAX=2.0, V_MAX=0.9999,
                GLM_CH=1.0, GLM_CP=0.1)
    cfg = dict(base, RECON=recon, LIMITER=lim, RIEMANN=riemann, N_PASSIVE=0, NG=ng,
               PASSIVE_OFFSET=5 if physics == "srhd" else 9, RESISTIVE_ENABLED=False,
               RESISTIVITY=0.0, FLUX_MODE="reference", PRECISION=precision)
    pr = make_state(31, n, ng, physics, noise=0.1, bamp=0.1, vjet=0.9, stripes=False)
    dd = tuple(1.0 / k for k in n)
    P = O.params_from_config(physics, cfg)
    m.configure(cfg)
    rhs_fn = {"muscl": m.compute_rhs_muscl if physics == "srhd" else m.compute_rhs_rmhd,
              "ppm": m.compute_rhs_ppm, "weno": m.compute_rhs_weno}[recon]
    t = torch.from_numpy(pr).to("cuda")
    r = rhs_fn(t, *pr.shape[1:], *dd).cpu().numpy()
    ref = O.rhs(P, pr, *dd)
    untouched = np.abs(ref).sum(axis=0) == 0.0  # cells outside the scheme's range
    assert untouched.any() and np.all(r[:, untouched] == 0.0)
    assert PT.normwise(r, ref) < (1e-10 if precision == "fp64" else 5e-3)
    dt = 0.2 * min(dd)
    out = m.step_ssprk3(t, *dd, dt).cpu().numpy()
    assert PT.normwise(out, O.step(P, pr, *dd, dt, 3)) < (1e-7 if precision == "fp64" else 5e-3)
