"""Ghost fills that the reference lacks, in the oracle, against independent
numpy statements: zero-gradient y/z faces, the nozzle's zero-gradient ambient
part of the x = 0 face and its toroidal B_phi(r) profile on the ambient axial
field (the jet set-up of the magnetised configurations: outflow on every face
but the nozzle, B_phi = b0 r/R inside the jet and b0 R/r outside)."""
import math

import numpy as np

import oracle as O


def _block(nv=11, n=12, ng=3, seed=0):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((nv, n + 2 * ng, n + 2 * ng, n + 2 * ng))


def test_outflow_yz_is_edge_padding_of_the_interior():
    ng = 3
    pr = _block()
    want = pr.copy()
    want[:, :, :, :] = np.pad(pr[:, :, ng:-ng, ng:-ng], ((0, 0), (0, 0), (ng, ng), (ng, ng)),
                              mode="edge")
    O.apply_outflow_yz(pr, ng)
    assert np.array_equal(pr, want)


def _cfg(ng, **kw):
    c = dict(NG=ng, JET_RADIUS=0.25, SHEAR_THICK=0.0, NOZZLE_PROFILE="top_hat", GAMMA_JET=10.0,
             ETA_RHO=0.1, P_EQ=0.01, RHO_AMB=1.0, VX_AMB=0.0, VY_AMB=0.0, VZ_AMB=0.0,
             NOZZLE_PERTURB="none", TURB_VAMP=0.0, TURB_PAMP=0.0, PHYSICS="rmhd",
             B_INIT="toroidal_phi", B0=2.5, B_AMB_X=0.1, NOZZLE_AMBIENT="outflow",
             N_TRACERS=0, TWO_TEMPERATURE=False)
    c.update(kw)
    return c


def test_nozzle_outflow_ambient_and_toroidal_phi():
    n, ng = 12, 3
    d = 1.0 / n
    pr = _block(nv=9, n=n, ng=ng, seed=1)
    before = pr.copy()
    cfg = _cfg(ng)
    O.apply_nozzle_left_x(pr, d, d, d, n, n, 0.5, 0.5, np.random.default_rng(0), cfg)
    beta = math.sqrt(1.0 - 1.0 / cfg["GAMMA_JET"] ** 2)
    jets = 0
    for g in range(ng):
        for j in range(ng, ng + n):
            y = (j - ng + 0.5) * d
            for k in range(ng, ng + n):
                z = (k - ng + 0.5) * d
                r = math.sqrt((y - 0.5) ** 2 + (z - 0.5) ** 2)
                if r > cfg["JET_RADIUS"]:
                    # zero-gradient from the first interior x layer
                    assert np.array_equal(pr[:, g, j, k], before[:, ng, j, k])
                    continue
                jets += 1
                R, b0 = cfg["JET_RADIUS"], cfg["B0"]
                bphi = b0 * r / R
                f = bphi / r if r > 0 else 0.0
                want = [0.1, beta, 0.0, 0.0, 0.01, 0.1, -f * (z - 0.5), f * (y - 0.5), 0.0]
                assert np.allclose(pr[:, g, j, k], want, rtol=1e-15, atol=0), (g, j, k)
                # B is toroidal: |B_perp| = B_phi(r), perpendicular to the radius
                assert math.isclose(math.hypot(pr[6, g, j, k], pr[7, g, j, k]), bphi,
                                    rel_tol=1e-14, abs_tol=1e-15)
                assert abs(pr[6, g, j, k] * (y - 0.5) + pr[7, g, j, k] * (z - 0.5)) < 1e-15
    assert jets > 0
    # x ghosts only; the interior is untouched
    assert np.array_equal(pr[:, ng:], before[:, ng:])


def test_reference_nozzle_unchanged_by_the_new_keys_defaults():
    n, ng = 12, 3
    d = 1.0 / n
    base = _cfg(ng, B_INIT="toroidal")
    del base["NOZZLE_AMBIENT"], base["B_AMB_X"]
    a = _block(nv=9, n=n, ng=ng, seed=2)
    b = a.copy()
    O.apply_nozzle_left_x(a, d, d, d, n, n, 0.5, 0.5, np.random.default_rng(0), base)
    O.apply_nozzle_left_x(b, d, d, d, n, n, 0.5, 0.5, np.random.default_rng(0),
                          dict(base, NOZZLE_AMBIENT="fixed", B_AMB_X=0.7))
    assert np.array_equal(a, b)
    # reference toroidal: By = B0 s, Bx = Bz = 0 on the whole x = 0 face
    assert np.all(a[5, :ng, ng:-ng, ng:-ng] == 0.0) and np.all(a[7, :ng, ng:-ng, ng:-ng] == 0.0)
