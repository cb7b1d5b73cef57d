"""Seeded synthetic primitive states for parity tests.

Test infrastructure only.  Every array is float64, C-contiguous, laid out as
the reference lays out its primitive block: ``pr[v, i, j, k]`` with shape
``(NV, nx + 2*ng, ny + 2*ng, nz + 2*ng)`` and k fastest
(reference: solvers/srhd3d_mpi_muscl.py:128-160, ``init_block``).

The states are deliberately rough (large noise, a relativistic jet core,
magnetic fields in random directions) so that limiter branches, floors, the
Riemann-solver fan cases and the con2prim fallbacks are all exercised.
"""
import numpy as np


def n_main(physics):
    return 5 if physics == "srhd" else 9


def make_state(seed, n, ng, physics, n_extra=0, vjet=0.99, noise=0.3,
               bamp=0.3, stripes=True, n_is=0):
    """Return a rough jet-like primitive block.

    n        interior cells: an int (a cube) or (nx, ny, nz); a cube draws
             the same random numbers in the same order either way
    ng       ghost layers
    physics  "srhd" (5 primitives) or "rmhd" (9 primitives)
    n_extra  extra passive variables appended after the base primitives
    stripes  leave every third x-plane ambient (strong shocks) when True
    n_is     Israel-Stewart fields (pi, pi^ij, q^i: 10) between the base
             primitives and the passives (SRHD blocks of 15+ variables)
    """
    rng = np.random.default_rng(seed)
    nx, ny, nz = (n, n, n) if np.isscalar(n) else n
    S = (nx + 2 * ng, ny + 2 * ng, nz + 2 * ng)
    nm = n_main(physics)
    nv = nm + n_is + n_extra
    pr = np.zeros((nv,) + S, dtype=np.float64)

    def u(*shape):
        return 2.0 * rng.random(shape) - 1.0

    pr[0] = 1.0 * (1.0 + noise * u(*S))
    pr[1] = 0.3 * u(*S)
    pr[2] = 0.3 * u(*S)
    pr[3] = 0.3 * u(*S)
    pr[4] = 0.01 * (1.0 + 0.5 * u(*S))

    # relativistic jet core along x through the middle of the y/z plane
    cy, cz = 0.5 * (S[1] - 1), 0.5 * (S[2] - 1)
    jj, kk = np.meshgrid(np.arange(S[1]), np.arange(S[2]), indexing="ij")
    r = np.sqrt((jj - cy) ** 2 + (kk - cz) ** 2)
    core = r < 0.3 * min(S[1], S[2])
    for i in range(S[0]):
        if stripes and i % 3 == 2:
            continue  # leave some ambient x-planes for strong jumps
        pr[0, i][core] = 0.1 * (1.0 + 0.1 * rng.random(core.sum()))
        pr[1, i][core] = vjet
        pr[2, i][core] = 0.01 * u(core.sum())
        pr[3, i][core] = 0.01 * u(core.sum())

    # keep |v| < 1
    v2 = pr[1] ** 2 + pr[2] ** 2 + pr[3] ** 2
    fac = np.where(v2 >= 0.998 ** 2, 0.998 / np.sqrt(v2 + 1e-32), 1.0)
    pr[1:4] *= fac

    if physics == "rmhd":
        pr[5] = bamp * u(*S)
        pr[6] = bamp * u(*S)
        pr[7] = bamp * u(*S)
        pr[8] = 0.01 * u(*S)

    for m in range(n_is):
        pr[nm + m] = 0.003 * u(*S)
    for t in range(n_extra):
        pr[nm + n_is + t] = rng.random(S)
    return np.ascontiguousarray(pr)


def make_c2p_batch(seed, count, gamma=4.0 / 3.0):
    """Random RMHD primitive states in the spirit of the learned-c2p sampler:
    rho, p, W log-uniform; isotropic velocity and field directions; field
    strength set from a log-uniform magnetisation sigma = B^2 / (rho h)."""
    rng = np.random.default_rng(seed)
    rho = 10.0 ** rng.uniform(-4.0, 1.0, count)
    p = 10.0 ** rng.uniform(-6.0, 1.0, count)
    W = 10.0 ** rng.uniform(0.0, np.log10(50.0), count)
    v = np.sqrt(1.0 - 1.0 / W ** 2)

    def iso(m):
        x = rng.normal(size=(3, m))
        return x / np.linalg.norm(x, axis=0)

    vd = iso(count)
    bd = iso(count)
    h = 1.0 + gamma / (gamma - 1.0) * p / rho
    sigma = 10.0 ** rng.uniform(-3.0, 1.0, count)
    bmag = np.sqrt(sigma * rho * h)
    pr = np.zeros((9, count))
    pr[0] = rho
    pr[1:4] = v * vd
    pr[4] = p
    pr[5:8] = bmag * bd
    return pr
