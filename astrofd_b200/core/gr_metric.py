"""Drop-in replacement of AstroFD's core/gr_metric.py: the scalar lapse
helpers of the fixed black-hole metrics (mass M at the origin).

The device evaluates the same formulas inside the GR right-hand sides
(astro_rhs_gr / astro_step_gr); these host functions keep the reference's
module surface for callers that use them directly.
"""
import math


def schwarzschild_iso_lapse_and_grad(x, y, z, M):
    """(alpha, d ln alpha / dx, dy, dz) of the isotropic Schwarzschild lapse
    alpha = (1 - a) / (1 + a), a = M / 2r (core/gr_metric.py:6)."""
    r = math.sqrt(x * x + y * y + z * z) + 1e-12
    a = M / (2.0 * r)
    alpha = (1.0 - a) / (1.0 + a)
    denom = 1.0 - a * a
    dlnadr = 0.0 if denom == 0.0 else (2.0 * a) / (r * denom)
    return alpha, dlnadr * (x / r), dlnadr * (y / r), dlnadr * (z / r)


def schwarzschild_ks_lapse_shift_and_grad(x, y, z, M):
    """(alpha, beta_x, beta_y, beta_z, d ln alpha / dx, dy, dz) of the
    Kerr-Schild form without spin: alpha = 1 / sqrt(1 + 2H), H = M / r,
    beta = 2H / (1 + 2H) r_hat (core/gr_metric.py:18)."""
    r = math.sqrt(x * x + y * y + z * z) + 1e-12
    H = M / r
    alpha = 1.0 / math.sqrt(1.0 + 2.0 * H)
    fac = 2.0 * H / (1.0 + 2.0 * H)
    lx, ly, lz = x / r, y / r, z / r
    dlnadr = H / (r * (1.0 + 2.0 * H))
    return alpha, fac * lx, fac * ly, fac * lz, dlnadr * lx, dlnadr * ly, dlnadr * lz


def kerr_schild_lapse_shift_and_grad(x, y, z, M, a):
    """The spin is ignored, as in the reference (core/gr_metric.py:36)."""
    return schwarzschild_ks_lapse_shift_and_grad(x, y, z, M)
