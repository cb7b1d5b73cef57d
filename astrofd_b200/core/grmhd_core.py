"""Drop-in replacement of AstroFD's core/grmhd_core.py: the rmhd_core right-hand side
and SSPRK steps with the reference's approximate fixed-metric terms, on the
device (astro_rhs_gr / astro_step_gr).

Same module globals and configure() keys as the reference (GR_METRIC,
GR_MASS, GR_SPIN, ORTHONORMAL_FLUX; core/grmhd_core.py:8-18); the scheme itself
(reconstruction, Riemann solver, gamma, caps, passives) is the one
configured in rmhd_core.  For "schwarzschild" and "kerr-schild" with
ORTHONORMAL_FLUX the fluxes see the interior velocities divided by the
Kerr-Schild lapse; every metric but "minkowski" adds the lapse-gradient
sources on the interior cells (the isotropic Schwarzschild lapse for
"schwarzschild", Kerr-Schild for any other name, as the reference's branches
do).  offs_x is the global x index of the block's first interior cell, ng
its ghost layers.
"""
from .. import _lib
from . import rmhd_core

GR_METRIC = "minkowski"
GR_MASS = 1.0
ORTHONORMAL_FLUX = True
GR_SPIN = 0.0

_METRICS = {"minkowski": _lib.GR_MINKOWSKI, "schwarzschild": _lib.GR_SCHWARZSCHILD,
            "kerr-schild": _lib.GR_KERR_SCHILD}


def configure(params):
    global GR_METRIC, GR_MASS, ORTHONORMAL_FLUX, GR_SPIN
    GR_METRIC = str(params.get("GR_METRIC", "minkowski")).lower()
    GR_MASS = float(params.get("GR_MASS", GR_MASS))
    GR_SPIN = float(params.get("GR_SPIN", GR_SPIN))
    ORTHONORMAL_FLUX = bool(params.get("ORTHONORMAL_FLUX", ORTHONORMAL_FLUX))


def _gr(offs_x, ng):
    g = _lib.AstroGR()
    g.metric = _METRICS.get(GR_METRIC, _lib.GR_OTHER)
    g.orthonormal_flux = 1 if ORTHONORMAL_FLUX else 0
    g.ng, g.offs_x = int(ng), int(offs_x)
    g.mass, g.spin = float(GR_MASS), float(GR_SPIN)
    return g


def compute_rhs_grmhd(pr, dx, dy, dz, offs_x, ng):
    return rmhd_core.engine().rhs_gr(_gr(offs_x, ng), pr, dx, dy, dz)


def step_ssprk2(pr, dx, dy, dz, dt, offs_x, ng, out=None):
    return rmhd_core.engine().step_gr(_gr(offs_x, ng), pr, dx, dy, dz, dt, 2, out)


def step_ssprk3(pr, dx, dy, dz, dt, offs_x, ng, out=None):
    return rmhd_core.engine().step_gr(_gr(offs_x, ng), pr, dx, dy, dz, dt, 3, out)
