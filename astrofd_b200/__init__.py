"""astrofd_b200: B200 (sm_100a) implementation of AstroFD's per-step
finite-volume right-hand side behind the reference's Python call surface.

    from astrofd_b200.core import srhd_core, rmhd_core, boundary, nozzle

The compute lives in libastrofd_b200.so (CUDA, C ABI in include/astrofd.h);
there is no CPU fallback.
"""
__version__ = "1.0.0"
