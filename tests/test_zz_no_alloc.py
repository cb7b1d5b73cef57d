"""astro_rhs_static: the right-hand side for callers that cannot allocate
device memory (an FFI host that owns only the arrays it passes and has no
device allocator to lend scratch from, or a step loop that must not call the
synchronising cudaMalloc).  Its scratch is a fixed 32 MiB array inside the
library's device memory, shared by every call.

The test calls it through the C ABI with ctypes and checks it against
astro_rhs (caller-owned workspace) on two calls in a row with different
inputs, so the second call runs on scratch that still holds the first call's
data.  It lives in its own file, collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import parity as PT
from astrofd_b200 import _lib
from states import make_state

pytestmark = pytest.mark.gpu


def _params(physics, recon, riemann, n_passive=0, precision=_lib.PREC_FP64,
            flux_mode=_lib.FLUX_REFERENCE):
    p = _lib.AstroParams()
    p.physics, p.recon, p.riemann, p.limiter = physics, recon, riemann, 0
    p.n_passive = n_passive
    p.passive_offset = 5 if physics == _lib.SRHD else 9
    p.gamma = 4.0 / 3.0 if physics == _lib.RMHD else 5.0 / 3.0
    p.srhd_gamma = 5.0 / 3.0
    p.p_max, p.v_max, p.glm_ch, p.glm_cp = 2.0, 0.9999, 1.0, 0.1
    p.flux_mode = flux_mode
    p.precision = precision
    return p


def _with_workspace(L, p, g, pr, out, stream):
    nb = L.astro_rhs_workspace_bytes(C.byref(p), C.byref(g))
    assert nb > 0
    w = torch.empty(nb, dtype=torch.uint8, device="cuda")
    rc = L.astro_rhs(C.byref(p), C.byref(g), C.c_void_p(pr.data_ptr()),
                     C.c_void_p(out.data_ptr()), C.c_void_p(w.data_ptr()), nb, stream)
    assert rc == 0, L.astro_error_string(rc)


@pytest.mark.parametrize("physics,recon,riemann,n_passive,precision,flux_mode", [
    # WENO5 + hlld, loop-carried x-face speeds
    (_lib.RMHD, 2, 1, 0, _lib.PREC_FP64, _lib.FLUX_REFERENCE),
    # MUSCL + HLLC with passive scalars
    (_lib.SRHD, 0, 1, 2, _lib.PREC_FP64, _lib.FLUX_REFERENCE),
    # float32 faces: the float32 primitive copy and the counter of faces to
    # redo in float64 also live in the shared scratch
    (_lib.RMHD, 2, 1, 0, _lib.PREC_MIXED, _lib.FLUX_CONSERVATIVE),
])
def test_static_scratch_rhs_matches_workspace_rhs(physics, recon, riemann, n_passive,
                                                  precision, flux_mode):
    L = _lib.load()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = _params(physics, recon, riemann, n_passive, precision, flux_mode)
    assert L.astro_rhs_static_max_bytes() == 32 << 20
    phys = "srhd" if physics == _lib.SRHD else "rmhd"
    nm = 5 if phys == "srhd" else 9
    for seed in (5, 6):  # two calls in a row, different data
        pr = torch.from_numpy(make_state(seed, 16, 3, phys, n_extra=n_passive, noise=0.1,
                                         bamp=0.1, vjet=0.9, stripes=False)).cuda()
        nv, nx, ny, nz = pr.shape
        g = _lib.AstroGrid(nv, nx, ny, nz, 1 / 16, 1 / 16, 1 / 16)
        assert L.astro_rhs_workspace_bytes(C.byref(p), C.byref(g)) <= (32 << 20)
        ref = torch.zeros((nm + n_passive, nx, ny, nz), dtype=torch.float64, device="cuda")
        got = torch.full_like(ref, float("nan"))
        _with_workspace(L, p, g, pr, ref, stream)
        rc = L.astro_rhs_static(C.byref(p), C.byref(g), C.c_void_p(pr.data_ptr()),
                                C.c_void_p(got.data_ptr()), stream)
        assert rc == 0, L.astro_error_string(rc)
        torch.cuda.synchronize()
        a, b = got.cpu().numpy(), ref.cpu().numpy()
        assert np.all(np.isfinite(a[:nm]))
        assert PT.normwise(a, b) < 1e-10


def test_static_scratch_rejects_grids_beyond_its_size():
    L = _lib.load()
    p = _params(_lib.RMHD, 2, 1)
    g = _lib.AstroGrid(9, 134, 134, 134, 1 / 128, 1 / 128, 1 / 128)
    assert L.astro_rhs_workspace_bytes(C.byref(p), C.byref(g)) > (32 << 20)
    pr = torch.zeros((9, 8, 8, 8), dtype=torch.float64, device="cuda")  # never read
    rc = L.astro_rhs_static(C.byref(p), C.byref(g), C.c_void_p(pr.data_ptr()),
                            C.c_void_p(pr.data_ptr()), None)
    assert rc == -3
    assert L.astro_error_string(rc) == b"workspace missing or too small"
