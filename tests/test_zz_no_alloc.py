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


def _static(L, p, g, pr, out, stream):
    rc = L.astro_rhs_static(C.byref(p), C.byref(g), C.c_void_p(pr.data_ptr()),
                            C.c_void_p(out.data_ptr()), stream)
    assert rc == 0, L.astro_error_string(rc)


@pytest.mark.parametrize("precision,flux_mode", [
    (_lib.PREC_FP64, _lib.FLUX_REFERENCE), (_lib.PREC_MIXED, _lib.FLUX_CONSERVATIVE)])
def test_static_scratch_large_grid_then_smaller_grids(precision, flux_mode):
    """A grid whose scratch fills most of the array, then smaller ones: each
    call's layout starts at the array's base, so the smaller calls read only
    what they wrote, never the larger call's leftovers."""
    L = _lib.load()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = _params(_lib.RMHD, 2, 1, 0, precision, flux_mode)
    big = 40 if precision == _lib.PREC_FP64 else 52  # ~29 MB of scratch either way
    sizes = (big, 12, 25, big)
    first = None
    for i, n in enumerate(sizes):
        pr = torch.from_numpy(make_state(70 + i, n, 3, "rmhd", noise=0.1, bamp=0.1,
                                         vjet=0.9, stripes=False)).cuda()
        nv, nx, ny, nz = pr.shape
        g = _lib.AstroGrid(nv, nx, ny, nz, 1 / n, 1 / n, 1 / n)
        nb = L.astro_rhs_workspace_bytes(C.byref(p), C.byref(g))
        if first is None:
            first = nb
            # the large call uses most of the array
            assert (24 << 20) < nb <= L.astro_rhs_static_max_bytes()
        ref = torch.zeros((9, nx, ny, nz), dtype=torch.float64, device="cuda")
        got = torch.full_like(ref, float("nan"))
        _with_workspace(L, p, g, pr, ref, stream)
        _static(L, p, g, pr, got, stream)
        torch.cuda.synchronize()
        assert PT.normwise(got.cpu().numpy(), ref.cpu().numpy()) < 1e-10, n


@pytest.mark.parametrize("name", ["r_weno_hlld_ragged", "s_muscl_mc_hllc_ragged"])
def test_static_scratch_rhs_matches_reference_fixture(name):
    """Against the right-hand side the reference itself computed (golden
    fixture), at the float64 parity bar of the other right-hand-side tests."""
    from astrofd_b200.core._engine import Engine
    L = _lib.load()
    d = PT.load(name)
    params = PT.params_of(d)
    phys = _lib.SRHD if name.startswith("s_") else _lib.RMHD
    E = Engine(phys)
    E.configure(dict(dict(RESISTIVE_ENABLED=False, RESISTIVITY=0.0, FLUX_MODE="reference",
                          PRECISION="fp64"), **params))
    pr = torch.from_numpy(d["pr_in"]).cuda()
    nv, nx, ny, nz = pr.shape
    ng = params["NG"]
    g = _lib.AstroGrid(nv, nx, ny, nz, 1 / (nx - 2 * ng), 1 / (ny - 2 * ng), 1 / (nz - 2 * ng))
    got = torch.full(d["rhs"].shape, float("nan"), dtype=torch.float64, device="cuda")
    for _ in range(2):  # twice in a row on the shared scratch
        _static(L, E.p, g, pr, got, None)
        torch.cuda.synchronize()
        assert PT.normwise(got.cpu().numpy(), d["rhs"]) < 1e-11


@pytest.mark.skipif(not torch.cuda.is_available() or torch.cuda.device_count() < 2,
                    reason="needs two GPUs")
def test_static_scratch_on_a_second_device():
    """Each device has its own copy of the array, looked up in its own
    context: a call on device 1 after one on device 0 uses device 1's."""
    L = _lib.load()
    p = _params(_lib.RMHD, 2, 1)
    for dev in (0, 1, 0):
        with torch.cuda.device(dev):
            pr = torch.from_numpy(make_state(80 + dev, 12, 3, "rmhd", noise=0.1, bamp=0.1,
                                             vjet=0.9, stripes=False)).cuda()
            nv, nx, ny, nz = pr.shape
            g = _lib.AstroGrid(nv, nx, ny, nz, 1 / 12, 1 / 12, 1 / 12)
            stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
            ref = torch.zeros((9, nx, ny, nz), dtype=torch.float64, device="cuda")
            got = torch.full_like(ref, float("nan"))
            _with_workspace(L, p, g, pr, ref, stream)
            _static(L, p, g, pr, got, stream)
            torch.cuda.synchronize()
            assert PT.normwise(got.cpu().numpy(), ref.cpu().numpy()) < 1e-10
