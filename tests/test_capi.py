"""CPU-side checks of the C ABI: the library loads and exports every entry
point include/astrofd.h declares, and host-side validation works without a
GPU (no compute calls here)."""
import ctypes as C
import os
import re

import pytest

from astrofd_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "astrofd.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(astro_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from astrofd_b200 import build
    if not os.path.exists(_lib.LIB_PATH):
        build.build()
    return _lib.load()


def test_every_declared_symbol_is_exported(lib):
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.PROTOS, f"{n} has no ctypes prototype"


def test_struct_sizes_match_header_layout():
    # 11 int32 fields (padded to 12 before the pointer), the pointer, 7 doubles
    assert C.sizeof(_lib.AstroParams) == 12 * 4 + 8 + 7 * 8
    assert C.sizeof(_lib.AstroGrid) == 4 * 4 + 3 * 8
    assert C.sizeof(_lib.AstroC2PStats) == 8 * 8
    assert C.sizeof(_lib.AstroNozzle) == 10 * 4 + 18 * 8 + 16 * 8 + 8 + 2 * 4 + 3 * 8
    assert C.sizeof(_lib.AstroChemistry) == 2 * 4 + 7 * 8
    assert C.sizeof(_lib.AstroDissipation) == 2 * 4 + 8 * 8
    assert C.sizeof(_lib.AstroGR) == 4 * 4 + 2 * 8


def test_error_strings_and_validation(lib):
    assert lib.astro_version() >= 10000
    assert lib.astro_error_string(-3) == b"workspace missing or too small"
    p = _lib.AstroParams()
    p.physics, p.recon, p.riemann = 1, 2, 2
    p.gamma = p.srhd_gamma = 4.0 / 3.0
    g = _lib.AstroGrid(9, 22, 22, 22, 0.1, 0.1, 0.1)
    nb = lib.astro_step_workspace_bytes(C.byref(p), C.byref(g))
    assert nb > 9 * 22 ** 3 * 8 * 3
    # invalid enum -> 0 bytes and an error code, no device work
    p.riemann = 7
    assert lib.astro_step_workspace_bytes(C.byref(p), C.byref(g)) == 0
    assert lib.astro_rhs(C.byref(p), C.byref(g), None, None, None, 0, None) == -1
    # SRHD blocks carrying Israel-Stewart fields (15 variables, passives from
    # 15) are accepted; a bulk-pressure offset past a 5-variable block is not
    p.physics, p.riemann = 0, 0
    p.passive_offset = 15
    g.nv = 15
    assert lib.astro_rhs_workspace_bytes(C.byref(p), C.byref(g)) > 0
    g.nv = 5
    assert lib.astro_rhs_workspace_bytes(C.byref(p), C.byref(g)) == 0


def test_empty_batches_are_no_ops(lib):
    """A count of 0 returns ASTRO_OK before any device work, null arrays
    allowed; a positive count with null arrays or a negative count is
    rejected on the host."""
    p = _lib.AstroParams()
    p.physics, p.recon, p.riemann = 1, 2, 2
    p.gamma = p.srhd_gamma = 4.0 / 3.0
    assert lib.astro_p2c(C.byref(p), None, None, 0, None) == 0
    assert lib.astro_c2p(C.byref(p), None, None, 0, None, None) == 0
    assert lib.astro_c2p_learned(C.byref(p), None, None, 0, 2, None, 0, None, None, None) == 0
    assert lib.astro_c2p_features(None, None, 0, None) == 0
    assert lib.astro_mlp_forward(C.c_void_p(8), None, None, 0, None, None) == 0
    assert lib.astro_p2c(C.byref(p), None, None, 4, None) == -1
    assert lib.astro_c2p(C.byref(p), None, None, -1, None, None) == -1
    assert lib.astro_c2p_learned(C.byref(p), None, None, 4, 2, None, 0, None, None, None) == -1
    assert lib.astro_c2p_features(None, None, -2, None) == -1
    assert lib.astro_mlp_forward(None, None, None, 0, None, None) == -1


def test_static_scratch_rhs_host_checks(lib):
    """The allocation-free right-hand side checks its arguments on the host,
    before it looks up its device scratch or launches anything: null arrays
    are invalid, and a grid whose scratch would not fit the fixed 32 MiB
    array is refused with ASTRO_E_WORKSPACE.  The non-null addresses below are
    never dereferenced."""
    cap = lib.astro_rhs_static_max_bytes()
    assert cap == 32 << 20
    p = _lib.AstroParams()
    p.physics, p.recon, p.riemann = _lib.RMHD, 2, 1
    p.passive_offset = 9
    p.gamma = p.srhd_gamma = 4.0 / 3.0
    g = _lib.AstroGrid(9, 22, 22, 22, 0.1, 0.1, 0.1)
    assert 0 < lib.astro_rhs_workspace_bytes(C.byref(p), C.byref(g)) <= cap
    assert lib.astro_rhs_static(C.byref(p), C.byref(g), None, None, None) == -1
    g = _lib.AstroGrid(9, 134, 134, 134, 0.1, 0.1, 0.1)
    assert lib.astro_rhs_workspace_bytes(C.byref(p), C.byref(g)) > cap
    dummy = C.c_void_p(16)
    assert lib.astro_rhs_static(C.byref(p), C.byref(g), dummy, dummy, None) == -3
    # invalid parameters are reported before the size check
    p.riemann = 7
    assert lib.astro_rhs_static(C.byref(p), C.byref(g), dummy, dummy, None) == -1


def test_product_raises_without_gpu_instead_of_falling_back():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    import numpy as np
    from astrofd_b200.core import srhd_core
    pr = np.ones((5, 12, 12, 12))
    with pytest.raises(_lib.AstroError):
        srhd_core.compute_rhs_muscl(pr, 12, 12, 12, 0.1, 0.1, 0.1)
