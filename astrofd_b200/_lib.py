"""ctypes binding of libastrofd_b200.so (declarations in include/astrofd.h).

The shared library is built in-tree (``astrofd_b200/libastrofd_b200.so``) by
``python -m astrofd_b200.build``.  There is no CPU fallback: if the library is
missing, or no CUDA device is present, every entry point raises.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libastrofd_b200.so")

# enums (include/astrofd.h)
SRHD, RMHD = 0, 1
RECON = {"muscl": 0, "ppm": 1, "weno": 2}
LIMITER = {"mc": 0, "minmod": 1, "vanleer": 2}
FLUX_REFERENCE, FLUX_CONSERVATIVE = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
GUESS_REFERENCE, GUESS_LEARNED = 0, 1

ERRORS = {0: "ok", -1: "invalid argument", -2: "grid shape incompatible",
          -3: "workspace missing or too small", -4: "configuration not supported",
          -5: "CUDA error"}


class AstroParams(C.Structure):
    _fields_ = [("physics", C.c_int32), ("recon", C.c_int32), ("limiter", C.c_int32),
                ("riemann", C.c_int32), ("n_passive", C.c_int32),
                ("passive_offset", C.c_int32), ("resistive", C.c_int32),
                ("flux_mode", C.c_int32), ("precision", C.c_int32),
                ("c2p_guess", C.c_int32), ("fused_stage", C.c_int32),
                ("mlp", C.c_void_p), ("gamma", C.c_double),
                ("srhd_gamma", C.c_double), ("p_max", C.c_double),
                ("v_max", C.c_double), ("glm_ch", C.c_double), ("glm_cp", C.c_double),
                ("resistivity", C.c_double)]


class AstroGrid(C.Structure):
    _fields_ = [("nv", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32),
                ("nz", C.c_int32), ("dx", C.c_double), ("dy", C.c_double),
                ("dz", C.c_double)]


class AstroNozzle(C.Structure):
    _fields_ = [("ng", C.c_int32), ("profile", C.c_int32), ("perturb", C.c_int32),
                ("physics", C.c_int32), ("b_init", C.c_int32), ("n_tracers", C.c_int32),
                ("tracer_offset", C.c_int32), ("two_temperature", C.c_int32),
                ("thermo_offset", C.c_int32), ("ambient_bc", C.c_int32),
                ("radius", C.c_double), ("shear_thick", C.c_double),
                ("gamma_jet", C.c_double), ("eta_rho", C.c_double), ("p_eq", C.c_double),
                ("rho_amb", C.c_double), ("vx_amb", C.c_double), ("vy_amb", C.c_double),
                ("vz_amb", C.c_double), ("turb_vamp", C.c_double),
                ("turb_pamp", C.c_double), ("b0", C.c_double), ("te", C.c_double),
                ("ti", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("y0", C.c_double), ("z0", C.c_double),
                ("tracer_nozzle", C.c_double * 8), ("tracer_amb", C.c_double * 8),
                ("b_amb_x", C.c_double), ("chemistry", C.c_int32),
                ("chem_offset", C.c_int32), ("chem_x", C.c_double * 3)]


class AstroChemistry(C.Structure):
    _fields_ = [("ng", C.c_int32), ("chem_offset", C.c_int32), ("x", C.c_double),
                ("y", C.c_double), ("tunit_k", C.c_double), ("rate_scale", C.c_double),
                ("energy_scale", C.c_double), ("tmin_k", C.c_double), ("gamma", C.c_double)]


class AstroDissipation(C.Structure):
    _fields_ = [("ng", C.c_int32), ("advect", C.c_int32), ("zeta", C.c_double),
                ("eta", C.c_double), ("kappa", C.c_double), ("tau_bulk", C.c_double),
                ("tau_shear", C.c_double), ("tau_heat", C.c_double), ("cap_frac", C.c_double),
                ("p_max", C.c_double)]


class AstroGR(C.Structure):
    _fields_ = [("metric", C.c_int32), ("orthonormal_flux", C.c_int32), ("ng", C.c_int32),
                ("offs_x", C.c_int32), ("mass", C.c_double), ("spin", C.c_double)]


GR_MINKOWSKI, GR_SCHWARZSCHILD, GR_KERR_SCHILD, GR_OTHER = 0, 1, 2, 3


class AstroC2PStats(C.Structure):
    _fields_ = [(n, C.c_ulonglong) for n in
                ("cells", "newton", "bisection", "hydro_fallback", "learned_polish",
                 "learned_fallback", "polish_steps", "wait_timeouts")]


class AstroKernelTimes(C.Structure):
    _fields_ = [("ms", C.c_double * 5), ("launches", C.c_int32 * 5)]


# every symbol include/astrofd.h declares, with its ctypes prototype
_VP, _DP = C.c_void_p, C.c_void_p
PROTOS = {
    "astro_version": (C.c_int, []),
    "astro_error_string": (C.c_char_p, [C.c_int]),
    "astro_rhs_workspace_bytes": (C.c_size_t, [C.POINTER(AstroParams), C.POINTER(AstroGrid)]),
    "astro_rhs": (C.c_int, [C.POINTER(AstroParams), C.POINTER(AstroGrid), _DP, _DP, _VP,
                            C.c_size_t, _VP]),
    "astro_rhs_static_max_bytes": (C.c_size_t, []),
    "astro_rhs_static": (C.c_int, [C.POINTER(AstroParams), C.POINTER(AstroGrid), _DP, _DP,
                                   _VP]),
    "astro_step_workspace_bytes": (C.c_size_t, [C.POINTER(AstroParams), C.POINTER(AstroGrid)]),
    "astro_step": (C.c_int, [C.POINTER(AstroParams), C.POINTER(AstroGrid), _DP, _DP,
                             C.c_double, C.c_int, _VP, C.c_size_t, _VP, _VP]),
    "astro_step_profiled": (C.c_int, [C.POINTER(AstroParams), C.POINTER(AstroGrid), _DP, _DP,
                                      C.c_double, C.c_int, _VP, C.c_size_t, _VP, _VP,
                                      C.POINTER(AstroKernelTimes)]),
    "astro_launch_count": (C.c_ulonglong, []),
    "astro_debug_set_mma_poll_limit": (C.c_int, [C.c_longlong]),
    "astro_debug_set_step_polish": (C.c_int, [C.c_int]),
    "astro_debug_set_tile_poll_limit": (C.c_int, [C.c_longlong]),
    "astro_debug_rcp_f64": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    "astro_max_char_speed_workspace_bytes": (C.c_size_t, []),
    "astro_max_char_speed": (C.c_int, [C.POINTER(AstroParams), C.POINTER(AstroGrid), _DP,
                                       _DP, _VP, C.c_size_t, _VP]),
    "astro_periodic_yz": (C.c_int, [_DP, C.POINTER(AstroGrid), C.c_int, _VP]),
    "astro_outflow_right_x": (C.c_int, [_DP, C.POINTER(AstroGrid), C.c_int, _VP]),
    "astro_outflow_yz": (C.c_int, [_DP, C.POINTER(AstroGrid), C.c_int, _VP]),
    "astro_ion_chemistry": (C.c_int, [_DP, C.POINTER(AstroGrid), C.POINTER(AstroChemistry),
                                      C.c_double, _VP]),
    "astro_step_stage": (C.c_int, [C.POINTER(AstroParams), C.POINTER(AstroGrid), _DP, _DP, _DP,
                                   C.c_double, C.c_int, C.c_int, _VP, C.c_size_t, _VP, _VP]),
    "astro_prof_start": (C.c_int, [C.c_int, _VP]),
    "astro_prof_stop": (C.c_int, [C.POINTER(AstroKernelTimes)]),
    "astro_diagnostics": (C.c_int, [C.POINTER(AstroParams), C.POINTER(AstroGrid), C.c_int, _DP,
                                    C.c_double, _DP, _VP]),
    "astro_gr_workspace_bytes": (C.c_size_t, [C.POINTER(AstroParams), C.POINTER(AstroGrid),
                                              C.POINTER(AstroGR), C.c_int]),
    "astro_rhs_gr": (C.c_int, [C.POINTER(AstroParams), C.POINTER(AstroGrid), C.POINTER(AstroGR),
                               _DP, _DP, _VP, C.c_size_t, _VP]),
    "astro_step_gr": (C.c_int, [C.POINTER(AstroParams), C.POINTER(AstroGrid), C.POINTER(AstroGR),
                                _DP, _DP, C.c_double, C.c_int, _VP, C.c_size_t, _VP, _VP]),
    "astro_causal_dissipation_workspace_bytes": (C.c_size_t, [C.POINTER(AstroGrid)]),
    "astro_causal_dissipation": (C.c_int, [_DP, C.POINTER(AstroGrid), C.POINTER(AstroDissipation),
                                           C.c_double, _VP, C.c_size_t, _VP]),
    "astro_nozzle_left_x": (C.c_int, [_DP, C.POINTER(AstroGrid), C.POINTER(AstroNozzle),
                                      _DP, _VP, C.c_int32, _VP]),
    "astro_p2c": (C.c_int, [C.POINTER(AstroParams), _DP, _DP, C.c_int64, _VP]),
    "astro_c2p": (C.c_int, [C.POINTER(AstroParams), _DP, _DP, C.c_int64, _VP, _VP]),
    "astro_mlp_param_bytes": (C.c_size_t, []),
    "astro_mlp_trainable": (C.c_int, []),
    "astro_c2p_features": (C.c_int, [_DP, _DP, C.c_int64, _VP]),
    "astro_mlp_forward": (C.c_int, [_VP, _DP, _DP, C.c_int64, _VP, _VP]),
    "astro_mlp_train_grad": (C.c_int, [_VP, _DP, _DP, C.c_int64, _DP, _DP, _VP, _VP]),
    "astro_mlp_adam": (C.c_int, [_VP, _DP, _DP, _DP, C.c_float, C.c_float, C.c_float,
                                 C.c_float, C.c_int, _VP]),
    "astro_c2p_learned_workspace_bytes": (C.c_size_t, [C.c_int64]),
    "astro_c2p_learned": (C.c_int, [C.POINTER(AstroParams), _DP, _DP, C.c_int64, C.c_int,
                                    _VP, C.c_size_t, _VP, _VP, _VP]),
    "astro_cooling_heating": (C.c_int, [_DP, C.POINTER(AstroGrid), C.c_int, C.c_double,
                                        C.c_double, C.c_double, C.c_double, _VP]),
    "astro_two_temperature": (C.c_int, [_DP, C.POINTER(AstroGrid), C.c_int, C.c_double,
                                        C.c_double, C.c_int, _VP]),
}

_lib = None


class AstroError(RuntimeError):
    pass


def load():
    """Load the shared library; raises when it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise AstroError(
            f"{LIB_PATH} not found: build it with `python -m astrofd_b200.build` "
            "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in PROTOS.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(rc, what):
    if rc != 0:
        raise AstroError(f"{what} failed: {ERRORS.get(rc, rc)}")
