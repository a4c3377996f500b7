"""ctypes binding of libpincflow_poisson.so (include/pincflow_poisson.h).

The library is the product: there is no fallback.  Loading fails loudly if
the shared object is missing; calls fail loudly (PoissonError) on any
non-zero return code.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# PCF_LIB_VARIANT=checked selects the bounds-checked build (build.py --checked)
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libpincflow_poisson_checked.so"
                        if os.environ.get("PCF_LIB_VARIANT") == "checked" else "libpincflow_poisson.so")

# enum values of include/pincflow_poisson.h
PCF_OK = 0
PCF_EINVAL = -1
PCF_ENOMEM = -2
PCF_ECUDA = -3
PCF_ENOTREADY = -4
PCF_EBREAKDOWN = -5
PCF_ENONFINITE = -6
PCF_ENODEVICE = -7
PCF_ERANGE = -8

MODEL = {"Boussinesq": 0, "PseudoIncompressible": 1, "Compressible": 2}
PRECISION = {"fp64": 0, "mixed": 1, "fp32": 2}
RESIDUAL = {"recursive": 0, "true": 1}
TOTAL, HORIZONTAL = 0, 1
NCOEF = 25

EXPORTS = [
    "pcf_params_default", "pcf_create", "pcf_destroy", "pcf_strerror", "pcf_set_grid",
    "pcf_set_background", "pcf_solve", "pcf_solve_device", "pcf_compute_operator",
    "pcf_set_operator", "pcf_apply_operator", "pcf_apply_preconditioner", "pcf_bicgstab",
    "pcf_global_dot", "pcf_device_bytes", "pcf_launch_count", "pcf_profile_enable", "pcf_profile_read",
    "pcf_residual_history", "pcf_multigrid_levels", "pcf_multigrid_operator", "pcf_apply_multigrid",
    "pcf_autotune_entries", "pcf_autotune_clear", "pcf_ensemble_create", "pcf_ensemble_destroy",
    "pcf_ensemble_solve_device", "pcf_ensemble_launch_count", "pcf_compute_lhs", "pcf_compute_lhs_device",
    "pcf_correct", "pcf_correct_device", "pcf_apply_corrector_device",
    "pcf_set_predictand_boundaries_device", "pcf_modify_compressible_wind_device",
    "pcf_implicit_predictor_device", "pcf_implicit_step_device", "pcf_implicit_step",
    "pcf_test_stall_staged_copy", "pcf_bounds_check_status",
]
TUNE_KERNELS = ["total32", "total32_diff", "horiz32", "total64", "horiz64"]
PROF_TAGS = ["apply32", "apply64", "pseudo32", "pseudo64", "thomas32", "thomas64", "update32", "update64",
             "assemble", "reliable64", "mg", "learned", "predict", "correct", "mg_bf16"]


class PcfDims(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("nbx", ctypes.c_int), ("nby", ctypes.c_int), ("nbz", ctypes.c_int),
                ("model", ctypes.c_int), ("device", ctypes.c_int)]


class PcfParams(ctypes.Structure):
    _fields_ = [("tolerance", ctypes.c_double), ("poisson_iterations", ctypes.c_int),
                ("preconditioner", ctypes.c_int), ("dtau", ctypes.c_double),
                ("preconditioner_iterations", ctypes.c_int),
                ("tolerance_is_relative", ctypes.c_int),
                ("damp_horizontal_wind_on_rhs", ctypes.c_int), ("precision", ctypes.c_int),
                ("residual", ctypes.c_int), ("inner_tolerance", ctypes.c_double),
                ("max_refinements", ctypes.c_int), ("learned", ctypes.c_int),
                ("check_interval", ctypes.c_int), ("restart_interval", ctypes.c_int),
                ("multigrid", ctypes.c_int), ("mg_dtau", ctypes.c_double),
                ("mg_coarse_iterations", ctypes.c_int), ("mg_min_columns", ctypes.c_int),
                ("autotune", ctypes.c_int), ("mg_operator_bf16", ctypes.c_int),
                ("mg_fused_coarse", ctypes.c_int), ("mg_smoother_fp8", ctypes.c_int)]


class PcfTuneEntry(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("tile_x", ctypes.c_int), ("vec", ctypes.c_int), ("levels", ctypes.c_int),
                ("ms_best", ctypes.c_double), ("ms_default", ctypes.c_double)]


class PcfResult(ctypes.Structure):
    _fields_ = [("errflag", ctypes.c_int), ("niter", ctypes.c_int), ("nrefine", ctypes.c_int),
                ("status", ctypes.c_int), ("residual", ctypes.c_double),
                ("true_residual", ctypes.c_double), ("b_norm", ctypes.c_double),
                ("ms_upload", ctypes.c_double), ("ms_assemble", ctypes.c_double),
                ("ms_solve", ctypes.c_double), ("ms_download", ctypes.c_double),
                ("ms_total", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class PoissonError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        super().__init__(f"{what}: {strerror(code)} ({code})")


_lib = None


def load(path: str | None = None):
    """Loads the solver library (once).  Raises OSError if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise OSError(f"libpincflow_poisson.so not found at {p}; run pincflow.jl_b200/build.py")
    lib = ctypes.CDLL(p)
    P = ctypes.POINTER
    dp = P(ctypes.c_double)
    vp = ctypes.c_void_p
    lib.pcf_strerror.restype = ctypes.c_char_p
    lib.pcf_strerror.argtypes = [ctypes.c_int]
    lib.pcf_params_default.argtypes = [P(PcfParams)]
    lib.pcf_create.argtypes = [P(vp), P(PcfDims)]
    lib.pcf_destroy.argtypes = [vp]
    lib.pcf_set_grid.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, dp, dp, dp, dp]
    lib.pcf_set_background.argtypes = [vp, dp, dp, dp, dp]
    lib.pcf_solve.argtypes = [vp, dp, dp, dp, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                              P(PcfParams), dp, P(PcfResult)]
    lib.pcf_solve_device.argtypes = [vp, vp, vp, vp, vp, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, P(PcfParams), vp, P(PcfResult)]
    lib.pcf_compute_operator.argtypes = [vp, dp, dp, dp, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_int, dp]
    lib.pcf_set_operator.argtypes = [vp, dp]
    lib.pcf_apply_operator.argtypes = [vp, dp, dp, ctypes.c_int, ctypes.c_int]
    lib.pcf_apply_preconditioner.argtypes = [vp, dp, dp, P(PcfParams), ctypes.c_int]
    lib.pcf_bicgstab.argtypes = [vp, dp, ctypes.c_double, P(PcfParams), dp, P(PcfResult)]
    lib.pcf_global_dot.argtypes = [vp, dp, dp, dp]
    lib.pcf_device_bytes.restype = ctypes.c_longlong
    lib.pcf_device_bytes.argtypes = [vp]
    lib.pcf_launch_count.restype = ctypes.c_longlong
    lib.pcf_launch_count.argtypes = [vp]
    lib.pcf_profile_enable.argtypes = [vp, ctypes.c_int]
    lib.pcf_profile_read.argtypes = [vp, ctypes.c_int, dp, P(ctypes.c_longlong), dp]
    lib.pcf_residual_history.argtypes = [vp, dp, ctypes.c_int, P(ctypes.c_int)]
    lib.pcf_multigrid_levels.argtypes = [vp, P(PcfParams), ctypes.c_int, P(ctypes.c_int), P(ctypes.c_int)]
    lib.pcf_multigrid_operator.argtypes = [vp, ctypes.c_int, dp]
    lib.pcf_apply_multigrid.argtypes = [vp, dp, dp, P(PcfParams)]
    lib.pcf_autotune_entries.argtypes = [P(PcfTuneEntry), ctypes.c_int, P(ctypes.c_int)]
    lib.pcf_autotune_clear.argtypes = []
    lib.pcf_compute_lhs.argtypes = [vp, dp, dp, dp, dp, dp, dp]
    lib.pcf_compute_lhs_device.argtypes = [vp, vp, vp, vp, vp, vp, dp]
    lib.pcf_correct.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, dp, dp, dp, dp, dp, dp]
    lib.pcf_correct_device.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, vp, vp, vp, vp, vp, vp]
    lib.pcf_apply_corrector_device.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_double,
                                               ctypes.c_double, P(PcfParams), vp, P(PcfResult)]
    f64 = ctypes.c_double
    lib.pcf_set_predictand_boundaries_device.argtypes = [vp] + [vp] * 7
    lib.pcf_modify_compressible_wind_device.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int]
    lib.pcf_implicit_predictor_device.argtypes = [vp, f64, f64, ctypes.c_int] + [vp] * 11
    lib.pcf_implicit_step_device.argtypes = [vp, f64, f64, P(PcfParams)] + [vp] * 13 + [P(PcfResult)]
    lib.pcf_implicit_step.argtypes = [vp, f64, f64, P(PcfParams)] + [dp] * 13 + [P(PcfResult)]
    lib.pcf_test_stall_staged_copy.argtypes = [vp, ctypes.c_int, f64]
    lib.pcf_bounds_check_status.argtypes = [P(ctypes.c_int), P(ctypes.c_longlong), P(ctypes.c_longlong)]
    for name in EXPORTS:
        getattr(lib, name).restype = getattr(lib, name).restype or ctypes.c_int
    lib.pcf_strerror.restype = ctypes.c_char_p
    lib.pcf_device_bytes.restype = ctypes.c_longlong
    lib.pcf_launch_count.restype = ctypes.c_longlong
    _lib = lib
    return lib


def strerror(code: int) -> str:
    try:
        return load().pcf_strerror(int(code)).decode()
    except OSError:
        return f"error {code}"


def check(code: int, what: str):
    if code != PCF_OK:
        raise PoissonError(code, what)


def dptr(a):
    """Pointer of a C-contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]):
        raise TypeError("expected a C-contiguous float64 numpy array")
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def bounds_check_status():
    """(enabled, site, index) of pcf_bounds_check_status: whether the loaded
    library is the bounds-checked build, and its first out-of-range access
    since the last call (site 0: none)."""
    lib = load()
    en, site, idx = ctypes.c_int(), ctypes.c_longlong(), ctypes.c_longlong()
    check(lib.pcf_bounds_check_status(ctypes.byref(en), ctypes.byref(site), ctypes.byref(idx)),
          "pcf_bounds_check_status")
    return bool(en.value), int(site.value), int(idx.value)
