"""ctypes binding of libddcb.so (the C-ABI declared in include/ddcb.h).

The library is built in-tree (ddc_b200/build.py). There is no fallback: if the shared library is
missing or a CUDA call fails, the functions here raise.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# DDCB_CHECK_BOUNDS=1 in the environment selects the bounds-checked build (libddcb_check.so): the
# same kernels, each computed array index checked on the device (ddcb_last_device_error)
LIB_PATH = os.path.join(HERE, "libddcb_check.so" if os.environ.get("DDCB_CHECK_BOUNDS") == "1" else "libddcb.so")

# enums (include/ddcb.h)
PERIODIC, HERMITE, HOMOGENEOUS_HERMITE, GREVILLE = 0, 1, 2, 3
EXTRAP_PERIODIC, EXTRAP_NULL, EXTRAP_CONSTANT = 0, 1, 2
FP64, FP32_REFINE = 0, 1

STATUS = {
    0: "DDCB_SUCCESS",
    1: "DDCB_ERR_INVALID_ARGUMENT",
    2: "DDCB_ERR_BAD_GRID",
    3: "DDCB_ERR_SINGULAR",
    4: "DDCB_ERR_CUDA",
    5: "DDCB_ERR_UNSUPPORTED",
    6: "DDCB_ERR_NOT_CONVERGED",
    7: "DDCB_ERR_DEVICE",
}


class DdcbError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class Lines(C.Structure):
    _fields_ = [("n", C.c_int64), ("stride", C.c_int64), ("inner", C.c_int64), ("outer", C.c_int64),
                ("outer_stride", C.c_int64)]

    def __repr__(self):
        return f"Lines(n={self.n}, stride={self.stride}, inner={self.inner}, outer={self.outer}, outer_stride={self.outer_stride})"


class BSplinesInfo(C.Structure):
    _fields_ = [("degree", C.c_int32), ("periodic", C.c_int32), ("uniform", C.c_int32), ("ncells", C.c_int64),
                ("nbasis", C.c_int64), ("size", C.c_int64), ("rmin", C.c_double), ("rmax", C.c_double)]


class BuilderOptions(C.Structure):
    _fields_ = [("precision", C.c_int32), ("refine_rounds", C.c_int32), ("tile_lines", C.c_int32),
                ("chunks", C.c_int32), ("refine_tolerance", C.c_double)]


class BuilderInfo(C.Structure):
    _fields_ = [("nbasis", C.c_int64), ("size", C.c_int64), ("npoints", C.c_int64), ("nbe_lo", C.c_int32),
                ("nbe_hi", C.c_int32), ("nbv_lo", C.c_int32), ("nbv_hi", C.c_int32), ("offset", C.c_int32),
                ("dx", C.c_double), ("border", C.c_int32), ("kl", C.c_int32), ("ku", C.c_int32),
                ("pivoting", C.c_int32), ("chunks", C.c_int32), ("tile_lines", C.c_int32)]


class UnevenInfo(C.Structure):
    _fields_ = [("count", C.c_int64), ("total_vals", C.c_int64), ("total_derivs_lo", C.c_int64),
                ("total_derivs_hi", C.c_int64), ("total_coefs", C.c_int64), ("total_evals", C.c_int64),
                ("threads", C.c_int32), ("blocks_per_sm", C.c_int32), ("order", C.c_int32),
                ("shared_bytes", C.c_int32), ("tuned_us", C.c_double), ("warp_schedule", C.c_int32)]


_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
_pp = C.POINTER(C.c_void_p)

# name -> argtypes (every function returns ddcb_status, except the two string getters)
SIGNATURES = {
    "ddcb_bsplines_create_uniform": [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_int64, _pp],
    "ddcb_bsplines_create_non_uniform": [C.c_int32, C.c_int32, _vp, C.c_int64, _pp],
    "ddcb_bsplines_destroy": [_vp],
    "ddcb_bsplines_get_info": [_vp, C.POINTER(BSplinesInfo)],
    "ddcb_bsplines_knots": [_vp, C.c_int64, C.c_int64, _vp],
    "ddcb_greville_points": [_vp, C.c_int, C.c_int, _vp, C.c_int64, C.POINTER(C.c_int64)],
    "ddcb_bsplines_integrals": [_vp, _vp],
    "ddcb_builder_create": [_vp, _vp, C.c_int64, C.c_int, C.c_int, C.POINTER(BuilderOptions), _pp],
    "ddcb_builder_destroy": [_vp],
    "ddcb_builder_get_info": [_vp, C.POINTER(BuilderInfo)],
    "ddcb_builder_device_status": [_vp, _vp],
    "ddcb_last_device_error": [_vp],
    "ddcb_build": [_vp, _vp, Lines, _vp, Lines, _vp, Lines, _vp, Lines, _vp],
    "ddcb_solve_multirhs": [_vp, _vp, C.c_int64, C.c_int64, C.c_int32, _vp],
    "ddcb_quadrature_coefficients": [_vp, _vp, _vp, _vp],
    "ddcb_quadrature_coefficients_device": [_vp, _vp, _vp],
    "ddcb_integrate_samples": [_vp, _vp, C.c_int64, _vp, Lines, _vp, Lines, _vp, Lines, _vp],
    "ddcb_evaluator_create": [_vp, C.c_int, C.c_int, _pp],
    "ddcb_evaluator_destroy": [_vp],
    "ddcb_eval": [_vp, _vp, Lines, _vp, Lines, _vp, Lines, _vp],
    "ddcb_eval_deriv": [_vp, C.c_int32, _vp, Lines, _vp, Lines, _vp, Lines, _vp],
    "ddcb_integrate": [_vp, _vp, C.c_int64, _vp, Lines, _vp],
    "ddcb_batch_uneven_create": [_vp, _vp, _vp, C.c_int64, _pp],
    "ddcb_batch_uneven_destroy": [_vp],
    "ddcb_batch_uneven_get_info": [_vp, C.POINTER(UnevenInfo)],
    "ddcb_batch_uneven_offsets": [_vp, _vp, _vp, _vp, _vp, _vp],
    "ddcb_batch_uneven_tune": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int32, _vp],
    "ddcb_batch_uneven_run": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "ddcb_host_pipeline_create": [_vp, _vp, C.c_int32, C.c_int64, C.c_int64, _pp],
    "ddcb_host_pipeline_destroy": [_vp],
    "ddcb_host_pipeline_run": [_vp, _vp, Lines, _vp, Lines, _vp, Lines, _vp, Lines, _vp, Lines, _vp, Lines, _vp],
    "ddcb_build2d_workspace_bytes": [_vp, _vp, C.c_int64, C.POINTER(C.c_uint64)],
    "ddcb_build2d": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int64, _vp, C.c_uint64, _vp],
    "ddcb_eval2d": [_vp, _vp, C.c_int32, C.c_int32, _vp, _vp, _vp, C.c_int64, C.c_int64, _vp],
    "ddcb_integrate2d": [_vp, _vp, _vp, _vp, C.c_int64, _vp],
    "ddcb_build3d_workspace_bytes": [_vp, _vp, _vp, C.c_int64, C.POINTER(C.c_uint64)],
    "ddcb_build3d": [_vp, _vp, _vp, _vp, _vp, C.c_int64, _vp, C.c_uint64, _vp],
    "ddcb_evalnd": [_vp, C.c_int32, _vp, _vp, _vp, _vp, C.c_int64, C.c_int64, _vp],
    "ddcb_integratend": [_vp, C.c_int32, _vp, _vp, C.c_int64, _vp],
    "ddcb_build_eval": [_vp, _vp, C.c_int32, _vp, Lines, _vp, Lines, _vp, Lines, _vp, Lines, _vp, Lines, _vp, Lines,
                        C.POINTER(C.c_int32), _vp],
    "ddcb_advect": [_vp, _vp, C.c_double, _vp, C.c_int64, C.c_double, _vp, Lines, _vp, Lines, _vp, Lines, _vp, Lines,
                    _vp, Lines, C.POINTER(C.c_int32), _vp],
    "ddcb_build_adjoint": [_vp, _vp, Lines, _vp, Lines, _vp, Lines, _vp, Lines, _vp],
    "ddcb_eval_adjoint": [_vp, C.c_int32, _vp, Lines, _vp, Lines, _vp, Lines, _vp, Lines, _vp, Lines, _vp],
    "ddcb_build_eval_adjoint": [_vp, _vp, C.c_int32, _vp, Lines, _vp, Lines, _vp, Lines, _vp, Lines, _vp, Lines, _vp,
                                Lines, _vp, Lines, C.POINTER(C.c_int32), _vp],
}

_lib = None


def load():
    """Load libddcb.so; raises if it is absent (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m ddc_b200.build` (nvcc, sm_100a)")
    L = C.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.ddcb_status_string.argtypes = [C.c_int]
    L.ddcb_status_string.restype = C.c_char_p
    L.ddcb_last_error_message.argtypes = []
    L.ddcb_last_error_message.restype = C.c_char_p
    L.ddcb_bounds_checked.argtypes = []
    L.ddcb_bounds_checked.restype = C.c_int32
    _lib = L
    return L


def check(status: int):
    if status != 0:
        msg = load().ddcb_last_error_message().decode()
        raise DdcbError(status, msg)


def call(name: str, *args):
    check(getattr(load(), name)(*args))
