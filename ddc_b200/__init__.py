"""B200-native batched spline builder / evaluator (DDC's SplineBuilder / SplineEvaluator hot path).

The compute runs in hand-written sm_100a CUDA kernels inside libddcb.so, reached through the C-ABI
of include/ddcb.h; this package is the host-side mirror of the reference's spline API.
"""
from . import _lib
from ._lib import DdcbError
from .splines import (BSplines, Extrapolation, HostPipeline, NonUniformBSplines, SplineBuilder, SplineBuilder2D,
                      SplineBuilder3D, SplineBuilderClosure, SplineEvaluator, SplineEvaluator2D, SplineEvaluator3D,
                      SplineEvaluatorND, UnevenBatch, UniformBSplines, greville_points, lines_of, n_boundary_equations)

__all__ = [
    "BSplines", "UniformBSplines", "NonUniformBSplines", "SplineBuilder", "SplineEvaluator", "SplineBuilder2D",
    "SplineEvaluator2D", "SplineBuilder3D", "SplineEvaluator3D", "SplineEvaluatorND", "SplineBuilderClosure",
    "UnevenBatch", "HostPipeline",
    "Extrapolation", "greville_points", "lines_of", "n_boundary_equations", "DdcbError", "load_library",
    "last_device_error", "bounds_checked",
]


def load_library():
    """Load libddcb.so (raises if it has not been built)."""
    return _lib.load()


def last_device_error(stream=None):
    """Wait for `stream` (torch's current stream by default) and raise DdcbError for a device-side
    failure of the work queued on it (ddcb_last_device_error): a failed kernel, or, in the
    bounds-checked build, an array index a kernel found out of range."""
    from .splines import _stream_handle

    _lib.call("ddcb_last_device_error", _stream_handle(stream))


def bounds_checked() -> bool:
    """Whether the loaded library is the bounds-checked build (DDCB_CHECK_BOUNDS=1)."""
    return bool(_lib.load().ddcb_bounds_checked())
