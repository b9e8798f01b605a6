"""Host-side mirror of DDC's spline API (src/ddc/kernels/splines/) over the C-ABI.

Class and argument names follow the reference: UniformBSplines / NonUniformBSplines
(bsplines_uniform.hpp, bsplines_non_uniform.hpp), GrevilleInterpolationPoints
(greville_interpolation_points.hpp), SplineBuilder (spline_builder.hpp) and SplineEvaluator
(spline_evaluator.hpp). Batched data are CUDA tensors (the reference's ChunkSpans in a device
memory space); the dimension of interest is given by `dim`, every other dimension is a batch
dimension, in any order (the reference's 1DX / 2DXB1 / 2DB1X ... layouts).

Errors follow the reference: invalid grids raise RuntimeError with the reference's messages
(check_valid_grid), and every failing C call raises ddc_b200._lib.DdcbError.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import (EXTRAP_CONSTANT, EXTRAP_NULL, EXTRAP_PERIODIC, FP32_REFINE, FP64, GREVILLE, HERMITE,
                   HOMOGENEOUS_HERMITE, PERIODIC, BuilderInfo, BuilderOptions, BSplinesInfo, Lines, UnevenInfo)


class SplineBuilderClosure:
    """ddc::SplineBuilderClosure (spline_builder_closures.hpp:18-23)."""

    PERIODIC = PERIODIC
    HERMITE = HERMITE
    HOMOGENEOUS_HERMITE = HOMOGENEOUS_HERMITE
    GREVILLE = GREVILLE


class Extrapolation:
    PERIODIC = EXTRAP_PERIODIC
    NULL = EXTRAP_NULL
    CONSTANT = EXTRAP_CONSTANT


def n_boundary_equations(closure: int, degree: int) -> int:
    """spline_builder_closures.hpp:43-55."""
    return degree // 2 if closure in (HERMITE, HOMOGENEOUS_HERMITE) else 0


def _stream_handle(stream):
    import torch

    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


def lines_of(t, dim: int) -> Lines:
    """ddcb_lines of tensor `t` with interest dimension `dim`; batch = all other dims (row-major)."""
    shape = list(t.shape)
    stride = list(t.stride())
    nd = len(shape)
    dim = dim % nd if nd else 0
    n = shape[dim] if nd else 1
    inner_dims = list(range(dim + 1, nd))
    outer_dims = list(range(0, dim))
    inner = math.prod(shape[d] for d in inner_dims)
    outer = math.prod(shape[d] for d in outer_dims)
    exp = 1
    for d in reversed(inner_dims):
        if shape[d] > 1 and stride[d] != exp:
            raise ValueError("the batch dimensions after the interest dimension must be contiguous")
        exp *= shape[d]
    os_ = 0
    if outer_dims:
        os_ = stride[outer_dims[-1]] if shape[outer_dims[-1]] > 1 else 0
        exp = os_
        for d in reversed(outer_dims):
            if shape[d] > 1 and stride[d] != exp:
                raise ValueError("the batch dimensions before the interest dimension must be regularly strided")
            exp *= shape[d]
    return Lines(n, stride[dim] if nd else 1, inner, outer, os_)


def _ptr(t):
    return C.c_void_p(0 if t is None else t.data_ptr())


def _dev_f64(t, name):
    import torch

    if t is None:
        return None
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64):
        raise TypeError(f"{name} must be a CUDA float64 tensor")
    return t


class BSplines:
    """A B-spline basis: UniformBSplines<CDim, D>::Impl or NonUniformBSplines<CDim, D>::Impl."""

    def __init__(self, degree: int, periodic: bool, *, rmin=None, rmax=None, ncells=None, breaks=None):
        h = C.c_void_p()
        if breaks is None:
            _lib.call("ddcb_bsplines_create_uniform", int(degree), int(bool(periodic)), float(rmin), float(rmax),
                      int(ncells), C.byref(h))
        else:
            b = np.ascontiguousarray(breaks, dtype=np.float64)
            _lib.call("ddcb_bsplines_create_non_uniform", int(degree), int(bool(periodic)),
                      b.ctypes.data_as(C.c_void_p), b.size, C.byref(h))
        self._h = h
        info = BSplinesInfo()
        _lib.call("ddcb_bsplines_get_info", h, C.byref(info))
        self.degree = info.degree
        self.periodic = bool(info.periodic)
        self.uniform = bool(info.uniform)
        self.ncells = info.ncells
        self.nbasis = info.nbasis
        self.size = info.size
        self.rmin = info.rmin
        self.rmax = info.rmax

    def __del__(self):
        h = getattr(self, "_h", None)
        L = getattr(_lib, "_lib", None) if _lib is not None else None
        if h and L is not None:
            L.ddcb_bsplines_destroy(h)
            self._h = None

    @property
    def length(self):
        return self.rmax - self.rmin

    def knots(self) -> np.ndarray:
        n = self.ncells + 1 + 2 * self.degree
        out = np.zeros(n)
        _lib.call("ddcb_bsplines_knots", self._h, 0, n, out.ctypes.data_as(C.c_void_p))
        return out

    def integrals(self) -> np.ndarray:
        """integrals() of integrals.hpp:165-177: one value per B-spline (size() entries)."""
        out = np.zeros(self.size)
        _lib.call("ddcb_bsplines_integrals", self._h, out.ctypes.data_as(C.c_void_p))
        return out


def UniformBSplines(degree, periodic, rmin, rmax, ncells) -> BSplines:
    return BSplines(degree, periodic, rmin=rmin, rmax=rmax, ncells=ncells)


def NonUniformBSplines(degree, periodic, breaks) -> BSplines:
    return BSplines(degree, periodic, breaks=breaks)


def greville_points(bsplines: BSplines, lower: int, upper: int) -> np.ndarray:
    """GrevilleInterpolationPoints<BSplines, lower, upper>::get_sampling() coordinates."""
    n = C.c_int64()
    _lib.call("ddcb_greville_points", bsplines._h, int(lower), int(upper), None, 0, C.byref(n))
    out = np.zeros(n.value)
    _lib.call("ddcb_greville_points", bsplines._h, int(lower), int(upper), out.ctypes.data_as(C.c_void_p), out.size,
              C.byref(n))
    return out


class SplineBuilder:
    """ddc::SplineBuilder with the B200 solver: operator() builds spline coefficients on the GPU."""

    def __init__(self, bsplines: BSplines, interpolation_points: Optional[Sequence[float]] = None,
                 lower: int = GREVILLE, upper: int = GREVILLE, *, precision: str = "fp64", refine_rounds: int = 2,
                 tile_lines: int = 0, chunks: int = 0, refine_tolerance: float = 0.0):
        if bsplines.periodic:
            lower = upper = PERIODIC
        self.bsplines = bsplines
        self.lower, self.upper = lower, upper
        if interpolation_points is None:
            interpolation_points = greville_points(bsplines, lower, upper)
        pts = np.ascontiguousarray(interpolation_points, dtype=np.float64)
        self.interpolation_points = pts
        opts = BuilderOptions(FP32_REFINE if precision == "fp32_refine" else FP64, int(refine_rounds),
                              int(tile_lines), int(chunks), float(refine_tolerance))
        h = C.c_void_p()
        _lib.call("ddcb_builder_create", bsplines._h, pts.ctypes.data_as(C.c_void_p), pts.size, int(lower),
                  int(upper), C.byref(opts), C.byref(h))
        self._h = h
        info = BuilderInfo()
        _lib.call("ddcb_builder_get_info", h, C.byref(info))
        self.info = info
        self.s_nbe_xmin, self.s_nbe_xmax = info.nbe_lo, info.nbe_hi
        self.s_nbv_xmin, self.s_nbv_xmax = info.nbv_lo, info.nbv_hi
        self.s_odd = bsplines.degree % 2
        self.offset = info.offset
        self.dx = info.dx

    def __del__(self):
        h = getattr(self, "_h", None)
        L = getattr(_lib, "_lib", None) if _lib is not None else None
        if h and L is not None:
            L.ddcb_builder_destroy(h)
            self._h = None

    @property
    def npoints(self):
        return self.info.npoints

    def device_status(self, stream=None):
        """Raise DdcbError(DDCB_ERR_NOT_CONVERGED) if a refined solve queued so far missed its
        bound (ddcb_builder_device_status: waits for the stream, clears the flag)."""
        _lib.call("ddcb_builder_device_status", self._h, _stream_handle(stream))

    def __call__(self, spline, vals, derivs_xmin=None, derivs_xmax=None, *, dim: int = 0, stream=None):
        """SplineBuilder::operator()(spline, vals, derivs_xmin, derivs_xmax) (spline_builder.hpp:896-1101)."""
        spline = _dev_f64(spline, "spline")
        vals = _dev_f64(vals, "vals")
        dlo = _dev_f64(derivs_xmin, "derivs_xmin")
        dhi = _dev_f64(derivs_xmax, "derivs_xmax")
        lc, lv = lines_of(spline, dim), lines_of(vals, dim)
        llo = lines_of(dlo, dim) if dlo is not None else Lines(0, 1, 0, 0, 0)
        lhi = lines_of(dhi, dim) if dhi is not None else Lines(0, 1, 0, 0, 0)
        _lib.call("ddcb_build", self._h, _ptr(spline), lc, _ptr(vals), lv, _ptr(dlo), llo, _ptr(dhi), lhi,
                  _stream_handle(stream))
        return spline

    def build_and_evaluate(self, evaluator: "SplineEvaluator", spline, vals, coords_eval, spline_eval, derivs_xmin=None,
                           derivs_xmax=None, *, order: int = 0, dim: int = 0, stream=None) -> bool:
        """operator()(spline, vals, ...) then evaluator(spline_eval, coords_eval, spline) (order 0) or
        evaluator.deriv(order, ...) on the same lines, fused into one kernel when one exists.
        Returns True when the fused kernel ran."""
        spline = _dev_f64(spline, "spline")
        vals = _dev_f64(vals, "vals")
        dlo = _dev_f64(derivs_xmin, "derivs_xmin")
        dhi = _dev_f64(derivs_xmax, "derivs_xmax")
        x = _dev_f64(coords_eval, "coords_eval")
        out = _dev_f64(spline_eval, "spline_eval")
        llo = lines_of(dlo, dim) if dlo is not None else Lines(0, 1, 0, 0, 0)
        lhi = lines_of(dhi, dim) if dhi is not None else Lines(0, 1, 0, 0, 0)
        fused = C.c_int32(0)
        _lib.call("ddcb_build_eval", self._h, evaluator._h, int(order), _ptr(spline), lines_of(spline, dim), _ptr(vals),
                  lines_of(vals, dim), _ptr(dlo), llo, _ptr(dhi), lhi, _ptr(x), lines_of(x, dim), _ptr(out),
                  lines_of(out, dim), C.byref(fused), _stream_handle(stream))
        return bool(fused.value)

    def advect(self, evaluator: "SplineEvaluator", f_out, f_in, dt: float, velocity=0.0, derivs_xmin=None,
               derivs_xmax=None, spline=None, *, velocity_div: int = 1, dim: int = 0, stream=None) -> bool:
        """One semi-Lagrangian advection step (examples/characteristics_advection.cpp:243-259): the
        spline of every line of f_in evaluated at the feet x_q - dt * v of the interpolation points,
        into f_out. velocity: a float (every line) or a CUDA float64 tensor, line b taking
        velocity[b // velocity_div] (batch lines in the layout's order). spline, when given, receives
        the coefficients. Returns True when one fused kernel did the step."""
        out = _dev_f64(f_out, "f_out")
        vals = _dev_f64(f_in, "f_in")
        dlo = _dev_f64(derivs_xmin, "derivs_xmin")
        dhi = _dev_f64(derivs_xmax, "derivs_xmax")
        c = _dev_f64(spline, "spline")
        vt = None
        vconst = 0.0
        if isinstance(velocity, (int, float)):
            vconst = float(velocity)
        else:
            vt = _dev_f64(velocity, "velocity")
            assert vt.is_contiguous()
        empty = Lines(0, 1, 0, 0, 0)
        fused = C.c_int32(0)
        _lib.call("ddcb_advect", self._h, evaluator._h, float(dt), _ptr(vt), int(velocity_div), vconst, _ptr(out),
                  lines_of(out, dim), _ptr(vals), lines_of(vals, dim), _ptr(dlo),
                  lines_of(dlo, dim) if dlo is not None else empty, _ptr(dhi),
                  lines_of(dhi, dim) if dhi is not None else empty, _ptr(c), lines_of(c, dim) if c is not None else empty,
                  C.byref(fused), _stream_handle(stream))
        return bool(fused.value)

    def adjoint(self, g_spline, g_vals, g_derivs_xmin=None, g_derivs_xmax=None, *, dim: int = 0, stream=None):
        """Reverse mode of operator(): given the cotangents g_spline of the coefficients, writes the
        cotangents of vals (and of the Hermite derivatives, when tensors are given) -- the transposed
        solve of the interpolation matrix with the periodic duplicates folded back."""
        gc = _dev_f64(g_spline, "g_spline")
        gv = _dev_f64(g_vals, "g_vals")
        glo = _dev_f64(g_derivs_xmin, "g_derivs_xmin")
        ghi = _dev_f64(g_derivs_xmax, "g_derivs_xmax")
        llo = lines_of(glo, dim) if glo is not None else Lines(0, 1, 0, 0, 0)
        lhi = lines_of(ghi, dim) if ghi is not None else Lines(0, 1, 0, 0, 0)
        _lib.call("ddcb_build_adjoint", self._h, _ptr(gc), lines_of(gc, dim), _ptr(gv), lines_of(gv, dim), _ptr(glo),
                  llo, _ptr(ghi), lhi, _stream_handle(stream))
        return gv

    def build_and_evaluate_adjoint(self, evaluator: "SplineEvaluator", coords_eval, spline_coef, g_spline_eval, g_vals,
                                   g_coords=None, g_derivs_xmin=None, g_derivs_xmax=None, *, order: int = 0,
                                   dim: int = 0, stream=None) -> bool:
        """Reverse mode of build_and_evaluate: from the cotangents of the evaluated values, the
        cotangents of vals (and Hermite derivatives) and, when g_coords is given, of the coordinates
        (spline_coef is then read). Returns True when one fused kernel ran."""
        x = _dev_f64(coords_eval, "coords_eval")
        c = _dev_f64(spline_coef, "spline_coef")
        gy = _dev_f64(g_spline_eval, "g_spline_eval")
        gv = _dev_f64(g_vals, "g_vals")
        gx = _dev_f64(g_coords, "g_coords")
        glo = _dev_f64(g_derivs_xmin, "g_derivs_xmin")
        ghi = _dev_f64(g_derivs_xmax, "g_derivs_xmax")
        empty = Lines(0, 1, 0, 0, 0)
        fused = C.c_int32(0)
        _lib.call("ddcb_build_eval_adjoint", self._h, evaluator._h, int(order), _ptr(x), lines_of(x, dim), _ptr(c),
                  lines_of(c, dim) if c is not None else empty, _ptr(gy), lines_of(gy, dim), _ptr(gv), lines_of(gv, dim),
                  _ptr(glo), lines_of(glo, dim) if glo is not None else empty, _ptr(ghi),
                  lines_of(ghi, dim) if ghi is not None else empty, _ptr(gx),
                  lines_of(gx, dim) if gx is not None else empty, C.byref(fused), _stream_handle(stream))
        return bool(fused.value)

    def solve(self, rhs, transpose: bool = False, stream=None):
        """In-place SplinesLinearProblem::solve on a (nbasis, nrhs) CUDA float64 matrix."""
        rhs = _dev_f64(rhs, "rhs")
        assert rhs.ndim == 2 and rhs.shape[0] == self.info.nbasis and rhs.stride(1) == 1
        _lib.call("ddcb_solve_multirhs", self._h, _ptr(rhs), rhs.stride(0), rhs.shape[1], int(transpose),
                  _stream_handle(stream))
        return rhs

    def quadrature_coefficients(self):
        """quadrature_coefficients() (spline_builder.hpp:1103-1234): (q_derivs_xmin, q, q_derivs_xmax)."""
        nb = self.info.nbasis
        qlo = np.zeros(max(self.s_nbv_xmin, 1))
        q = np.zeros(nb - self.s_nbv_xmin - self.s_nbv_xmax)
        qhi = np.zeros(max(self.s_nbv_xmax, 1))
        _lib.call("ddcb_quadrature_coefficients", self._h, qlo.ctypes.data_as(C.c_void_p),
                  q.ctypes.data_as(C.c_void_p), qhi.ctypes.data_as(C.c_void_p))
        return qlo[: self.s_nbv_xmin], q, qhi[: self.s_nbv_xmax]

    def quadrature_coefficients_device(self, stream=None):
        """The quadrature weights as one CUDA float64 tensor of nbasis entries, [q_derivs_xmin, q,
        q_derivs_xmax] (quadrature_coefficients<OutMemorySpace>() with a device memory space)."""
        import torch

        out = torch.empty(self.info.nbasis, dtype=torch.float64, device="cuda")
        _lib.call("ddcb_quadrature_coefficients_device", self._h, _ptr(out), _stream_handle(stream))
        return out

    def integrate_samples(self, integrals, vals, derivs_xmin=None, derivs_xmax=None, *, dim: int = 0, stream=None):
        """The integral of the spline interpolating each batch line of vals (and its Hermite
        derivatives): operator() then SplineEvaluator::integrate in one pass over the samples.
        integrals has the batch shape of vals."""
        out = _dev_f64(integrals, "integrals")
        vals = _dev_f64(vals, "vals")
        dlo = _dev_f64(derivs_xmin, "derivs_xmin")
        dhi = _dev_f64(derivs_xmax, "derivs_xmax")
        lv = lines_of(vals, dim)
        assert out.numel() == lv.inner * lv.outer and out.is_contiguous()
        llo = lines_of(dlo, dim) if dlo is not None else Lines(0, 1, 0, 0, 0)
        lhi = lines_of(dhi, dim) if dhi is not None else Lines(0, 1, 0, 0, 0)
        _lib.call("ddcb_integrate_samples", self._h, _ptr(out), lv.inner, _ptr(vals), lv, _ptr(dlo), llo, _ptr(dhi), lhi,
                  _stream_handle(stream))
        return out


class SplineEvaluator:
    """ddc::SplineEvaluator<..., LowerExtrapolationRule, UpperExtrapolationRule>."""

    def __init__(self, bsplines: BSplines, lower_extrapolation: int = EXTRAP_NULL,
                 upper_extrapolation: int = EXTRAP_NULL):
        if bsplines.periodic:
            lower_extrapolation = upper_extrapolation = EXTRAP_PERIODIC
        self.bsplines = bsplines
        h = C.c_void_p()
        _lib.call("ddcb_evaluator_create", bsplines._h, int(lower_extrapolation), int(upper_extrapolation), C.byref(h))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        L = getattr(_lib, "_lib", None) if _lib is not None else None
        if h and L is not None:
            L.ddcb_evaluator_destroy(h)
            self._h = None

    def __call__(self, spline_eval, coords_eval, spline_coef, *, dim: int = 0, stream=None):
        """SplineEvaluator::operator()(spline_eval, coords_eval, spline_coef)."""
        out = _dev_f64(spline_eval, "spline_eval")
        x = _dev_f64(coords_eval, "coords_eval")
        c = _dev_f64(spline_coef, "spline_coef")
        _lib.call("ddcb_eval", self._h, _ptr(out), lines_of(out, dim), _ptr(x), lines_of(x, dim), _ptr(c),
                  lines_of(c, dim), _stream_handle(stream))
        return out

    def deriv(self, order: int, spline_eval, coords_eval, spline_coef, *, dim: int = 0, stream=None):
        """SplineEvaluator::deriv(DiscreteElement<Deriv<X>>(order), spline_eval, coords_eval, spline_coef)."""
        out = _dev_f64(spline_eval, "spline_eval")
        x = _dev_f64(coords_eval, "coords_eval")
        c = _dev_f64(spline_coef, "spline_coef")
        _lib.call("ddcb_eval_deriv", self._h, int(order), _ptr(out), lines_of(out, dim), _ptr(x), lines_of(x, dim),
                  _ptr(c), lines_of(c, dim), _stream_handle(stream))
        return out

    def adjoint(self, coords_eval, g_spline_eval, g_spline_coef, spline_coef=None, g_coords=None, *, order: int = 0,
                dim: int = 0, stream=None):
        """Reverse mode of operator() (order 0) / deriv(1, ...) (order 1): writes g_spline_coef, the
        cotangents of the coefficients (a scatter-add of basis-weighted cotangents), and, when
        g_coords is given, the cotangents of the coordinates (needs spline_coef)."""
        x = _dev_f64(coords_eval, "coords_eval")
        gy = _dev_f64(g_spline_eval, "g_spline_eval")
        gc = _dev_f64(g_spline_coef, "g_spline_coef")
        c = _dev_f64(spline_coef, "spline_coef")
        gx = _dev_f64(g_coords, "g_coords")
        empty = Lines(0, 1, 0, 0, 0)
        _lib.call("ddcb_eval_adjoint", self._h, int(order), _ptr(x), lines_of(x, dim), _ptr(c),
                  lines_of(c, dim) if c is not None else empty, _ptr(gy), lines_of(gy, dim), _ptr(gc),
                  lines_of(gc, dim), _ptr(gx), lines_of(gx, dim) if gx is not None else empty, _stream_handle(stream))
        return gc

    def integrate(self, integrals, spline_coef, *, dim: int = 0, stream=None):
        """SplineEvaluator::integrate(integrals, spline_coef): integrals has the batch shape of spline_coef."""
        out = _dev_f64(integrals, "integrals")
        c = _dev_f64(spline_coef, "spline_coef")
        lc = lines_of(c, dim)
        assert out.numel() == lc.inner * lc.outer and out.is_contiguous()
        _lib.call("ddcb_integrate", self._h, _ptr(out), lc.inner, _ptr(c), lc, _stream_handle(stream))
        return out


class SplineBuilder2D:
    """ddc::SplineBuilder2D: two 1D builders applied as the reference does (spline_builder_2d.hpp:526-651).

    Data layout (x1, x2, batch...) with the batch contiguous: vals (np1, np2, *batch) ->
    spline (size1, size2, *batch).
    """

    def __init__(self, builder1: SplineBuilder, builder2: SplineBuilder):
        self.builder1, self.builder2 = builder1, builder2

    def workspace_bytes(self, nbatch: int) -> int:
        out = C.c_uint64()
        _lib.call("ddcb_build2d_workspace_bytes", self.builder1._h, self.builder2._h, int(nbatch), C.byref(out))
        return out.value

    def __call__(self, spline, vals, derivs_min1=None, derivs_max1=None, derivs_min2=None, derivs_max2=None,
                 mixed_derivs_min1_min2=None, mixed_derivs_max1_min2=None, mixed_derivs_min1_max2=None,
                 mixed_derivs_max1_max2=None, *, workspace=None, stream=None):
        spline = _dev_f64(spline, "spline")
        vals = _dev_f64(vals, "vals")
        assert spline.is_contiguous() and vals.is_contiguous()
        nbatch = vals[0, 0].numel()
        arrs = [derivs_min1, derivs_max1, derivs_min2, derivs_max2, mixed_derivs_min1_min2, mixed_derivs_max1_min2,
                mixed_derivs_min1_max2, mixed_derivs_max1_max2]
        arrs = [_dev_f64(a, "derivs") for a in arrs]
        for a in arrs:
            assert a is None or a.is_contiguous()
        ws_ptr, ws_bytes = C.c_void_p(0), 0
        if workspace is not None:
            ws_ptr, ws_bytes = C.c_void_p(workspace.data_ptr()), workspace.numel() * workspace.element_size()
        _lib.call("ddcb_build2d", self.builder1._h, self.builder2._h, _ptr(spline), _ptr(vals), *[_ptr(a) for a in arrs],
                  int(nbatch), ws_ptr, ws_bytes, _stream_handle(stream))
        return spline


class SplineEvaluator2D:
    """ddc::SplineEvaluator2D over two 1D evaluators (spline_evaluator_2d.hpp).

    coords_eval: (*points, *batch, 2) coordinate pairs; spline_coef: (size1, size2, *batch).
    """

    def __init__(self, evaluator1: SplineEvaluator, evaluator2: SplineEvaluator):
        self.evaluator1, self.evaluator2 = evaluator1, evaluator2

    def _run(self, o1, o2, spline_eval, coords_eval, spline_coef, stream):
        out = _dev_f64(spline_eval, "spline_eval")
        x = _dev_f64(coords_eval, "coords_eval")
        c = _dev_f64(spline_coef, "spline_coef")
        assert out.is_contiguous() and x.is_contiguous() and c.is_contiguous()
        nbatch = c[0, 0].numel()
        npoints = out.numel() // max(nbatch, 1)
        assert x.numel() == 2 * out.numel()
        _lib.call("ddcb_eval2d", self.evaluator1._h, self.evaluator2._h, int(o1), int(o2), _ptr(out), _ptr(x), _ptr(c),
                  int(npoints), int(nbatch), _stream_handle(stream))
        return out

    def __call__(self, spline_eval, coords_eval, spline_coef, *, stream=None):
        return self._run(0, 0, spline_eval, coords_eval, spline_coef, stream)

    def deriv_dim_1(self, spline_eval, coords_eval, spline_coef, *, stream=None):
        return self._run(1, 0, spline_eval, coords_eval, spline_coef, stream)

    def deriv_dim_2(self, spline_eval, coords_eval, spline_coef, *, stream=None):
        return self._run(0, 1, spline_eval, coords_eval, spline_coef, stream)

    def deriv_1_and_2(self, spline_eval, coords_eval, spline_coef, *, stream=None):
        return self._run(1, 1, spline_eval, coords_eval, spline_coef, stream)

    def integrate(self, integrals, spline_coef, *, stream=None):
        out = _dev_f64(integrals, "integrals")
        c = _dev_f64(spline_coef, "spline_coef")
        nbatch = c[0, 0].numel()
        assert out.numel() == nbatch and out.is_contiguous() and c.is_contiguous()
        _lib.call("ddcb_integrate2d", self.evaluator1._h, self.evaluator2._h, _ptr(out), _ptr(c), int(nbatch),
                  _stream_handle(stream))
        return out


class UnevenBatch:
    """Many independent one-line problems (own builder and evaluator each) built and evaluated by
    one graph launch (ddcb_batch_uneven_*): per group of problems a build kernel with a block per
    problem, then an evaluation kernel over the group's points. Data are packed flat CUDA float64
    arrays; `offsets()` gives every problem's slice. The builders and evaluators are kept alive by
    the batch."""

    def __init__(self, builders: Sequence[SplineBuilder], evaluators: Sequence[SplineEvaluator], nevals):
        self.builders, self.evaluators = list(builders), list(evaluators)
        n = len(self.builders)
        bh = (C.c_void_p * max(n, 1))(*[b._h.value for b in self.builders])
        eh = (C.c_void_p * max(n, 1))(*[e._h.value for e in self.evaluators])
        ne = np.ascontiguousarray(nevals, dtype=np.int64)
        h = C.c_void_p()
        _lib.call("ddcb_batch_uneven_create", C.cast(bh, C.c_void_p), C.cast(eh, C.c_void_p),
                  ne.ctypes.data_as(C.c_void_p), n, C.byref(h))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        L = getattr(_lib, "_lib", None) if _lib is not None else None
        if h and L is not None:
            L.ddcb_batch_uneven_destroy(h)
            self._h = None

    @property
    def info(self) -> UnevenInfo:
        info = UnevenInfo()
        _lib.call("ddcb_batch_uneven_get_info", self._h, C.byref(info))
        return info

    def offsets(self):
        n = len(self.builders) + 1
        keys = ("vals", "derivs_lo", "derivs_hi", "coefs", "evals")
        arrs = {k: np.zeros(n, dtype=np.int64) for k in keys}
        _lib.call("ddcb_batch_uneven_offsets", self._h, *[arrs[k].ctypes.data_as(C.c_void_p) for k in keys])
        return arrs

    def _ptrs(self, vals, derivs_lo, derivs_hi, coefs, coords, out):
        return [_ptr(_dev_f64(t, nm)) for t, nm in ((vals, "vals"), (derivs_lo, "derivs_lo"), (derivs_hi, "derivs_hi"),
                                                    (coefs, "coefs"), (coords, "coords"), (out, "out"))]

    def tune(self, vals, derivs_lo, derivs_hi, coefs, coords, out, reps: int = 3, stream=None):
        """Time the candidate schedules on these buffers and keep the fastest (returns the info)."""
        _lib.call("ddcb_batch_uneven_tune", self._h, *self._ptrs(vals, derivs_lo, derivs_hi, coefs, coords, out),
                  int(reps), _stream_handle(stream))
        return self.info

    def __call__(self, vals, derivs_lo, derivs_hi, coefs, coords, out, stream=None):
        _lib.call("ddcb_batch_uneven_run", self._h, *self._ptrs(vals, derivs_lo, derivs_hi, coefs, coords, out),
                  _stream_handle(stream))
        return out


def _host_f64(t, name):
    import torch

    if t is None:
        return None
    if not (isinstance(t, torch.Tensor) and t.device.type == "cpu" and t.dtype == torch.float64):
        raise TypeError(f"{name} must be a CPU float64 tensor (page-locked for asynchronous copies)")
    return t


class HostPipeline:
    """SplineBuilder::operator() then SplineEvaluator (order 0) or ::deriv(order) on HOST tensors
    (ddcb_host_pipeline_*): the batch runs in slices of `slice_lines` lines whose host-to-device
    copies, kernels and device-to-host copies overlap on three streams. Host tensors use the layouts
    of the device calls (interest dimension `dim`, batch in the other dimensions) with the batch
    either in rows or one contiguous line per batch index; pin them (`pin_memory()`) for
    asynchronous copies. The builder and evaluator are kept alive by the pipeline."""

    def __init__(self, builder: SplineBuilder, evaluator: SplineEvaluator, npoints: int, *, order: int = 0,
                 slice_lines: int = 8192):
        self.builder, self.evaluator = builder, evaluator
        h = C.c_void_p()
        _lib.call("ddcb_host_pipeline_create", builder._h, evaluator._h, int(order), int(npoints), int(slice_lines),
                  C.byref(h))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        L = getattr(_lib, "_lib", None) if _lib is not None else None
        if h and L is not None:
            L.ddcb_host_pipeline_destroy(h)
            self._h = None

    def __call__(self, vals, coords_eval, spline_eval, derivs_xmin=None, derivs_xmax=None, spline=None, *, dim: int = 0,
                 stream=None):
        """Reads vals / derivs / coords_eval and writes spline_eval (and spline, when given) on the
        host; the work is queued on `stream` (default: the current CUDA stream): synchronize it
        before reading the outputs."""
        vals = _host_f64(vals, "vals")
        x = _host_f64(coords_eval, "coords_eval")
        out = _host_f64(spline_eval, "spline_eval")
        dlo = _host_f64(derivs_xmin, "derivs_xmin")
        dhi = _host_f64(derivs_xmax, "derivs_xmax")
        coefs = _host_f64(spline, "spline")
        empty = Lines(0, 1, 0, 0, 0)
        _lib.call("ddcb_host_pipeline_run", self._h, _ptr(vals), lines_of(vals, dim), _ptr(dlo),
                  lines_of(dlo, dim) if dlo is not None else empty, _ptr(dhi),
                  lines_of(dhi, dim) if dhi is not None else empty, _ptr(x), lines_of(x, dim), _ptr(out),
                  lines_of(out, dim), _ptr(coefs), lines_of(coefs, dim) if coefs is not None else empty,
                  _stream_handle(stream))
        return spline_eval


class SplineBuilder3D:
    """ddc::SplineBuilder3D over three 1D builders (spline_builder_3d.hpp:597-1126).

    Data layout (x1, x2, x3, batch...) with the batch contiguous: vals (np1, np2, np3, *batch) ->
    spline (size1, size2, size3, *batch). Derivative arrays are passed by the reference's names;
    each has the rows of its derivative kind along the dimensions it names and the interpolation
    points along the others (e.g. derivs_min2: (np1, nbv_lo2, np3, *batch)).
    """

    # reference argument name -> (k1, k2, k3) with k = 0 values, 1 lower, 2 upper derivatives
    KINDS = {"derivs_min1": (1, 0, 0), "derivs_max1": (2, 0, 0), "derivs_min2": (0, 1, 0), "derivs_max2": (0, 2, 0),
             "derivs_min3": (0, 0, 1), "derivs_max3": (0, 0, 2)}
    for _a, _i in (("min", 1), ("max", 2)):
        for _b, _j in (("min", 1), ("max", 2)):
            KINDS[f"mixed_derivs_{_a}1_{_b}2"] = (_i, _j, 0)
            KINDS[f"mixed_derivs_{_a}2_{_b}3"] = (0, _i, _j)
            KINDS[f"mixed_derivs_{_a}1_{_b}3"] = (_i, 0, _j)
            for _c, _k in (("min", 1), ("max", 2)):
                KINDS[f"mixed_derivs_{_a}1_{_b}2_{_c}3"] = (_i, _j, _k)

    def __init__(self, builder1: SplineBuilder, builder2: SplineBuilder, builder3: SplineBuilder):
        self.builders = (builder1, builder2, builder3)

    def workspace_bytes(self, nbatch: int) -> int:
        out = C.c_uint64()
        _lib.call("ddcb_build3d_workspace_bytes", *[b._h for b in self.builders], int(nbatch), C.byref(out))
        return out.value

    def __call__(self, spline, vals, *, workspace=None, stream=None, **derivs):
        spline = _dev_f64(spline, "spline")
        vals = _dev_f64(vals, "vals")
        assert spline.is_contiguous() and vals.is_contiguous()
        nbatch = vals[0, 0, 0].numel()
        ptrs = (C.c_void_p * 27)()
        ptrs[0] = vals.data_ptr()
        keep = [vals]
        for name, arr in derivs.items():
            if name not in self.KINDS:
                raise TypeError(f"unknown derivative argument {name}")
            if arr is None:
                continue
            arr = _dev_f64(arr, name)
            assert arr.is_contiguous()
            k1, k2, k3 = self.KINDS[name]
            ptrs[k1 + 3 * k2 + 9 * k3] = arr.data_ptr()
            keep.append(arr)
        ws_ptr, ws_bytes = C.c_void_p(0), 0
        if workspace is not None:
            ws_ptr, ws_bytes = C.c_void_p(workspace.data_ptr()), workspace.numel() * workspace.element_size()
        _lib.call("ddcb_build3d", *[b._h for b in self.builders], _ptr(spline), C.cast(ptrs, C.c_void_p), int(nbatch),
                  ws_ptr, ws_bytes, _stream_handle(stream))
        return spline


class SplineEvaluatorND:
    """ddc::SplineEvaluatorND (spline_evaluator_nd.hpp) over N 1D evaluators (N in 1..6); with N = 3
    it is ddc::SplineEvaluator3D. coords_eval: (*points, *batch, N) coordinate tuples;
    spline_coef: (size_1, ..., size_N, *batch)."""

    def __init__(self, *evaluators: SplineEvaluator):
        if not 1 <= len(evaluators) <= 6:
            raise ValueError("1 to 6 evaluators")
        self.evaluators = tuple(evaluators)
        self.ndims = len(evaluators)
        self._handles = (C.c_void_p * self.ndims)(*[e._h.value for e in evaluators])

    def _run(self, orders, spline_eval, coords_eval, spline_coef, stream):
        out = _dev_f64(spline_eval, "spline_eval")
        x = _dev_f64(coords_eval, "coords_eval")
        c = _dev_f64(spline_coef, "spline_coef")
        assert out.is_contiguous() and x.is_contiguous() and c.is_contiguous()
        nbatch = c[(0,) * self.ndims].numel()
        npoints = out.numel() // max(nbatch, 1)
        assert x.numel() == self.ndims * out.numel()
        o = None if orders is None else (C.c_int32 * self.ndims)(*[int(v) for v in orders])
        _lib.call("ddcb_evalnd", C.cast(self._handles, C.c_void_p), self.ndims,
                  C.cast(o, C.c_void_p) if o is not None else None, _ptr(out), _ptr(x), _ptr(c), int(npoints),
                  int(nbatch), _stream_handle(stream))
        return out

    def __call__(self, spline_eval, coords_eval, spline_coef, *, stream=None):
        """operator(): values with the periodic wraps and extrapolation rules."""
        return self._run(None, spline_eval, coords_eval, spline_coef, stream)

    def deriv(self, orders, spline_eval, coords_eval, spline_coef, *, stream=None):
        """deriv(DiscreteElement<Deriv<X1>, ...>(orders...), ...): orders[d] in 0..degree_d."""
        assert len(orders) == self.ndims
        return self._run(orders, spline_eval, coords_eval, spline_coef, stream)

    def integrate(self, integrals, spline_coef, *, stream=None):
        out = _dev_f64(integrals, "integrals")
        c = _dev_f64(spline_coef, "spline_coef")
        nbatch = c[(0,) * self.ndims].numel()
        assert out.numel() == nbatch and out.is_contiguous() and c.is_contiguous()
        _lib.call("ddcb_integratend", C.cast(self._handles, C.c_void_p), self.ndims, _ptr(out), _ptr(c), int(nbatch),
                  _stream_handle(stream))
        return out


def SplineEvaluator3D(evaluator1: SplineEvaluator, evaluator2: SplineEvaluator, evaluator3: SplineEvaluator):
    """ddc::SplineEvaluator3D (spline_evaluator_3d.hpp): the N-dimensional evaluator with N = 3."""
    return SplineEvaluatorND(evaluator1, evaluator2, evaluator3)
