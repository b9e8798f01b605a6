"""ctypes front-end of the CPU oracle (oracle/ddc_oracle.cpp) -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may import this module. It
restates the reference's SplineBuilder / SplineEvaluator (CExA-project/ddc,
src/ddc/kernels/splines/) on the CPU so that the CUDA path can be checked against it; it is never
the thing measured or shipped.

Batched arrays use the (row, line) layout with the line index contiguous (numpy C order, shape
(rows, B)), which is DDC's (x, batch) layout_right ordering.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

PERIODIC, HERMITE, HOMOGENEOUS_HERMITE, GREVILLE = 0, 1, 2, 3
EX_PERIODIC, EX_NULL, EX_CONSTANT = 0, 1, 2

_lib = None
_dp = C.POINTER(C.c_double)
_lp = C.POINTER(C.c_long)


def build() -> str:
    """Compile the oracle with its Makefile (system g++ with OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp = C.c_void_p
        sig = {
            "orc_last_error": (C.c_char_p, []),
            "orc_bsplines_uniform": (vp, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_long]),
            "orc_bsplines_non_uniform": (vp, [C.c_int, C.c_int, _dp, C.c_long]),
            "orc_bsplines_free": (None, [vp]),
            "orc_bsplines_info": (None, [vp, _lp, _dp]),
            "orc_knot": (C.c_double, [vp, C.c_long]),
            "orc_eval_basis": (C.c_long, [vp, C.c_double, _dp]),
            "orc_eval_basis_and_n_derivs": (C.c_long, [vp, C.c_double, C.c_int, _dp]),
            "orc_integrals": (None, [vp, _dp]),
            "orc_greville": (C.c_long, [vp, C.c_int, C.c_int, _dp, C.c_long]),
            "orc_builder_create": (vp, [vp, _dp, C.c_long, C.c_int, C.c_int]),
            "orc_builder_free": (None, [vp]),
            "orc_builder_info": (None, [vp, _lp, _dp]),
            "orc_builder_structure": (C.c_long, [vp, C.c_char_p, C.c_long]),
            "orc_builder_matrix": (None, [vp, _dp]),
            "orc_build": (None, [vp, _dp, _dp, _dp, _dp, C.c_long, C.c_int]),
            "orc_solve": (None, [vp, _dp, C.c_long, C.c_int, C.c_int]),
            "orc_quadrature": (None, [vp, _dp, _dp, _dp]),
            "orc_eval": (None, [vp, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.c_long, C.c_long, C.c_int]),
            "orc_integrate": (None, [vp, _dp, _dp, C.c_long, C.c_int]),
            "orc_build2d": (None, [vp, vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, C.c_long, C.c_int]),
            "orc_eval2d": (None, [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                  _dp, _dp, _dp, _dp, C.c_long, C.c_long, C.c_int]),
            "orc_lp_create": (vp, [C.c_int, C.c_long, C.c_long, C.c_long, C.c_int, C.c_long, C.c_long]),
            "orc_lp_free": (None, [vp]),
            "orc_lp_set": (None, [vp, C.c_long, C.c_long, C.c_double]),
            "orc_lp_get": (C.c_double, [vp, C.c_long, C.c_long]),
            "orc_lp_required_rows": (C.c_long, [vp]),
            "orc_lp_setup": (C.c_int, [vp]),
            "orc_lp_solve": (None, [vp, _dp, C.c_long, C.c_int]),
            "orc_lp_describe": (C.c_long, [vp, C.c_char_p, C.c_long]),
            "orc_max_threads": (C.c_int, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _err():
    return lib().orc_last_error().decode()


def max_threads() -> int:
    return lib().orc_max_threads()


class BSplines:
    """UniformBSplines / NonUniformBSplines restatement (bsplines_uniform.hpp, bsplines_non_uniform.hpp)."""

    def __init__(self, degree, periodic, *, rmin=None, rmax=None, ncells=None, breaks=None):
        L = lib()
        if breaks is None:
            h = L.orc_bsplines_uniform(degree, int(periodic), float(rmin), float(rmax), int(ncells))
            self.uniform = True
        else:
            b = np.ascontiguousarray(breaks, dtype=np.float64)
            h = L.orc_bsplines_non_uniform(degree, int(periodic), _p(b), b.size)
            self.uniform = False
        if not h:
            raise RuntimeError(_err())
        self._h = h
        info = np.zeros(6, dtype=np.int64)
        rr = np.zeros(2)
        L.orc_bsplines_info(h, info.ctypes.data_as(_lp), _p(rr))
        self.degree, self.periodic = int(info[0]), bool(info[1])
        self.ncells, self.nbasis, self.size = int(info[3]), int(info[4]), int(info[5])
        self.rmin, self.rmax = float(rr[0]), float(rr[1])

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.orc_bsplines_free(self._h)
            self._h = None

    def knot(self, k):
        return lib().orc_knot(self._h, k)

    def eval_basis(self, x):
        v = np.zeros(self.degree + 1)
        j = lib().orc_eval_basis(self._h, float(x), _p(v))
        return j, v

    def eval_basis_and_n_derivs(self, x, n):
        out = np.zeros((self.degree + 1) * (n + 1))
        j = lib().orc_eval_basis_and_n_derivs(self._h, float(x), n, _p(out))
        return j, out.reshape(self.degree + 1, n + 1)

    def integrals(self):
        out = np.zeros(self.size)
        lib().orc_integrals(self._h, _p(out))
        return out

    def greville(self, lo, hi):
        out = np.zeros(self.nbasis + 2)
        n = lib().orc_greville(self._h, lo, hi, _p(out), out.size)
        if n < 0:
            raise RuntimeError(_err())
        return out[:n].copy()


class Builder:
    """SplineBuilder restatement (spline_builder.hpp), LAPACK solver path."""

    def __init__(self, bsplines: BSplines, points, lo, hi):
        self.bs = bsplines
        pts = np.ascontiguousarray(points, dtype=np.float64)
        h = lib().orc_builder_create(bsplines._h, _p(pts), pts.size, lo, hi)
        if not h:
            raise RuntimeError(_err())
        self._h = h
        self.points = pts
        info = np.zeros(7, dtype=np.int64)
        dx = np.zeros(1)
        lib().orc_builder_info(h, info.ctypes.data_as(_lp), _p(dx))
        (self.offset, self.nbe_lo, self.nbe_hi, self.nbv_lo, self.nbv_hi,
         self.required_rows, self.npoints) = (int(v) for v in info)
        self.dx = float(dx[0])
        self.lo, self.hi = lo, hi

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.orc_builder_free(self._h)
            self._h = None

    @property
    def structure(self) -> str:
        buf = C.create_string_buffer(256)
        lib().orc_builder_structure(self._h, buf, 256)
        return buf.value.decode()

    def matrix(self):
        n = self.bs.nbasis
        out = np.zeros((n, n))
        lib().orc_builder_matrix(self._h, _p(out))
        return out

    def __call__(self, vals, derivs_lo=None, derivs_hi=None, nthreads=None):
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        if vals.ndim == 1:
            vals = vals[:, None]
        B = vals.shape[1]
        out = np.zeros((self.bs.size, B))
        dlo = None if derivs_lo is None else np.ascontiguousarray(np.asarray(derivs_lo, dtype=np.float64).reshape(-1, B))
        dhi = None if derivs_hi is None else np.ascontiguousarray(np.asarray(derivs_hi, dtype=np.float64).reshape(-1, B))
        if self.lo == HERMITE:
            assert dlo is not None and dlo.shape == (self.nbv_lo, B)
        if self.hi == HERMITE:
            assert dhi is not None and dhi.shape == (self.nbv_hi, B)
        lib().orc_build(self._h, _p(out), _p(vals), _p(dlo), _p(dhi), B, nthreads or max_threads())
        return out

    def solve(self, rhs, transpose=False, nthreads=None):
        rhs = np.ascontiguousarray(rhs, dtype=np.float64).copy()
        lib().orc_solve(self._h, _p(rhs), rhs.shape[1], int(transpose), nthreads or max_threads())
        return rhs

    def quadrature_coefficients(self):
        qlo = np.zeros(max(self.nbv_lo, 1))
        q = np.zeros(self.bs.nbasis)
        qhi = np.zeros(max(self.nbv_hi, 1))
        lib().orc_quadrature(self._h, _p(qlo), _p(q), _p(qhi))
        n = self.bs.nbasis - self.nbv_lo - self.nbv_hi
        return qlo[: self.nbv_lo].copy(), q[:n].copy(), qhi[: self.nbv_hi].copy()


def evaluate(bs: BSplines, coords, coefs, order=None, ex_lo=EX_NULL, ex_hi=EX_NULL, nthreads=None):
    """SplineEvaluator::operator() (order None) or ::deriv(order) over (m, B) coordinates."""
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    coefs = np.ascontiguousarray(coefs, dtype=np.float64)
    m, B = coords.shape
    assert coefs.shape == (bs.size, B)
    out = np.zeros((m, B))
    o = -1 if order is None else int(order)
    lib().orc_eval(bs._h, o, ex_lo, ex_hi, _p(coords), _p(coefs), _p(out), m, B, nthreads or max_threads())
    return out


def integrate(bs: BSplines, coefs, nthreads=None):
    coefs = np.ascontiguousarray(coefs, dtype=np.float64)
    B = coefs.shape[1]
    out = np.zeros(B)
    lib().orc_integrate(bs._h, _p(coefs), _p(out), B, nthreads or max_threads())
    return out


def build2d(b1: Builder, b2: Builder, vals, derivs_min1=None, derivs_max1=None, derivs_min2=None,
            derivs_max2=None, mixed=(None, None, None, None), nthreads=None):
    """SplineBuilder2D::operator(). vals (np1, np2, B); returns (size1, size2, B)."""
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    np1, np2, B = vals.shape
    out = np.zeros((b1.bs.size, b2.bs.size, B))
    arrs = [derivs_min1, derivs_max1, derivs_min2, derivs_max2, *mixed]
    arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in arrs]
    lib().orc_build2d(b1._h, b2._h, _p(out), _p(vals), *[_p(a) for a in arrs], B, nthreads or max_threads())
    return out


def evaluate2d(bs1: BSplines, bs2: BSplines, c1, c2, coefs, orders=None,
               ex=(EX_NULL, EX_NULL, EX_NULL, EX_NULL), nthreads=None):
    """orders None: value with boundary handling; else (o1, o2) derivative orders (eval_no_bc)."""
    """SplineEvaluator2D::operator() / deriv. c1, c2: (m, B) coordinates; coefs (size1, size2, B)."""
    c1 = np.ascontiguousarray(c1, dtype=np.float64)
    c2 = np.ascontiguousarray(c2, dtype=np.float64)
    coefs = np.ascontiguousarray(coefs, dtype=np.float64)
    m, B = c1.shape
    out = np.zeros((m, B))
    o1, o2 = (-1, -1) if orders is None else orders
    lib().orc_eval2d(bs1._h, bs2._h, o1, o2, *ex, _p(c1), _p(c2), _p(coefs), _p(out), m, B,
                     nthreads or max_threads())
    return out


class LinearProblem:
    """The reference's SplinesLinearProblem classes on a user matrix (tests/splines/splines_linear_problem.cpp)."""

    KINDS = {"dense": 0, "band": 1, "pds_band": 2, "pds_tridiag": 3, "maker_band": 4,
             "block_band": 5, "periodic_band": 6, "2x2_dense": 7, "3x3_dense": 8}

    def __init__(self, kind, n, kl=0, ku=0, pds=False, bottom=0, top=0):
        h = lib().orc_lp_create(self.KINDS[kind], n, kl, ku, int(pds), bottom, top)
        if not h:
            raise RuntimeError(_err())
        self._h = h
        self.n = n

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.orc_lp_free(self._h)
            self._h = None

    def set(self, i, j, v):
        lib().orc_lp_set(self._h, i, j, float(v))

    def get(self, i, j):
        return lib().orc_lp_get(self._h, i, j)

    @property
    def required_rows(self):
        return lib().orc_lp_required_rows(self._h)

    @property
    def structure(self):
        buf = C.create_string_buffer(256)
        lib().orc_lp_describe(self._h, buf, 256)
        return buf.value.decode()

    def setup(self):
        if lib().orc_lp_setup(self._h) != 0:
            raise RuntimeError(_err())

    def solve(self, b, transpose=False):
        b = np.ascontiguousarray(b, dtype=np.float64).copy()
        lib().orc_lp_solve(self._h, _p(b), b.shape[1], int(transpose))
        return b


def _apply1(builder, arr, dlo=None, dhi=None, nthreads=None):
    """The 1D builder along axis 0 of arr (rows, *rest): returns (size, *rest)."""
    rest = arr.shape[1:]
    B = int(np.prod(rest)) if rest else 1
    flat = lambda a: None if a is None else np.ascontiguousarray(a).reshape(a.shape[0], B)
    out = builder(flat(arr), flat(dlo), flat(dhi), nthreads=nthreads)
    return out.reshape((builder.bs.size,) + tuple(rest))


def build3d(b1: Builder, b2: Builder, b3: Builder, vals, derivs=None, nthreads=None):
    """SplineBuilder3D::operator() (spline_builder_3d.hpp:934-1126), the reference's schedule: builder
    1 over the dimension-2 / dimension-3 derivative slabs and the (2, 3) mixed slabs, with the
    mixed derivatives involving dimension 1 as its Hermite data (:944-1101), builder 1 over the
    values (:1103-1110), then SplineBuilder2D over dimensions 2-3 with the results (:1112-1125),
    whose batch is (size1, batch). vals (np1, np2, np3, B); derivs maps the reference's argument
    names (derivs_min1, ..., mixed_derivs_max1_max2_max3) to arrays; returns (size1, size2, size3, B)."""
    derivs = derivs or {}
    g = lambda k: None if derivs.get(k) is None else np.ascontiguousarray(derivs[k], dtype=np.float64)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    s1 = b1.bs.size
    B = vals.shape[3]
    her = lambda b, side: (b.lo if side == "min" else b.hi) == HERMITE

    def slab(name, m1a, m1b, cond):
        if not cond:
            return None
        return _apply1(b1, g(name), g(m1a), g(m1b), nthreads)

    sd = {}
    for s2 in ("min", "max"):
        sd[f"2{s2}"] = slab(f"derivs_{s2}2", f"mixed_derivs_min1_{s2}2", f"mixed_derivs_max1_{s2}2", her(b2, s2))
        sd[f"3{s2}"] = slab(f"derivs_{s2}3", f"mixed_derivs_min1_{s2}3", f"mixed_derivs_max1_{s2}3", her(b3, s2))
    for s2 in ("min", "max"):
        for s3 in ("min", "max"):
            sd[f"23{s2}{s3}"] = slab(f"mixed_derivs_{s2}2_{s3}3", f"mixed_derivs_min1_{s2}2_{s3}3",
                                     f"mixed_derivs_max1_{s2}2_{s3}3", her(b2, s2) and her(b3, s3))
    spline1 = _apply1(b1, vals, g("derivs_min1"), g("derivs_max1"), nthreads)  # (s1, np2, np3, B)
    # dimensions (2, 3) with the batch (s1, B)
    to2d = lambda a: None if a is None else np.ascontiguousarray(np.moveaxis(a, 0, 2)).reshape(a.shape[1], a.shape[2], s1 * B)
    out = build2d(b2, b3, to2d(spline1), to2d(sd["2min"]), to2d(sd["2max"]), to2d(sd["3min"]), to2d(sd["3max"]),
                  (to2d(sd["23minmin"]), to2d(sd["23maxmin"]), to2d(sd["23minmax"]), to2d(sd["23maxmax"])), nthreads)
    out = out.reshape(b2.bs.size, b3.bs.size, s1, B)
    return np.ascontiguousarray(np.moveaxis(out, 2, 0))


def evaluatend(bss, coords, coefs, orders=None, ex=None):
    """SplineEvaluatorND: operator() (orders None; spline_evaluator_nd.hpp:636-720, periodic wraps,
    then the rule of the first non-periodic dimension outside its domain -- null: 0, constant: the
    value at that boundary with the other non-periodic coordinates clamped, the N-dimensional form
    of ConstantExtrapolationRule<DimI, DimNI>, constant_extrapolation_rule.hpp:143-193) or
    deriv(orders) (eval_no_bc, :766-825). coords (m, B, N); coefs (size_1, ..., size_N, B); ex: per
    dimension (lower, upper) rule codes. A per-point loop: for small cases."""
    N = len(bss)
    coords = np.asarray(coords, dtype=np.float64)
    m, B = coords.shape[:2]
    ex = ex or [(EX_NULL, EX_NULL)] * N
    out = np.zeros((m, B))
    for p in range(m):
        for b in range(B):
            x = [float(v) for v in coords[p, b]]
            if orders is None:
                for d, bs in enumerate(bss):
                    if bs.periodic and (x[d] < bs.rmin or x[d] > bs.rmax):
                        L = bs.rmax - bs.rmin
                        x[d] -= np.floor((x[d] - bs.rmin) / L) * L
                zero = False
                for d, bs in enumerate(bss):
                    if bs.periodic or bs.rmin <= x[d] <= bs.rmax:
                        continue
                    low = x[d] < bs.rmin
                    if ex[d][0 if low else 1] == EX_NULL:
                        zero = True
                    else:
                        x[d] = bs.rmin if low else bs.rmax
                        for e, be in enumerate(bss):
                            if e != d and not be.periodic:
                                x[e] = min(max(x[e], be.rmin), be.rmax)
                    break
                if zero:
                    continue
            jv = []
            for d, bs in enumerate(bss):
                o = 0 if orders is None else int(orders[d])
                if o == 0:
                    jv.append(bs.eval_basis(x[d]))
                else:
                    j, dv = bs.eval_basis_and_n_derivs(x[d], o)
                    jv.append((j, dv[:, o]))
            sub = coefs[tuple(slice(j, j + bs.degree + 1) for (j, _), bs in zip(jv, bss)) + (b,)]
            w = jv[0][1]
            for _, v in jv[1:]:
                w = np.multiply.outer(w, v)
            out[p, b] = float((sub * w).sum())
    return out
