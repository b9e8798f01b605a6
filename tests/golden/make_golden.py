"""Generate the golden fixtures in tests/golden/splines_golden.npz.

The fixtures pin the oracle (and, through it, the CUDA path) against an implementation that does
not share code with either: scipy.interpolate.BSpline's de Boor evaluation for the basis, and
numpy's LAPACK dense solve for the interpolation system. The reference itself cannot run in this
image (no Kokkos / LAPACKE / Ginkgo), so its own output cannot be captured; these vectors restate
its mathematics:

* knots: uniform knots are a ghosted uniform grid, rmin - degree*h + k*h (bsplines_uniform.hpp:145,
  uniform_point_sampling.hpp:170-192); non-uniform knots are the breaks padded with degree copies
  of each end point (clamped) or extended by the period (bsplines_non_uniform.hpp:432-455);
* the interpolation system: one row per interpolation point, plus Hermite rows holding the
  derivatives of order odd..odd+nbe-1 at rmin / rmax (spline_builder.hpp:784-886,
  spline_builder_closures.hpp:43-55); periodic bases share coefficients j and j+nbasis;
* outputs: coefficients indexed by B-spline (with the periodic copies c[nbasis+i] = c[i],
  spline_builder.hpp:1073-1100), values and first/second derivatives at seeded in-domain points,
  and the integral over [rmin, rmax].

The interpolation points are inputs of the builder; they are stored in the fixture (computed by the
Greville rules of greville_interpolation_points.hpp, restated independently below).

Run:  python tests/golden/make_golden.py   (writes tests/golden/splines_golden.npz)
"""
from __future__ import annotations

import os

import numpy as np
from scipy.interpolate import BSpline

PERIODIC, HERMITE, HOMOGENEOUS_HERMITE, GREVILLE = 0, 1, 2, 3
HERE = os.path.dirname(os.path.abspath(__file__))


def nbe(bc, d):
    return d // 2 if bc in (HERMITE, HOMOGENEOUS_HERMITE) else 0


def knots_of(d, periodic, uniform, breaks):
    nc = len(breaks) - 1
    if uniform:
        a, b = breaks[0], breaks[-1]
        h = (b - a) / nc
        origin = a - d * h
        return origin + np.arange(nc + 1 + 2 * d) * h
    t = np.zeros(nc + 1 + 2 * d)
    t[d:d + nc + 1] = breaks
    if periodic:
        per = breaks[-1] - breaks[0]
        for i in range(1, d + 1):
            t[d - i] = t[d + nc - i] - per
            t[d + nc + i] = t[d + i] + per
    else:
        t[:d] = breaks[0]
        t[d + nc + 1:] = breaks[-1]
    return t


def greville(d, periodic, uniform, t, nc, lo, hi):
    """Interpolation points of greville_interpolation_points.hpp:47-269."""
    nbasis = nc + (0 if periodic else d)
    rmin, rmax = t[d], t[d + nc]
    n_lo, n_hi = nbe(lo, d), nbe(hi, d)
    npts = nbasis - n_lo - n_hi
    if uniform:
        shift = 0.5 if d % 2 == 0 else 0.0
        dx = (rmax - rmin) / nc
        o = rmin + shift * dx
        if periodic or (n_lo and n_hi):
            return o + np.arange(npts) * dx
        pts = np.zeros(npts)
        if lo == GREVILLE:
            for i in range(d // 2 + 1):
                s = (d - i) * rmin
                last = i + d + 1
                for k in range(last - i, last):
                    s += t[k]
                pts[i] = s / d
        else:
            pts[0] = o
        n_start = d // 2 + 1 if lo == GREVILLE else 1
        for ip in range(1, nc):
            pts[ip - 1 + n_start] = o + ip * dx
        if hi == GREVILLE:
            for i in range(d // 2 + 1):
                s = (d - i) * rmax
                first = nbasis - 1 - i + 1
                for k in range(first, first + i):
                    s += t[k]
                pts[npts - 1 - i] = s / d
        else:
            pts[npts - 1] = o + (nc - 1 + d % 2) * dx
        return pts
    g = np.array([t[ib + 1: ib + 1 + d].sum() / d for ib in range(nbasis)])
    if periodic:
        npl = 0
        temp = []
        while g[npl] < rmin:
            temp.append(g[npl] + (rmax - rmin))
            npl += 1
        g = np.concatenate([g[npl:], np.array(temp)])
        return g[:npts]
    return g[n_lo: n_lo + npts]


def basis_matrix(t, d, x, order):
    nc = len(t) - d - 1
    spl = BSpline(t, np.eye(nc), d)
    if order:
        spl = spl.derivative(order)
    return np.atleast_2d(spl(np.atleast_1d(x)))


def solve_case(d, periodic, uniform, breaks, lo, hi, vals, dlo, dhi):
    t = knots_of(d, periodic, uniform, breaks)
    nc = len(breaks) - 1
    nbasis = nc + (0 if periodic else d)
    size = nc + d
    rmin, rmax = t[d], t[d + nc]
    dx = (rmax - rmin) / nc
    odd = d % 2
    pts = greville(d, periodic, uniform, t, nc, lo, hi)
    n_lo, n_hi = nbe(lo, d), nbe(hi, d)
    rows, rhs = [], []
    for i in range(n_lo):
        rows.append(basis_matrix(t, d, rmin, i + odd)[0] * dx ** (i + odd))
        rhs.append(dlo[i] * dx ** (i + odd) if lo == HERMITE else np.zeros(vals.shape[1]))
    Bm = basis_matrix(t, d, pts, 0)
    for i in range(len(pts)):
        rows.append(Bm[i])
        rhs.append(vals[i])
    for i in range(n_hi):
        rows.append(basis_matrix(t, d, rmax, i + odd)[0] * dx ** (i + odd))
        rhs.append(dhi[i] * dx ** (i + odd) if hi == HERMITE else np.zeros(vals.shape[1]))
    A = np.array(rows)
    if periodic:
        A = A[:, :nbasis] + np.pad(A[:, nbasis:], ((0, 0), (0, nbasis - d)))
    c = np.linalg.solve(A, np.array(rhs))
    coefs = np.zeros((size, c.shape[1]))
    coefs[:nbasis] = c
    if periodic:
        coefs[nbasis:] = c[:d]
    return t, pts, coefs


def cos_family(x, k, ph, order):
    return (2 * np.pi * k) ** order * np.cos(np.pi / 2 * order + 2 * np.pi * k * x + ph)


def main():
    rng = np.random.default_rng(0xDDC0)
    cases = {}
    idx = 0
    bcs_np = [(HERMITE, HERMITE), (GREVILLE, GREVILLE), (HERMITE, GREVILLE), (GREVILLE, HERMITE),
              (HOMOGENEOUS_HERMITE, HOMOGENEOUS_HERMITE)]
    for d in range(1, 6):
        for uniform in (True, False):
            for periodic in (True, False):
                for nc in (10, 23):
                    bcs = [(PERIODIC, PERIODIC)] if periodic else bcs_np
                    for lo, hi in bcs:
                        if not periodic and nc == 23 and (lo, hi) not in bcs_np[:2]:
                            continue
                        h = 1.0 / nc
                        breaks = np.arange(nc + 1) * h
                        if not uniform:
                            breaks[1:-1] += rng.uniform(-0.3 * h, 0.3 * h, nc - 1)
                            breaks.sort()
                        B = 3
                        k = rng.integers(1, 3, B).astype(float)
                        ph = rng.uniform(0, 2 * np.pi, B)
                        t = knots_of(d, periodic, uniform, breaks)
                        pts = greville(d, periodic, uniform, t, nc, lo, hi)
                        vals = cos_family(pts[:, None], k, ph, 0)
                        odd = d % 2
                        n_lo, n_hi = nbe(lo, d), nbe(hi, d)
                        dlo = np.array([cos_family(0.0, k, ph, i + odd) for i in range(n_lo)]).reshape(n_lo, B)
                        dhi = np.array([cos_family(1.0, k, ph, i + odd) for i in range(n_hi)]).reshape(n_hi, B)
                        t, pts, coefs = solve_case(d, periodic, uniform, breaks, lo, hi, vals, dlo, dhi)
                        m = 40
                        coords = rng.uniform(0.0, 1.0, (m, B))
                        # domain ends as the basis computes them (uniform rmax can round below 1.0,
                        # and points beyond rmax take the extrapolation rule)
                        coords[0] = t[d]
                        coords[1] = t[d + nc]
                        spl = [BSpline(t, coefs[:, b], d) for b in range(B)]
                        ev = np.stack([spl[b](coords[:, b]) for b in range(B)], axis=1)
                        d1 = np.stack([spl[b].derivative(1)(coords[:, b]) for b in range(B)], axis=1)
                        d2 = np.stack([spl[b].derivative(2)(coords[:, b]) for b in range(B)], axis=1) if d >= 2 else np.zeros_like(ev)
                        integ = np.array([spl[b].integrate(t[d], t[d + nc]) for b in range(B)])
                        key = f"c{idx:03d}"
                        meta = np.array([d, int(uniform), int(periodic), nc, lo, hi], dtype=np.int64)
                        for name, arr in dict(meta=meta, breaks=breaks, knots=t, points=pts, vals=vals, dlo=dlo,
                                              dhi=dhi, coefs=coefs, coords=coords, ev=ev, d1=d1, d2=d2,
                                              integ=integ).items():
                            cases[f"{key}_{name}"] = arr
                        idx += 1
    np.savez_compressed(os.path.join(HERE, "splines_golden.npz"), ncases=np.array(idx), **cases)
    print(f"wrote {idx} cases")


if __name__ == "__main__":
    main()
