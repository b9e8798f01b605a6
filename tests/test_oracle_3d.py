"""The oracle's 3D builder and N-dimensional evaluator (test infrastructure) against known answers:
a separable sample set gives the tensor product of the 1D coefficient vectors, and a tensor-product
polynomial of degree <= d in each dimension is reproduced with its derivatives and integral
(the 3D form of tests/splines/non_periodic_spline_builder.cpp:297-301)."""
import numpy as np
import pytest

H, G, P = 1, 3, 0


def poly1(c, x, der=0):
    x = np.asarray(x, dtype=float)
    out = np.zeros_like(x)
    for i in range(der, len(c)):
        f = 1.0
        for k in range(der):
            f *= i - k
        out = out + c[i] * f * x ** (i - der)
    return out


def _dims(O):
    specs = [(3, P), (4, H), (5, G)]
    out = []
    for d, (deg, cl) in enumerate(specs):
        if cl == P:
            bs = O.BSplines(deg, True, rmin=0.0, rmax=1.0, ncells=9)
        else:
            br = np.linspace(0.0, 1.0, 8 + d)
            br[1:-1] += np.random.default_rng(d).uniform(-0.2, 0.2, br.size - 2) / br.size
            bs = O.BSplines(deg, False, breaks=br)
        pts = bs.greville(cl, cl)
        out.append((bs, O.Builder(bs, pts, cl, cl), pts, cl))
    return out


def test_build3d_separable_is_tensor_product(oracle_mod):
    O = oracle_mod
    dims = _dims(O)
    rng = np.random.default_rng(7)
    f = [rng.standard_normal(pts.size) for _, _, pts, _ in dims]
    d_lo = [rng.standard_normal(b.nbv_lo) if cl == H else None for _, b, _, cl in dims]
    d_hi = [rng.standard_normal(b.nbv_hi) if cl == H else None for _, b, _, cl in dims]
    c1d = [b(fi[:, None], None if lo is None else lo[:, None], None if hi is None else hi[:, None])[:, 0]
           for (_, b, _, _), fi, lo, hi in zip(dims, f, d_lo, d_hi)]
    # kinds along each dimension: values, lower and upper derivatives
    rows = [[f[d], d_lo[d], d_hi[d]] for d in range(3)]
    vals = np.einsum("i,j,k->ijk", rows[0][0], rows[1][0], rows[2][0])[..., None]
    names = {}
    for k1, a in ((1, "min1"), (2, "max1"), (0, None)):
        for k2, b_ in ((1, "min2"), (2, "max2"), (0, None)):
            for k3, c in ((1, "min3"), (2, "max3"), (0, None)):
                parts = [p for p in (a, b_, c) if p]
                if not parts:
                    continue
                r = [rows[0][k1], rows[1][k2], rows[2][k3]]
                if any(x is None for x in r):
                    continue
                key = ("derivs_" if len(parts) == 1 else "mixed_derivs_") + "_".join(parts)
                names[key] = np.einsum("i,j,k->ijk", *r)[..., None]
    got = O.build3d(dims[0][1], dims[1][1], dims[2][1], vals, names)[..., 0]
    want = np.einsum("i,j,k->ijk", *c1d)
    assert np.abs(got - want).max() / np.abs(want).max() <= 1e-13


def test_polynomial_3d_reproduced(oracle_mod):
    O = oracle_mod
    specs = [(2, G), (3, H), (4, H)]
    dims = []
    for d, (deg, cl) in enumerate(specs):
        bs = O.BSplines(deg, False, rmin=0.0, rmax=1.0, ncells=6 + d)
        pts = bs.greville(cl, cl)
        dims.append((bs, O.Builder(bs, pts, cl, cl), pts, cl, deg))
    rng = np.random.default_rng(11)
    cs = [rng.uniform(0.5, 1.0, deg + 1) for *_, deg in dims]

    def kind_rows(d, k):
        bs, b, pts, cl, deg = dims[d]
        odd = deg % 2
        if k == 0:
            return poly1(cs[d], pts)
        n = b.nbv_lo if k == 1 else b.nbv_hi
        if cl != H or n == 0:
            return None
        x = 0.0 if k == 1 else 1.0
        return np.array([poly1(cs[d], x, i + odd) for i in range(n)])

    vals = np.einsum("i,j,k->ijk", kind_rows(0, 0), kind_rows(1, 0), kind_rows(2, 0))[..., None]
    derivs = {}
    lab = {1: "min", 2: "max"}
    for k1 in range(3):
        for k2 in range(3):
            for k3 in range(3):
                if (k1, k2, k3) == (0, 0, 0):
                    continue
                r = [kind_rows(0, k1), kind_rows(1, k2), kind_rows(2, k3)]
                if any(x is None for x in r):
                    continue
                parts = [f"{lab[k]}{d + 1}" for d, k in enumerate((k1, k2, k3)) if k]
                key = ("derivs_" if len(parts) == 1 else "mixed_derivs_") + "_".join(parts)
                derivs[key] = np.einsum("i,j,k->ijk", *r)[..., None]
    c = O.build3d(dims[0][1], dims[1][1], dims[2][1], vals, derivs)
    x = rng.uniform(0.0, 1.0, (40, 1, 3))
    exact = lambda o: np.prod([poly1(cs[d], x[:, 0, d], o[d]) for d in range(3)], axis=0)
    bss = [d[0] for d in dims]
    y = O.evaluatend(bss, x, c)[:, 0]
    assert np.abs(y - exact((0, 0, 0))).max() / np.abs(exact((0, 0, 0))).max() <= 1e-13
    for o in ((1, 0, 0), (0, 2, 1), (1, 1, 1)):
        y = O.evaluatend(bss, x, c, orders=o)[:, 0]
        assert np.abs(y - exact(o)).max() / np.abs(exact(o)).max() <= 1e-10
