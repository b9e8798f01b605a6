"""Pins the CPU oracle against the golden fixtures (scipy / numpy LAPACK, tests/golden/make_golden.py).

Error metric: max-norm relative error max|y - y_ref| / max|y_ref|, as in
tests/splines/non_periodic_spline_builder.cpp:298-301 of the reference.
"""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "splines_golden.npz")


def load_cases():
    z = np.load(GOLDEN)
    n = int(z["ncases"])
    out = []
    for i in range(n):
        k = f"c{i:03d}"
        out.append({name: z[f"{k}_{name}"] for name in
                    ("meta", "breaks", "knots", "points", "vals", "dlo", "dhi", "coefs", "coords", "ev", "d1", "d2",
                     "integ")})
    return out


CASES = load_cases()


def relerr(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def make_oracle(O, c):
    d, uniform, periodic, nc, lo, hi = (int(v) for v in c["meta"])
    if uniform:
        bs = O.BSplines(d, periodic, rmin=c["breaks"][0], rmax=c["breaks"][-1], ncells=nc)
    else:
        bs = O.BSplines(d, periodic, breaks=c["breaks"])
    return bs, O.Builder(bs, c["points"], lo, hi)


@pytest.mark.parametrize("i", range(len(CASES)))
def test_oracle_matches_golden(oracle_mod, i):
    O = oracle_mod
    c = CASES[i]
    d, uniform, periodic, nc, lo, hi = (int(v) for v in c["meta"])
    bs, b = make_oracle(O, c)
    knots = np.array([bs.knot(k) for k in range(len(c["knots"]))])
    assert np.allclose(knots, c["knots"], rtol=0, atol=1e-15)
    pts = bs.greville(lo, hi)
    np.testing.assert_allclose(pts, c["points"], rtol=0, atol=1e-15)
    coefs = b(c["vals"], c["dlo"] if lo == O.HERMITE else None, c["dhi"] if hi == O.HERMITE else None)
    # Two backward-stable FP64 solves agree to about cond(A)*eps; the uniform quintic Greville
    # systems have cond ~1.4e3, so the bound is 1e-12 or 10*cond*eps, whichever is larger.
    tol = max(1e-12, 10 * np.linalg.cond(b.matrix()) * np.finfo(float).eps)
    assert relerr(coefs, c["coefs"]) < tol
    ev = O.evaluate(bs, c["coords"], coefs)
    assert relerr(ev, c["ev"]) < tol
    d1 = O.evaluate(bs, c["coords"], coefs, order=1)
    assert relerr(d1, c["d1"]) < tol
    if d >= 2:
        d2 = O.evaluate(bs, c["coords"], coefs, order=2)
        assert relerr(d2, c["d2"]) < 10 * tol
    integ = O.integrate(bs, coefs)
    # integrals of full-period cosines vanish: scale by the coefficient magnitude times the length
    scale = np.abs(c["coefs"]).max() * (c["breaks"][-1] - c["breaks"][0])
    assert np.abs(integ - c["integ"]).max() / scale < 1e-13
