"""The reference's own known-answer tests for the spline path, restated against the CPU oracle.

Each test names the reference test it restates (tests/splines/*.cpp of CExA-project/ddc). The
reference ships no golden data files; its tests pin results against analytic answers, and those
answers are what is checked here.
"""
import numpy as np
import pytest

P, H, HH, G = 0, 1, 2, 3


def cos_eval(x, c0=1.0, c1=0.0, deriv=0):
    """tests/splines/cosine_evaluator.hpp:12-82."""
    return (2 * np.pi * c0) ** deriv * np.cos(np.pi / 2 * deriv + 2 * np.pi * (c0 * x + c1))


TIKHOMIROV = [1 / 2, 1 / 8, 1 / 24, 5 / 384, 1 / 240, 61 / 46080, 17 / 40320, 277 / 2064384, 31 / 725760,
              50521 / 3715891200]


def tikhomirov(h, degree, max_norm):
    """tests/splines/spline_error_bounds.hpp:34-39."""
    degree = min(degree, 9)
    return TIKHOMIROV[degree] * h ** (degree + 1) * max_norm


# --- tests/splines/bsplines.cpp:67-136: partition of unity -------------------------------------
@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("ncells", [10, 20, 100])
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("uniform", [True, False])
def test_partition_of_unity(oracle_mod, degree, ncells, periodic, uniform):
    O = oracle_mod
    xmin, xmax = 0.0, 0.2
    if uniform:
        bs = O.BSplines(degree, periodic, rmin=xmin, rmax=xmax, ncells=ncells)
    else:
        bs = O.BSplines(degree, periodic, breaks=xmin + np.arange(ncells + 1) * (xmax - xmin) / ncells)
    n = ncells * 30
    dx = (xmax - xmin) / (n - 1)
    for i in range(n):
        _, v = bs.eval_basis(xmin + dx * i)
        assert abs(v.sum() - 1.0) <= 1e-15


# --- tests/splines/bsplines.cpp:168-216: rounding at the domain ends ----------------------------
@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("ncells", [10, 20, 100])
@pytest.mark.parametrize("uniform", [True, False])
def test_rounding_at_ends(oracle_mod, degree, ncells, uniform):
    O = oracle_mod
    xmin, xmax = 0.0, 0.2
    if uniform:
        bs = O.BSplines(degree, False, rmin=xmin, rmax=xmax, ncells=ncells)
    else:
        bs = O.BSplines(degree, False, breaks=xmin + np.arange(ncells + 1) * (xmax - xmin) / ncells)
    eps = np.finfo(float).eps
    j, _ = bs.eval_basis(xmin - eps)
    assert j == 0
    j, _ = bs.eval_basis(xmax + eps)
    assert j == bs.size - 1 - degree


# --- tests/splines/splines_linear_problem.cpp:49-472: A * A^-1 = I for every solver ------------
def nonsym_matrix(lp, N, k):
    for i in range(N):
        lp.set(i, i, 3.0 / 4 * ((N + 1) * i + 1))
        for j in range(max(0, i - k), i):
            lp.set(i, j, -(1.0 / 4) / k * (N * i + j + 1))
        for j in range(i + 1, min(N, i + k + 1)):
            lp.set(i, j, -(1.0 / 4) / k * (N * i + j + 1))


def pds_matrix(lp, N, k):
    for i in range(N):
        lp.set(i, i, 2.0 * k + 1)
        for j in range(max(0, i - k), i):
            lp.set(i, j, -1.0)
        for j in range(i + 1, min(N, i + k + 1)):
            lp.set(i, j, -1.0)


def solve_and_validate(lp):
    N = lp.n
    A = np.array([[lp.get(i, j) for j in range(N)] for i in range(N)])
    lp.setup()
    rows = lp.required_rows
    inv = np.zeros((rows, N))
    inv[:N] = np.eye(N)
    inv = lp.solve(inv, transpose=False)[:N]
    inv_tr = np.zeros((rows, N))
    inv_tr[:N] = np.eye(N)
    inv_tr = lp.solve(inv_tr, transpose=True)[:N]
    np.testing.assert_allclose(A @ inv, np.eye(N), atol=1e-10)
    np.testing.assert_allclose(A @ inv_tr.T, np.eye(N), atol=1e-10)


def test_lp_dense(oracle_mod):
    lp = oracle_mod.LinearProblem("dense", 10)
    nonsym_matrix(lp, 10, 10)
    solve_and_validate(lp)


def test_lp_band(oracle_mod):
    lp = oracle_mod.LinearProblem("band", 10, kl=3, ku=3)
    nonsym_matrix(lp, 10, 3)
    solve_and_validate(lp)


def test_lp_pds_band(oracle_mod):
    lp = oracle_mod.LinearProblem("pds_band", 10, kl=3)
    pds_matrix(lp, 10, 3)
    solve_and_validate(lp)


def test_lp_pds_tridiag(oracle_mod):
    lp = oracle_mod.LinearProblem("pds_tridiag", 10)
    pds_matrix(lp, 10, 1)
    solve_and_validate(lp)


def test_lp_2x2_blocks(oracle_mod):
    lp = oracle_mod.LinearProblem("2x2_dense", 10, bottom=3)
    nonsym_matrix(lp, 10, 10)
    solve_and_validate(lp)


def test_lp_3x3_blocks(oracle_mod):
    lp = oracle_mod.LinearProblem("3x3_dense", 10, bottom=3, top=2)
    nonsym_matrix(lp, 10, 10)
    solve_and_validate(lp)


SIZES = [(N, k) for N in (10, 20) for k in range(1, 7)]


@pytest.mark.parametrize("N,k", SIZES)
def test_lp_sizes_nonsymmetric(oracle_mod, N, k):
    lp = oracle_mod.LinearProblem("maker_band", N, kl=k, ku=k, pds=False)
    nonsym_matrix(lp, N, k)
    solve_and_validate(lp)


@pytest.mark.parametrize("N,k", SIZES)
def test_lp_sizes_pds(oracle_mod, N, k):
    lp = oracle_mod.LinearProblem("maker_band", N, kl=k, ku=k, pds=True)
    pds_matrix(lp, N, k)
    solve_and_validate(lp)


@pytest.mark.parametrize("N,k", SIZES)
def test_lp_sizes_offset_banded(oracle_mod, N, k):
    lp = oracle_mod.LinearProblem("maker_band", N, kl=0, ku=2 * k, pds=True)
    for i in range(N):
        for j in range(i, min(N, i + k)):
            lp.set(i, i, -1.0)
        if i + k < N:
            lp.set(i, i + k, 2.0 * k + 1)
    solve_and_validate(lp)


@pytest.mark.parametrize("N,k", SIZES)
def test_lp_sizes_2x2(oracle_mod, N, k):
    lp = oracle_mod.LinearProblem("block_band", N, kl=k, ku=k, pds=False, bottom=3)
    nonsym_matrix(lp, N, k)
    solve_and_validate(lp)


@pytest.mark.parametrize("N,k", SIZES)
def test_lp_sizes_3x3(oracle_mod, N, k):
    lp = oracle_mod.LinearProblem("block_band", N, kl=k, ku=k, pds=False, bottom=3, top=2)
    nonsym_matrix(lp, N, k)
    solve_and_validate(lp)


@pytest.mark.parametrize("N,k", SIZES)
def test_lp_sizes_periodic_band(oracle_mod, N, k):
    for s in range(-k + k // 2 + 1, k - k // 2):
        lp = oracle_mod.LinearProblem("periodic_band", N, kl=k - s, ku=k + s, pds=False)
        for i in range(N):
            for j in range(N):
                diag = (j - i) % N
                if diag == s or diag == N + s:
                    lp.set(i, j, 2.0 * k + 1)
                elif diag <= s + k or diag >= N + s - k:
                    lp.set(i, j, -1.0)
        solve_and_validate(lp)


# --- builder + evaluator identity / error bounds -----------------------------------------------
# tests/splines/non_periodic_spline_builder.cpp:75-317 and periodic_spline_builder.cpp
def make_basis(O, degree, periodic, uniform, ncells, x0=0.0, xN=1.0):
    if uniform:
        return O.BSplines(degree, periodic, rmin=x0, rmax=xN, ncells=ncells)
    return O.BSplines(degree, periodic, breaks=x0 + np.arange(ncells + 1) * (xN - x0) / ncells)


NP_BCS = [(H, H), (G, G), (H, G), (G, H)]


@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("uniform", [True, False])
@pytest.mark.parametrize("bcs", NP_BCS)
def test_non_periodic_polynomial_exactness(oracle_mod, degree, uniform, bcs):
    """non_periodic_spline_builder.cpp:297-301 (PolynomialEvaluator, relative errors)."""
    O = oracle_mod
    lo, hi = bcs
    bs = make_basis(O, degree, False, uniform, 10)
    pts = bs.greville(lo, hi)
    b = O.Builder(bs, pts, lo, hi)
    rng = np.random.default_rng(1234 + degree)
    coeffs = rng.uniform(0, 1, degree + 1)

    def poly(x, der=0):
        res = np.zeros_like(np.asarray(x, dtype=float))
        for i in range(max(der, 0), degree + 1):
            ff = 1.0
            if der >= 0:
                for kk in range(der):
                    ff *= i - kk
            else:
                for kk in range(-1, der - 1, -1):
                    ff /= i - kk
            res = res + coeffs[i] * ff * np.power(x, i - der)
        return res

    odd = degree % 2
    vals = poly(pts)[:, None]
    dlo = np.array([poly(0.0, i + odd) for i in range(b.nbv_lo)]).reshape(b.nbv_lo, 1) if lo == H else None
    dhi = np.array([poly(1.0, i + odd) for i in range(b.nbv_hi)]).reshape(b.nbv_hi, 1) if hi == H else None
    c = b(vals, dlo, dhi)
    ev = O.evaluate(bs, pts[:, None], c)
    d1 = O.evaluate(bs, pts[:, None], c, order=1)
    integ = O.integrate(bs, c)[0]
    qlo, q, qhi = b.quadrature_coefficients()
    qint = q @ vals[:, 0]
    if lo == H:
        qint += qlo @ dlo[:, 0]
    if hi == H:
        qint += qhi @ dhi[:, 0]
    xn = 1.0
    max_norm = abs(poly(xn))
    max_norm_diff = abs(poly(xn, 1))
    max_norm_int = abs(poly(xn, -1))
    exact_int = poly(1.0, -1) - poly(0.0, -1)
    assert np.abs(ev[:, 0] - vals[:, 0]).max() / max_norm <= 1e-14
    assert np.abs(d1[:, 0] - poly(pts, 1)).max() / max_norm_diff <= 1e-11
    assert abs(integ - exact_int) / max_norm_int <= 1e-14
    assert abs(qint - exact_int) / max_norm_int <= 1e-14


@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("uniform", [True, False])
@pytest.mark.parametrize("bcs", NP_BCS + [(P, P)])
def test_cosine_error_bounds(oracle_mod, degree, uniform, bcs):
    """non_periodic_spline_builder.cpp:303-316 / periodic_spline_builder.cpp (CosineEvaluator)."""
    O = oracle_mod
    lo, hi = bcs
    periodic = lo == P
    ncells = 10
    bs = make_basis(O, degree, periodic, uniform, ncells)
    pts = bs.greville(lo, hi)
    b = O.Builder(bs, pts, lo, hi)
    odd = degree % 2
    vals = cos_eval(pts)[:, None]
    dlo = np.array([cos_eval(0.0, deriv=i + odd) for i in range(b.nbv_lo)]).reshape(b.nbv_lo, 1) if lo == H else None
    dhi = np.array([cos_eval(1.0, deriv=i + odd) for i in range(b.nbv_hi)]).reshape(b.nbv_hi, 1) if hi == H else None
    c = b(vals, dlo, dhi)
    ev = O.evaluate(bs, pts[:, None], c)
    d1 = O.evaluate(bs, pts[:, None], c, order=1)
    integ = O.integrate(bs, c)[0]
    h = 1.0 / ncells
    max_norm = 1.0
    max_norm_diff = 2 * np.pi
    max_norm_int = 1.0 / (2 * np.pi)
    err = np.abs(ev[:, 0] - vals[:, 0]).max()
    err_d = np.abs(d1[:, 0] - cos_eval(pts, deriv=1)).max()
    assert err <= max(tikhomirov(h, degree, (2 * np.pi) ** (degree + 1)), 1e-14 * max_norm)
    assert err_d <= max(tikhomirov(h, degree - 1, (2 * np.pi) ** (degree + 1)), 1e-12 * max_norm_diff)
    assert abs(integ - 0.0) <= max(tikhomirov(h, degree + 1, (2 * np.pi) ** (degree + 1)), 1e-14 * max_norm_int)


@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("uniform", [True, False])
def test_periodicity(oracle_mod, degree, uniform):
    """periodicity_spline_builder.cpp:178-205: f(x+1.5) = -f(x) for cos(2 pi x)."""
    O = oracle_mod
    bs = make_basis(O, degree, True, uniform, 10)
    pts = bs.greville(P, P)
    b = O.Builder(bs, pts, P, P)
    c = b(cos_eval(pts)[:, None])
    x = pts[:, None] + 1.5
    ev = O.evaluate(bs, x, c)
    h = 0.1
    bound = max(tikhomirov(h, degree, (2 * np.pi) ** (degree + 1)), 1e-14)
    assert np.abs(ev[:, 0] + cos_eval(pts)).max() <= bound


def test_grid_validation(oracle_mod):
    """tests/splines/spline_builder.cpp:36-135: wrong point counts and overconstrained cells throw."""
    O = oracle_mod
    bs = O.BSplines(3, False, rmin=0.0, rmax=1.0, ncells=10)
    pts = bs.greville(G, G)
    with pytest.raises(RuntimeError, match="Incorrect number of points"):
        O.Builder(bs, pts[:-1], G, G)
    bad = pts.copy()
    bad[1:6] = np.linspace(0.01, 0.05, 5)
    with pytest.raises(RuntimeError, match="overconstrained"):
        O.Builder(bs, np.sort(bad), G, G)


@pytest.mark.parametrize("rule", [1, 2])
def test_extrapolation_rules(oracle_mod, rule):
    """extrapolation_rule.cpp: null returns 0, constant returns the boundary value."""
    O = oracle_mod
    bs = O.BSplines(3, False, rmin=0.0, rmax=1.0, ncells=10)
    pts = bs.greville(G, G)
    b = O.Builder(bs, pts, G, G)
    c = b(cos_eval(pts)[:, None])
    x = np.array([[-0.5], [1.5]])
    ev = O.evaluate(bs, x, c, ex_lo=rule, ex_hi=rule)
    if rule == O.EX_NULL:
        assert ev[0, 0] == 0.0 and ev[1, 0] == 0.0
    else:
        edge = O.evaluate(bs, np.array([[bs.rmin], [bs.rmax]]), c)
        assert abs(ev[0, 0] - edge[0, 0]) <= 1e-14 and abs(ev[1, 0] - edge[1, 0]) <= 1e-14


def test_scipy_lapack_factorisations_agree(oracle_mod):
    """The oracle's factorisations restate LAPACK; cross-check a band solve against scipy's dgbsv."""
    from scipy.linalg import solve_banded

    O = oracle_mod
    N, k = 20, 3
    lp = O.LinearProblem("band", N, kl=k, ku=k)
    nonsym_matrix(lp, N, k)
    A = np.array([[lp.get(i, j) for j in range(N)] for i in range(N)])
    ab = np.zeros((2 * k + 1, N))
    for i in range(N):
        for j in range(max(0, i - k), min(N, i + k + 1)):
            ab[k + i - j, j] = A[i, j]
    rhs = np.random.default_rng(0).standard_normal((N, 4))
    ref = solve_banded((k, k), ab, rhs)
    lp.setup()
    np.testing.assert_allclose(lp.solve(rhs), ref, rtol=1e-13, atol=1e-13)
