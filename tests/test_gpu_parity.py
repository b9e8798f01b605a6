"""CUDA path vs the CPU oracle (and the golden fixtures), through the C-ABI.

Tolerance: the max-norm relative error of every output is <= 1e-12 (BASELINE's FP64 bound), or
10*cond(A)*eps for the few ill-conditioned small systems of the fixtures (two backward-stable FP64
solves agree to about cond(A)*eps).
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "splines_golden.npz")


def relerr(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


@pytest.fixture(scope="module")
def D():
    import ddc_b200

    ddc_b200.load_library()
    assert torch.cuda.is_available()
    return ddc_b200


def load_cases():
    z = np.load(GOLDEN)
    out = []
    for i in range(int(z["ncases"])):
        k = f"c{i:03d}"
        out.append({n: z[f"{k}_{n}"] for n in ("meta", "breaks", "points", "vals", "dlo", "dhi", "coefs", "coords",
                                               "ev", "d1", "d2", "integ")})
    return out


CASES = load_cases()


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def make_both(D, O, c):
    d, uniform, periodic, nc, lo, hi = (int(v) for v in c["meta"])
    if uniform:
        bs = D.UniformBSplines(d, periodic, c["breaks"][0], c["breaks"][-1], nc)
        obs = O.BSplines(d, periodic, rmin=c["breaks"][0], rmax=c["breaks"][-1], ncells=nc)
    else:
        bs = D.NonUniformBSplines(d, periodic, c["breaks"])
        obs = O.BSplines(d, periodic, breaks=c["breaks"])
    return bs, obs


@pytest.mark.parametrize("i", range(len(CASES)))
def test_golden_case(D, oracle_mod, i):
    O = oracle_mod
    c = CASES[i]
    d, uniform, periodic, nc, lo, hi = (int(v) for v in c["meta"])
    bs, obs = make_both(D, O, c)
    builder = D.SplineBuilder(bs, c["points"], lo, hi)
    ob = O.Builder(obs, c["points"], lo, hi)
    tol = max(1e-12, 10 * np.linalg.cond(ob.matrix()) * np.finfo(float).eps)
    dlo = c["dlo"] if lo == O.HERMITE else None
    dhi = c["dhi"] if hi == O.HERMITE else None
    ref = ob(c["vals"], dlo, dhi)
    B = c["vals"].shape[1]
    coefs = torch.zeros((bs.size, B), dtype=torch.float64, device="cuda")
    builder(coefs, cuda(c["vals"]), None if dlo is None else cuda(dlo), None if dhi is None else cuda(dhi))
    got = coefs.cpu().numpy()
    assert relerr(got, ref) <= tol
    assert relerr(got, c["coefs"]) <= tol
    ev = D.SplineEvaluator(bs)
    out = torch.zeros(c["coords"].shape, dtype=torch.float64, device="cuda")
    ev(out, cuda(c["coords"]), coefs)
    assert relerr(out.cpu().numpy(), O.evaluate(obs, c["coords"], ref)) <= tol
    for order in range(1, min(d, 2) + 1):
        ev.deriv(order, out, cuda(c["coords"]), coefs)
        assert relerr(out.cpu().numpy(), O.evaluate(obs, c["coords"], ref, order=order)) <= 10 * tol
    integ = torch.zeros(B, dtype=torch.float64, device="cuda")
    ev.integrate(integ, coefs)
    scale = np.abs(ref).max() * (c["breaks"][-1] - c["breaks"][0])
    assert np.abs(integ.cpu().numpy() - O.integrate(obs, ref)).max() / scale <= 1e-13


def test_config1_build_eval(D, oracle_mod):
    """Periodic uniform cubic, 1000 cells x 1000 lines, evaluation at 1000 points per line."""
    from ddc_b200 import workloads

    O = oracle_mod
    w = workloads.config1()
    bs = D.UniformBSplines(3, True, 0.0, 1.0, 1000)
    obs = O.BSplines(3, True, rmin=0.0, rmax=1.0, ncells=1000)
    pts = D.greville_points(bs, 0, 0)
    np.testing.assert_array_equal(pts, obs.greville(0, 0))
    builder = D.SplineBuilder(bs, pts, 0, 0)
    ob = O.Builder(obs, pts, 0, 0)
    ref = ob(w["vals"])
    coefs = torch.zeros((bs.size, 1000), dtype=torch.float64, device="cuda")
    builder(coefs, cuda(w["vals"]))
    ec = relerr(coefs.cpu().numpy(), ref)
    ev = D.SplineEvaluator(bs)
    out = torch.zeros_like(cuda(w["coords"]))
    ev(out, cuda(w["coords"]), coefs)
    ey = relerr(out.cpu().numpy(), O.evaluate(obs, w["coords"], ref))
    print(f"PARITY config1 coefs={ec:.2e} values={ey:.2e}")
    assert ec <= 1e-12 and ey <= 1e-12


def test_config2_reduced_batch(D, oracle_mod):
    """Non-uniform quintic Hermite, 1024 cells, first-derivative evaluation, 384 lines (ragged tile)."""
    from ddc_b200 import workloads

    O = oracle_mod
    br = workloads.config2_breaks()
    bs = D.NonUniformBSplines(5, False, br)
    obs = O.BSplines(5, False, breaks=br)
    pts = D.greville_points(bs, 1, 1)
    np.testing.assert_array_equal(pts, obs.greville(1, 1))
    w = workloads.config2(B=387, points=pts)
    builder = D.SplineBuilder(bs, pts, 1, 1)
    ob = O.Builder(obs, pts, 1, 1)
    ref = ob(w["vals"], w["dlo"], w["dhi"])
    coefs = torch.zeros((bs.size, 387), dtype=torch.float64, device="cuda")
    builder(coefs, cuda(w["vals"]), cuda(w["dlo"]), cuda(w["dhi"]))
    ec = relerr(coefs.cpu().numpy(), ref)
    ev = D.SplineEvaluator(bs)
    out = torch.zeros_like(cuda(w["coords"]))
    ev.deriv(1, out, cuda(w["coords"]), coefs)
    ed = relerr(out.cpu().numpy(), O.evaluate(obs, w["coords"], ref, order=1))
    print(f"PARITY config2 coefs={ec:.2e} d/dx={ed:.2e}")
    assert ec <= 1e-12 and ed <= 1e-12


@pytest.mark.parametrize("layout", ["XB", "BX", "B1XB2"])
def test_layouts(D, oracle_mod, layout):
    """Interest dimension first, last and in the middle (batched_spline_builder.cpp:393-515)."""
    O = oracle_mod
    br = np.linspace(0.0, 1.0, 42)
    br[1:-1] += np.random.default_rng(1).uniform(-0.006, 0.006, 40)
    bs = D.NonUniformBSplines(3, True, br)
    obs = O.BSplines(3, True, breaks=br)
    pts = D.greville_points(bs, 0, 0)
    builder = D.SplineBuilder(bs, pts, 0, 0)
    ob = O.Builder(obs, pts, 0, 0)
    rng = np.random.default_rng(7)
    nb1, nb2 = 5, 7
    vals = rng.standard_normal((pts.size, nb1 * nb2))
    ref = ob(vals)
    if layout == "XB":
        v, dim, shape_c = vals.reshape(pts.size, nb1, nb2), 0, (bs.size, nb1, nb2)
    elif layout == "BX":
        v, dim, shape_c = vals.T.reshape(nb1, nb2, pts.size), 2, (nb1, nb2, bs.size)
    else:
        v, dim, shape_c = vals.reshape(pts.size, nb1, nb2).transpose(1, 0, 2), 1, (nb1, bs.size, nb2)
    coefs = torch.zeros(shape_c, dtype=torch.float64, device="cuda")
    builder(coefs, cuda(v), dim=dim)
    got = coefs.cpu().numpy()
    if layout == "BX":
        got = got.reshape(nb1 * nb2, bs.size).T
    elif layout == "B1XB2":
        got = got.transpose(1, 0, 2).reshape(bs.size, nb1 * nb2)
    else:
        got = got.reshape(bs.size, nb1 * nb2)
    assert relerr(got, ref) <= 1e-12


@pytest.mark.parametrize("transpose", [False, True])
@pytest.mark.parametrize("degree,uniform,periodic", [(3, True, True), (5, False, False), (4, False, True), (2, True, False)])
def test_solve_multirhs_inverse(D, oracle_mod, degree, uniform, periodic, transpose):
    """A * A^-1 = I and A * A^-T^T = I at TOL 1e-10 (splines_linear_problem.cpp:49-142)."""
    O = oracle_mod
    lo = hi = 0 if periodic else 3
    if uniform:
        bs = D.UniformBSplines(degree, periodic, 0.0, 1.0, 40)
        obs = O.BSplines(degree, periodic, rmin=0.0, rmax=1.0, ncells=40)
    else:
        br = np.linspace(0, 1, 41)
        br[1:-1] += np.random.default_rng(3).uniform(-0.008, 0.008, 39)
        bs = D.NonUniformBSplines(degree, periodic, br)
        obs = O.BSplines(degree, periodic, breaks=br)
    pts = D.greville_points(bs, lo, hi)
    builder = D.SplineBuilder(bs, pts, lo, hi)
    A = O.Builder(obs, pts, lo, hi).matrix()
    n = A.shape[0]
    X = torch.eye(n, dtype=torch.float64, device="cuda").contiguous()
    builder.solve(X, transpose=transpose)
    Xn = X.cpu().numpy()
    I = A @ Xn if not transpose else A.T @ Xn
    np.testing.assert_allclose(I, np.eye(n), atol=1e-10)


@pytest.mark.parametrize("case", ["c1", "c2", "np_cubic_greville", "per_quartic_nonuniform"])
def test_fused_build_eval_matches_two_calls(D, oracle_mod, case):
    """ddcb_build_eval gives the same coefficients and values as ddcb_build + ddcb_eval(_deriv)."""
    from ddc_b200 import workloads

    O = oracle_mod
    rng = np.random.default_rng(11)
    if case == "c1":
        bs, lo, order, B = D.UniformBSplines(3, True, 0.0, 1.0, 1000), 0, 0, 203
    elif case == "c2":
        bs, lo, order, B = D.NonUniformBSplines(5, False, workloads.config2_breaks()), 1, 1, 77
    elif case == "np_cubic_greville":
        bs, lo, order, B = D.UniformBSplines(3, False, 0.0, 2.0, 300), 3, 0, 64
    else:
        br = np.linspace(0.0, 1.0, 101)
        br[1:-1] += rng.uniform(-0.003, 0.003, 99)
        bs, lo, order, B = D.NonUniformBSplines(4, True, br), 0, 1, 50
    pts = D.greville_points(bs, lo, lo)
    builder = D.SplineBuilder(bs, pts, lo, lo)
    ev = D.SplineEvaluator(bs)
    vals = cuda(rng.standard_normal((pts.size, B)))
    nd = builder.s_nbv_xmin
    dlo = cuda(rng.standard_normal((nd, B))) if lo == 1 else None
    dhi = cuda(rng.standard_normal((nd, B))) if lo == 1 else None
    x = cuda(rng.uniform(bs.rmin, bs.rmax, (333, B)))
    c1 = torch.zeros((bs.size, B), dtype=torch.float64, device="cuda")
    o1 = torch.zeros((333, B), dtype=torch.float64, device="cuda")
    fused = builder.build_and_evaluate(ev, c1, vals, x, o1, dlo, dhi, order=order)
    c2 = torch.zeros_like(c1)
    o2 = torch.zeros_like(o1)
    builder(c2, vals, dlo, dhi)
    if order == 0:
        ev(o2, x, c2)
    else:
        ev.deriv(order, o2, x, c2)
    assert torch.equal(c1, c2)
    assert relerr(o1.cpu().numpy(), o2.cpu().numpy()) <= 1e-14
    # one kernel on uniform bases; the builder and evaluator kernels on non-uniform ones
    assert fused == (case in ("c1", "np_cubic_greville"))
