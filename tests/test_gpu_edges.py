"""Edge cases of the CUDA path, through the C-ABI, against the oracle: empty batches and empty point
sets (no work, no error, as the reference returns early, spline_builder.hpp:929-931), one line and
ragged tiles, the smallest grids each degree and closure accepts, and evaluation exactly at the
break points and the domain ends (where the cell search and the end rules of
bsplines_non_uniform.hpp:666-695 and bsplines_uniform.hpp:465-470 decide). Tolerance: max-norm
relative error <= 1e-12, or 10 cond(A) eps for an ill-conditioned small system."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

P, H, G = 0, 1, 3


def relerr(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def D():
    import ddc_b200

    ddc_b200.load_library()
    assert torch.cuda.is_available()
    return ddc_b200


def bases(D, O, degree, periodic, uniform, nc, seed=0):
    if uniform:
        return D.UniformBSplines(degree, periodic, 0.0, 2.0, nc), O.BSplines(degree, periodic, rmin=0.0, rmax=2.0, ncells=nc)
    br = np.linspace(0.0, 2.0, nc + 1)
    br[1:-1] += np.random.default_rng(seed).uniform(-0.2, 0.2, nc - 1) * (2.0 / nc)
    return D.NonUniformBSplines(degree, periodic, br), O.BSplines(degree, periodic, breaks=br)


def derivs(builder, c, B, rng):
    if c != H:
        return None, None
    return rng.standard_normal((builder.s_nbv_xmin, B)), rng.standard_normal((builder.s_nbv_xmax, B))


def test_empty_batch_and_empty_point_sets(D):
    bs = D.NonUniformBSplines(5, False, np.linspace(0.0, 1.0, 40))
    b, e = D.SplineBuilder(bs, None, H, H), D.SplineEvaluator(bs)
    z = lambda *s: torch.zeros(s, dtype=torch.float64, device="cuda")
    c0 = z(bs.size, 0)
    b(c0, z(b.npoints, 0), z(b.s_nbv_xmin, 0), z(b.s_nbv_xmax, 0))
    e(z(7, 0), z(7, 0), c0)
    e.deriv(1, z(7, 0), z(7, 0), c0)
    e.integrate(z(0), c0)
    b.build_and_evaluate(e, c0, z(b.npoints, 0), z(7, 0), z(7, 0), z(b.s_nbv_xmin, 0), z(b.s_nbv_xmax, 0))
    # lines present, no evaluation point
    B = 5
    c = z(bs.size, B)
    vals, dlo, dhi = z(b.npoints, B) + 1.0, z(b.s_nbv_xmin, B), z(b.s_nbv_xmax, B)
    b(c, vals, dlo, dhi)
    e(z(0, B), z(0, B), c)
    b.build_and_evaluate(e, c, vals, z(0, B), z(0, B), dlo, dhi)
    torch.cuda.synchronize()
    # a constant function: every coefficient is 1
    assert torch.allclose(c, torch.ones_like(c), rtol=0, atol=1e-13)
    pbs = D.UniformBSplines(3, True, 0.0, 1.0, 32)
    pb, pe = D.SplineBuilder(pbs), D.SplineEvaluator(pbs)
    pc = z(pbs.size, 0)
    g = z(32, 0)
    pb.build_and_evaluate_adjoint(pe, z(9, 0), pc, z(9, 0), g, z(9, 0))
    pb.advect(pe, z(32, 0), z(32, 0), 0.1, velocity=1.0)


@pytest.mark.parametrize("B", [1, 3, 9, 17])
@pytest.mark.parametrize("kind", ["quintic_hermite_nonuniform", "cubic_periodic_uniform", "quadratic_greville"])
def test_one_line_and_ragged_tiles(D, oracle_mod, B, kind):
    O = oracle_mod
    rng = np.random.default_rng(B)
    degree, periodic, uniform, c = {"quintic_hermite_nonuniform": (5, False, False, H),
                                   "cubic_periodic_uniform": (3, True, True, P),
                                   "quadratic_greville": (2, False, True, G)}[kind]
    bs, obs = bases(D, O, degree, periodic, uniform, 50, seed=B)
    b, e = D.SplineBuilder(bs, None, c, c), D.SplineEvaluator(bs)
    ob = O.Builder(obs, b.interpolation_points, c, c)
    tol = max(1e-12, 10 * np.linalg.cond(ob.matrix()) * np.finfo(float).eps)
    vals = rng.standard_normal((b.npoints, B))
    dlo, dhi = derivs(b, c, B, rng)
    ref = ob(vals, dlo, dhi)
    coefs = torch.zeros((bs.size, B), dtype=torch.float64, device="cuda")
    b(coefs, cuda(vals), None if dlo is None or dlo.size == 0 else cuda(dlo), None if dhi is None or dhi.size == 0 else cuda(dhi))
    assert relerr(coefs.cpu().numpy(), ref) <= tol
    x = rng.uniform(-0.3, 2.3, (41, B))
    y = torch.zeros((41, B), dtype=torch.float64, device="cuda")
    e(y, cuda(x), coefs)
    assert relerr(y.cpu().numpy(), O.evaluate(obs, x, ref)) <= tol
    # the fused path (uniform bases) on the same lines
    c2 = torch.zeros_like(coefs)
    y2 = torch.zeros_like(y)
    b.build_and_evaluate(e, c2, cuda(vals), cuda(x), y2, None if dlo is None or dlo.size == 0 else cuda(dlo),
                         None if dhi is None or dhi.size == 0 else cuda(dhi))
    assert torch.equal(c2, coefs)
    assert relerr(y2.cpu().numpy(), y.cpu().numpy()) <= 1e-14


@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("c", [P, H, G])
@pytest.mark.parametrize("uniform", [True, False])
def test_smallest_grids(D, oracle_mod, degree, c, uniform):
    """The smallest grids the reference's construction handles -- ncells = degree (non-periodic),
    degree + 1 (periodic; fewer cells are refused, DDCB_ERR_BAD_GRID) -- built and evaluated."""
    O = oracle_mod
    rng = np.random.default_rng(degree * 10 + c)
    nc = degree + 1 if c == P else max(degree, 2 if not uniform else 1)
    if c == P:
        with pytest.raises(D.DdcbError):
            D.SplineBuilder(bases(D, O, degree, True, uniform, degree, seed=nc)[0], None, c, c)
    bs, obs = bases(D, O, degree, c == P, uniform, nc, seed=nc)
    b = D.SplineBuilder(bs, None, c, c)
    ob = O.Builder(obs, b.interpolation_points, c, c)
    tol = max(1e-12, 10 * np.linalg.cond(ob.matrix()) * np.finfo(float).eps)
    B = 4
    vals = rng.standard_normal((b.npoints, B))
    dlo, dhi = derivs(b, c, B, rng)
    ref = ob(vals, dlo, dhi)
    coefs = torch.zeros((bs.size, B), dtype=torch.float64, device="cuda")
    b(coefs, cuda(vals), None if dlo is None or dlo.size == 0 else cuda(dlo), None if dhi is None or dhi.size == 0 else cuda(dhi))
    assert relerr(coefs.cpu().numpy(), ref) <= tol, (nc, b.npoints)
    x = rng.uniform(0.0, 2.0, (23, B))
    y = torch.zeros((23, B), dtype=torch.float64, device="cuda")
    D.SplineEvaluator(bs)(y, cuda(x), coefs)
    assert relerr(y.cpu().numpy(), O.evaluate(obs, x, ref)) <= tol


@pytest.mark.parametrize("degree", [1, 3, 4, 5])
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("uniform", [True, False])
def test_points_on_breaks_and_ends(D, oracle_mod, degree, periodic, uniform):
    O = oracle_mod
    rng = np.random.default_rng(degree)
    bs, obs = bases(D, O, degree, periodic, uniform, 17, seed=degree)
    knots = np.array(bs.knots())
    br = knots[degree:degree + 18]
    x1 = np.concatenate([br, [0.0, 2.0, np.nextafter(2.0, 0.0), np.nextafter(0.0, 1.0)],
                         np.nextafter(br[1:-1], 0.0), np.nextafter(br[1:-1], 3.0)])
    B = 3
    x = np.repeat(x1[:, None], B, axis=1)
    coefs = rng.standard_normal((bs.size, B))
    if periodic:
        coefs[bs.nbasis:] = coefs[: bs.size - bs.nbasis]  # the periodic copies
    e = D.SplineEvaluator(bs)
    y = torch.zeros(x.shape, dtype=torch.float64, device="cuda")
    e(y, cuda(x), cuda(coefs))
    assert relerr(y.cpu().numpy(), O.evaluate(obs, x, coefs)) <= 1e-12
    e.deriv(1, y, cuda(x), cuda(coefs))
    assert relerr(y.cpu().numpy(), O.evaluate(obs, x, coefs, order=1)) <= 1e-12
