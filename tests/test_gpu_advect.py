"""One semi-Lagrangian advection step (ddcb_advect; examples/characteristics_advection.cpp:243-259)
against the oracle: the splines of the lines built from f_in, evaluated at the feet x_q - dt v of
the interpolation points with the evaluator's boundary handling. <= 1e-12 relative (max norm).
Uniform bases run the step as one kernel with the feet computed in it; other bases run the build,
a feet kernel and the evaluator."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def D():
    import ddc_b200

    ddc_b200.load_library()
    return ddc_b200


def test_advect_periodic_constant_velocity(D, oracle_mod):
    """The characteristics-advection example's step: periodic uniform cubic, constant velocity,
    batch of lines in the (x, y) layout; feet cross the periodic boundary."""
    O = oracle_mod
    nc, B = 100, 37
    bs = D.UniformBSplines(3, True, -1.0, 1.0, nc)
    obs = O.BSplines(3, True, rmin=-1.0, rmax=1.0, ncells=nc)
    b, e = D.SplineBuilder(bs), D.SplineEvaluator(bs)
    pts = b.interpolation_points
    rng = np.random.default_rng(1)
    f = rng.standard_normal((pts.size, B))
    dt, v = 0.013, 1.7
    out = torch.empty((pts.size, B), dtype=torch.float64, device="cuda")
    coefs = torch.empty((bs.size, B), dtype=torch.float64, device="cuda")
    fused = b.advect(e, out, cuda(f), dt, v, spline=coefs)
    ref_c = O.Builder(obs, pts, 0, 0)(f)
    feet = np.repeat((pts - dt * v)[:, None], B, axis=1)
    want = O.evaluate(obs, feet, ref_c, ex_lo=0, ex_hi=0)
    assert fused
    assert relerr(coefs.cpu().numpy(), ref_c) <= 1e-12
    assert relerr(out.cpu().numpy(), want) <= 1e-12
    # without the coefficient output: the same values
    out2 = torch.empty_like(out)
    b.advect(e, out2, cuda(f), dt, v)
    assert torch.equal(out, out2)


def test_advect_velocity_per_row(D, oracle_mod):
    """The 2D step's x-advection: (x, y, field) data, velocity per y row (velocity_div = fields)."""
    O = oracle_mod
    nx, ny, F = 64, 9, 5
    bs = D.UniformBSplines(3, True, 0.0, 1.0, nx)
    obs = O.BSplines(3, True, rmin=0.0, rmax=1.0, ncells=nx)
    b, e = D.SplineBuilder(bs), D.SplineEvaluator(bs)
    pts = b.interpolation_points
    rng = np.random.default_rng(2)
    f = rng.standard_normal((pts.size, ny, F))
    vy = rng.uniform(-1.0, 1.0, ny)
    dt = 0.5 / nx
    out = torch.empty(f.shape, dtype=torch.float64, device="cuda")
    assert b.advect(e, out, cuda(f), dt, cuda(vy), velocity_div=F)
    ref_c = O.Builder(obs, pts, 0, 0)(f.reshape(pts.size, ny * F))
    feet = pts[:, None] - dt * np.repeat(vy, F)[None, :]
    want = O.evaluate(obs, feet, ref_c, ex_lo=0, ex_hi=0).reshape(f.shape)
    assert relerr(out.cpu().numpy(), want) <= 1e-12


@pytest.mark.parametrize("rules", [(1, 1), (2, 2)])
def test_advect_non_uniform_hermite(D, oracle_mod, rules):
    """Non-uniform quintic with Hermite derivatives (build, feet kernel, evaluator), feet leaving
    the domain at both ends under the null and constant rules."""
    O = oracle_mod
    rng = np.random.default_rng(3)
    nc, B = 40, 20
    br = np.linspace(0.0, 1.0, nc + 1)
    br[1:-1] += rng.uniform(-0.25, 0.25, nc - 1) / nc
    bs = D.NonUniformBSplines(5, False, br)
    obs = O.BSplines(5, False, breaks=br)
    b = D.SplineBuilder(bs, None, 1, 1)
    e = D.SplineEvaluator(bs, *rules)
    pts = b.interpolation_points
    f = rng.standard_normal((pts.size, B))
    dlo = rng.standard_normal((b.s_nbv_xmin, B))
    dhi = rng.standard_normal((b.s_nbv_xmax, B))
    v = rng.uniform(-2.0, 2.0, B)
    dt = 0.02
    out = torch.empty((pts.size, B), dtype=torch.float64, device="cuda")
    fused = b.advect(e, out, cuda(f), dt, cuda(v), cuda(dlo), cuda(dhi))
    assert not fused
    ref_c = O.Builder(obs, pts, 1, 1)(f, dlo, dhi)
    feet = pts[:, None] - dt * v[None, :]
    want = O.evaluate(obs, feet, ref_c, ex_lo=rules[0], ex_hi=rules[1])
    assert relerr(out.cpu().numpy(), want) <= 1e-12
