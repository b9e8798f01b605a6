"""The reference's own known-answer tests for the spline path, run on the CUDA path itself (through
the C-ABI, no oracle): the analytic answers and error bounds of tests/splines/*.cpp of
CExA-project/ddc. They pin the product to the reference's test expectations directly, beside the
oracle comparisons of the other -m gpu tests."""
import numpy as np
import pytest

from tests.test_oracle_known_answers import NP_BCS, cos_eval, tikhomirov

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

P, H, HH, G = 0, 1, 2, 3


@pytest.fixture(scope="module")
def D():
    import ddc_b200

    ddc_b200.load_library()
    assert torch.cuda.is_available()
    return ddc_b200


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def make_basis(D, degree, periodic, uniform, ncells):
    if uniform:
        return D.UniformBSplines(degree, periodic, 0.0, 1.0, ncells)
    return D.NonUniformBSplines(degree, periodic, np.arange(ncells + 1) / ncells)


@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("uniform", [True, False])
@pytest.mark.parametrize("bcs", NP_BCS + [(P, P)])
def test_cosine_error_bounds_cuda(D, degree, uniform, bcs):
    """non_periodic_spline_builder.cpp:303-316 / periodic_spline_builder.cpp:198-208: the spline of
    cos(2 pi x) on 10 cells at its interpolation points, its first derivative and its integral, within
    the Tikhomirov bounds of spline_error_bounds.hpp:34-39."""
    lo, hi = bcs
    bs = make_basis(D, degree, lo == P, uniform, 10)
    b = D.SplineBuilder(bs, None, lo, hi)
    pts = b.interpolation_points
    odd = degree % 2
    vals = cos_eval(pts)[:, None]
    dlo = np.array([cos_eval(0.0, deriv=i + odd) for i in range(b.s_nbv_xmin)]).reshape(-1, 1) if lo == H else None
    dhi = np.array([cos_eval(1.0, deriv=i + odd) for i in range(b.s_nbv_xmax)]).reshape(-1, 1) if hi == H else None
    c = torch.zeros((bs.size, 1), dtype=torch.float64, device="cuda")
    b(c, cuda(vals), None if dlo is None or dlo.size == 0 else cuda(dlo), None if dhi is None or dhi.size == 0 else cuda(dhi))
    e = D.SplineEvaluator(bs)
    y = torch.zeros((pts.size, 1), dtype=torch.float64, device="cuda")
    e(y, cuda(pts[:, None]), c)
    err = np.abs(y.cpu().numpy()[:, 0] - vals[:, 0]).max()
    e.deriv(1, y, cuda(pts[:, None]), c)
    err_d = np.abs(y.cpu().numpy()[:, 0] - cos_eval(pts, deriv=1)).max()
    integ = torch.zeros(1, dtype=torch.float64, device="cuda")
    e.integrate(integ, c)
    h = 0.1
    assert err <= max(tikhomirov(h, degree, (2 * np.pi) ** (degree + 1)), 1e-14)
    assert err_d <= max(tikhomirov(h, degree - 1, (2 * np.pi) ** (degree + 1)), 1e-12 * 2 * np.pi)
    assert abs(float(integ[0])) <= max(tikhomirov(h, degree + 1, (2 * np.pi) ** (degree + 1)), 1e-14 / (2 * np.pi))


@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("uniform", [True, False])
def test_periodicity_cuda(D, degree, uniform):
    """periodicity_spline_builder.cpp:178-205: for cos(2 pi x), s(x + 1.5) = -s(x) at the points."""
    bs = make_basis(D, degree, True, uniform, 10)
    b = D.SplineBuilder(bs, None, P, P)
    pts = b.interpolation_points
    c = torch.zeros((bs.size, 1), dtype=torch.float64, device="cuda")
    b(c, cuda(cos_eval(pts)[:, None]))
    y = torch.zeros((pts.size, 1), dtype=torch.float64, device="cuda")
    D.SplineEvaluator(bs)(y, cuda(pts[:, None] + 1.5), c)
    bound = max(tikhomirov(0.1, degree, (2 * np.pi) ** (degree + 1)), 1e-14)
    assert np.abs(y.cpu().numpy()[:, 0] + cos_eval(pts)).max() <= bound


@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("uniform", [True, False])
def test_partition_of_unity_cuda(D, degree, periodic, uniform):
    """bsplines.cpp:67-136: the B-splines sum to one -- the spline with every coefficient 1 is 1 at
    every point of the domain, and its derivatives vanish."""
    bs = make_basis(D, degree, periodic, uniform, 20)
    x = np.linspace(0.0, 1.0, 1001)[:, None]
    c = torch.ones((bs.size, 1), dtype=torch.float64, device="cuda")
    e = D.SplineEvaluator(bs)
    y = torch.zeros((1001, 1), dtype=torch.float64, device="cuda")
    e(y, cuda(x), c)
    assert np.abs(y.cpu().numpy() - 1.0).max() <= 1e-15 * 8
    e.deriv(1, y, cuda(x), c)
    assert np.abs(y.cpu().numpy()).max() <= 1e-11


@pytest.mark.parametrize("rule", ["null", "constant"])
def test_extrapolation_rules_cuda(D, rule):
    """extrapolation_rule.cpp: outside the domain the null rule gives 0 and the constant rule the
    value at the nearest end."""
    bs = D.UniformBSplines(3, False, 0.0, 1.0, 12)
    b = D.SplineBuilder(bs, None, G, G)
    pts = b.interpolation_points
    c = torch.zeros((bs.size, 1), dtype=torch.float64, device="cuda")
    b(c, cuda(cos_eval(pts, c1=0.1)[:, None]))
    r = D.Extrapolation.NULL if rule == "null" else D.Extrapolation.CONSTANT
    e = D.SplineEvaluator(bs, r, r)
    x = np.array([-0.5, -1e-9, 0.0, 1.0, 1.0 + 1e-9, 3.0])[:, None]
    y = torch.zeros((6, 1), dtype=torch.float64, device="cuda")
    e(y, cuda(x), c)
    got = y.cpu().numpy()[:, 0]
    ends = torch.zeros((2, 1), dtype=torch.float64, device="cuda")
    D.SplineEvaluator(bs)(ends, cuda(np.array([[0.0], [1.0]])), c)
    s0, s1 = ends.cpu().numpy()[:, 0]
    if rule == "null":
        np.testing.assert_array_equal(got[[0, 1, 4, 5]], 0.0)
    else:
        np.testing.assert_array_equal(got[[0, 1]], s0)
        np.testing.assert_array_equal(got[[4, 5]], s1)
    assert got[2] == s0 and got[3] == s1
