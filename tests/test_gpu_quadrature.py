"""Quadrature weights, the fused build + integrate, and polynomial exactness on the CUDA path.

* ddcb_quadrature_coefficients (device transposed solve) against the oracle's restatement of
  SplineBuilder::quadrature_coefficients (spline_builder.hpp:1103-1234) on every golden case:
  max-norm relative error <= 1e-12 (10 cond(A) eps for the few ill-conditioned fixtures, as in
  test_gpu_parity.py);
* ddcb_integrate_samples against the builder followed by SplineEvaluator::integrate, both on the
  GPU, and against the oracle's build followed by its integrate: |difference| <= 1e-12 times
  max|samples| x (rmax - rmin), the size of the integrals of such data (the integrals themselves can
  cancel to round-off, as periodic cosines do). The reference's quadrature weights are not the
  right weights here on non-uniform periodic bases with a non-zero offset (they skip the offset's
  rotation), so the fused kernel uses the builder's adjoint of the integrals instead;
* the polynomial-exactness test of tests/splines/non_periodic_spline_builder.cpp:297-301 run on the
  CUDA builder, evaluator, integral, quadrature weights and fused integral, degrees 1-5, every
  non-periodic closure pair, uniform, evenly spaced non-uniform and perturbed non-uniform meshes,
  with the reference's bounds (1e-14 values and integrals, 1e-11 first derivatives), at the
  interpolation points and at random points inside the domain.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from tests.test_gpu_parity import CASES, cuda, make_both, relerr  # noqa: E402


@pytest.fixture(scope="module")
def D():
    import ddc_b200

    ddc_b200.load_library()
    assert torch.cuda.is_available()
    return ddc_b200


def cond_tol(b):
    A = b.matrix()
    return max(1e-12, 10 * np.linalg.cond(A) * np.finfo(float).eps)


@pytest.mark.parametrize("i", range(len(CASES)))
def test_quadrature_coefficients_vs_oracle(D, oracle_mod, i):
    O = oracle_mod
    c = CASES[i]
    d, uniform, periodic, nc, lo, hi = (int(v) for v in c["meta"])
    bs, obs = make_both(D, O, c)
    b = D.SplineBuilder(bs, c["points"], lo, hi)
    ob = O.Builder(obs, c["points"], lo, hi)
    qlo, q, qhi = b.quadrature_coefficients()
    rlo, rq, rhi = ob.quadrature_coefficients()
    got = np.concatenate([qlo, q, qhi])
    ref = np.concatenate([rlo, rq, rhi])
    assert got.shape == ref.shape
    assert relerr(got, ref) <= cond_tol(ob)
    # the device copy holds the same numbers
    qd = b.quadrature_coefficients_device().cpu().numpy()
    assert np.array_equal(qd, got)


@pytest.mark.parametrize("i", range(0, len(CASES), 3))
def test_integrate_samples_vs_build_integrate(D, oracle_mod, i):
    O = oracle_mod
    c = CASES[i]
    d, uniform, periodic, nc, lo, hi = (int(v) for v in c["meta"])
    bs, obs = make_both(D, O, c)
    b = D.SplineBuilder(bs, c["points"], lo, hi)
    e = D.SplineEvaluator(bs)
    vals = cuda(c["vals"])
    B = vals.shape[1]
    dlo = cuda(c["dlo"]) if lo == 1 and c["dlo"].size else None
    dhi = cuda(c["dhi"]) if hi == 1 and c["dhi"].size else None
    fused = torch.empty(B, dtype=torch.float64, device="cuda")
    b.integrate_samples(fused, vals, dlo, dhi)
    coefs = torch.empty((bs.size, B), dtype=torch.float64, device="cuda")
    b(coefs, vals, dlo, dhi)
    two = torch.empty(B, dtype=torch.float64, device="cuda")
    e.integrate(two, coefs)
    f, t = fused.cpu().numpy(), two.cpu().numpy()
    ob = O.Builder(obs, c["points"], lo, hi)
    scale = max(np.abs(c["vals"]).max(), np.abs(c["dlo"]).max() if dlo is not None else 0.0,
                np.abs(c["dhi"]).max() if dhi is not None else 0.0) * (bs.rmax - bs.rmin)
    tol = cond_tol(ob) * scale
    assert np.abs(f - t).max() <= tol
    ref = O.integrate(obs, ob(c["vals"], c["dlo"] if lo == 1 else None, c["dhi"] if hi == 1 else None))
    assert np.abs(f - ref).max() <= tol


def test_integrate_samples_batch_layouts(D):
    """(x, batch), (batch, x) and (b1, x, b2) layouts give the same integrals."""
    bs = D.UniformBSplines(3, False, 0.0, 2.0, 40)
    b = D.SplineBuilder(bs, None, D.SplineBuilderClosure.GREVILLE, D.SplineBuilderClosure.GREVILLE)
    g = torch.Generator(device="cuda").manual_seed(3)
    v = torch.randn((b.npoints, 6, 5), dtype=torch.float64, device="cuda", generator=g)
    out_xb = torch.empty((6, 5), dtype=torch.float64, device="cuda")
    b.integrate_samples(out_xb, v)
    vb = v.permute(1, 2, 0).contiguous()  # (6, 5, x)
    out_bx = torch.empty((6, 5), dtype=torch.float64, device="cuda")
    b.integrate_samples(out_bx, vb, dim=2)
    vm = v.permute(1, 0, 2).contiguous()  # (6, x, 5)
    out_m = torch.empty((6, 5), dtype=torch.float64, device="cuda")
    b.integrate_samples(out_m, vm, dim=1)
    assert relerr(out_bx.cpu(), out_xb.cpu()) <= 1e-14
    assert relerr(out_m.cpu(), out_xb.cpu()) <= 1e-14


H, G = 1, 3
NP_BCS = [(H, H), (G, G), (H, G), (G, H)]


def _breaks(kind, ncells):
    if kind == "uniform":
        return None
    br = np.arange(ncells + 1) / ncells
    if kind == "perturbed":
        rng = np.random.default_rng(ncells)
        br[1:-1] += rng.uniform(-0.3, 0.3, ncells - 1) / ncells
    return br


@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("mesh", ["uniform", "even", "perturbed"])
@pytest.mark.parametrize("bcs", NP_BCS)
@pytest.mark.parametrize("ncells", [10, 97])
def test_polynomial_exactness_cuda(D, degree, mesh, bcs, ncells):
    """non_periodic_spline_builder.cpp:297-301 on the CUDA path: a degree-d spline reproduces a
    degree-d polynomial to round-off (values, first derivative, integral, quadrature)."""
    lo, hi = bcs
    br = _breaks(mesh, ncells)
    bs = D.UniformBSplines(degree, False, 0.0, 1.0, ncells) if br is None else D.NonUniformBSplines(degree, False, br)
    b = D.SplineBuilder(bs, None, lo, hi)
    e = D.SplineEvaluator(bs)
    pts = b.interpolation_points
    rng = np.random.default_rng(1234 + degree)
    coeffs = rng.uniform(0, 1, degree + 1)

    def poly(x, der=0):
        x = np.asarray(x, dtype=float)
        res = np.zeros_like(x)
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

    # the reference's bounds at its own size (10 cells); at 97 cells the uniform systems carry the
    # reference's symmetric storage of the centre block, whose entries take one side's round-off of
    # the basis values at the points (growing with the point's distance from rmin), so values and
    # integrals reproduce the polynomial to about 2e-14 there: bound 1e-13
    vtol = 1e-14 if ncells == 10 else 1e-13
    odd = degree % 2
    B = 4  # a few identical lines: the batch path, not one thread
    vals = np.repeat(poly(pts)[:, None], B, axis=1)
    dlo = np.repeat(np.array([poly(0.0, i + odd) for i in range(b.s_nbv_xmin)])[:, None], B, axis=1) if lo == H and b.s_nbv_xmin else None
    dhi = np.repeat(np.array([poly(1.0, i + odd) for i in range(b.s_nbv_xmax)])[:, None], B, axis=1) if hi == H and b.s_nbv_xmax else None
    coefs = torch.empty((bs.size, B), dtype=torch.float64, device="cuda")
    b(coefs, cuda(vals), cuda(dlo) if dlo is not None else None, cuda(dhi) if dhi is not None else None)
    xr = np.sort(rng.uniform(0.0, 1.0, 64))
    for x in (pts, xr):
        xs = cuda(np.repeat(x[:, None], B, axis=1))
        y = torch.empty_like(xs)
        dy = torch.empty_like(xs)
        e(y, xs, coefs)
        e.deriv(1, dy, xs, coefs)
        assert np.abs(y.cpu().numpy() - poly(x)[:, None]).max() / abs(poly(1.0)) <= vtol
        assert np.abs(dy.cpu().numpy() - poly(x, 1)[:, None]).max() / abs(poly(1.0, 1)) <= 1e-11
    exact = poly(1.0, -1) - poly(0.0, -1)
    max_norm_int = abs(poly(1.0, -1))
    integ = torch.empty(B, dtype=torch.float64, device="cuda")
    e.integrate(integ, coefs)
    assert np.abs(integ.cpu().numpy() - exact).max() / max_norm_int <= vtol
    qlo, q, qhi = b.quadrature_coefficients()
    qint = q @ vals[:, 0]
    if dlo is not None:
        qint += qlo @ dlo[:, 0]
    if dhi is not None:
        qint += qhi @ dhi[:, 0]
    assert abs(qint - exact) / max_norm_int <= vtol
    fused = torch.empty(B, dtype=torch.float64, device="cuda")
    b.integrate_samples(fused, cuda(vals), cuda(dlo) if dlo is not None else None, cuda(dhi) if dhi is not None else None)
    assert np.abs(fused.cpu().numpy() - exact).max() / max_norm_int <= vtol
