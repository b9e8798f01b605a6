"""CUDA builder on meshes chosen against the plan's decision to factorise without row
interchanges: strongly graded cells (widths over six decades), one near-degenerate cell (1e-9 of
its neighbours), alternating wide and narrow cells (1000:1), and a 1e4-long domain whose Hermite
rows carry dx^k factors up to 1e11. The oracle always pivots (the reference's LAPACK path); the
device coefficients must agree within max(1e-12, 10 cond(A) eps) relative, and the evaluated
spline must reproduce the samples at the interpolation points."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


@pytest.fixture(scope="module")
def D():
    import ddc_b200

    ddc_b200.load_library()
    assert torch.cuda.is_available()
    return ddc_b200


def breaks_of(kind, nc=60, seed=3):
    rng = np.random.default_rng(seed)
    if kind == "graded":
        w = 1e6 ** (np.arange(nc) / (nc - 1))
    elif kind == "tiny_cell":
        w = np.ones(nc)
        w[nc // 2] = 1e-9
    elif kind == "alternating":
        w = np.where(np.arange(nc) % 2 == 1, 1e-3, 1.0)
    else:  # long domain, mildly perturbed cells
        w = 1.0 + 0.3 * rng.uniform(-1, 1, nc)
    length = 1e4 if kind == "long_domain" else 1.0
    br = np.concatenate([[0.0], np.cumsum(w)]) * (length / w.sum())
    br[-1] = length
    return br


@pytest.mark.parametrize("kind", ["graded", "tiny_cell", "alternating", "long_domain"])
@pytest.mark.parametrize("degree", [1, 3, 5])
@pytest.mark.parametrize("closure", ["periodic", "hermite", "greville"])
def test_adversarial_mesh(D, oracle_mod, kind, degree, closure):
    O = oracle_mod
    br = breaks_of(kind)
    periodic = closure == "periodic"
    c = {"periodic": O.PERIODIC, "hermite": O.HERMITE, "greville": O.GREVILLE}[closure]
    bs = D.NonUniformBSplines(degree, periodic, br)
    obs = O.BSplines(degree, periodic, breaks=br)
    builder = D.SplineBuilder(bs, None, c, c)
    pts = builder.interpolation_points
    ob = O.Builder(obs, pts, c, c)
    tol = max(1e-12, 10 * np.linalg.cond(ob.matrix()) * np.finfo(float).eps)
    rng = np.random.default_rng(degree * 7 + len(kind))
    B = 6
    L = br[-1] - br[0]
    vals = np.cos(2 * np.pi * pts[:, None] / L * np.arange(1, B + 1)[None, :])
    nlo = builder.s_nbv_xmin if c == O.HERMITE else 0
    nhi = builder.s_nbv_xmax if c == O.HERMITE else 0
    her = c == O.HERMITE
    dlo = rng.uniform(-1, 1, (nlo, B)) / L if her else None
    dhi = rng.uniform(-1, 1, (nhi, B)) / L if her else None
    ref = ob(vals, dlo, dhi)
    # the device call takes no derivative array where there are no derivative rows
    cu = lambda a: None if a is None or a.size == 0 else torch.from_numpy(np.ascontiguousarray(a)).cuda()
    coefs = torch.zeros((bs.size, B), dtype=torch.float64, device="cuda")
    builder(coefs, cu(vals), cu(dlo), cu(dhi))
    got = coefs.cpu().numpy()
    assert relerr(got, ref) <= tol, (relerr(got, ref), tol)
    ev = D.SplineEvaluator(bs)
    y = torch.zeros((len(pts), B), dtype=torch.float64, device="cuda")
    ev(y, cu(np.repeat(pts[:, None], B, axis=1)), coefs)
    assert relerr(y.cpu().numpy(), vals) <= max(1e-11, tol)
