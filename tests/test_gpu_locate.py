"""Cell location on non-uniform meshes, CUDA evaluator against the oracle's bisection.

The evaluator guesses a point's cell from a bucket table ({first knot inside the bucket, cell at
the bucket start}) and checks the guess against the knots it loads for the basis; a wrong guess
(a bucket holding several knots, or a point within rounding of a bucket edge) falls back to a walk
over the knots. Graded and clustered meshes put many knots into single buckets, so both paths
run. Points sit at random, exactly on the break points and next to them, on bucket edges, and
(for values, with the null and constant extrapolation rules) outside the domain.

Tolerance: per point, |got - ref| <= 1e-12 * (|ref| + max|coef| * (degree / h)^order), h the width
of the point's cell, which bounds the FP64 rounding of the basis sums. A point evaluated on the
wrong cell would miss this by orders of magnitude away from the knots.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def D():
    import ddc_b200

    ddc_b200.load_library()
    return ddc_b200


def mesh(kind, nc):
    u = np.linspace(0.0, 1.0, nc + 1)
    if kind == "quadratic":
        br = u ** 2
    elif kind == "cluster":
        # uniform cells plus 40 break points squeezed into [0.5, 0.5 + 1e-6]
        br = np.unique(np.concatenate([u, 0.5 + np.linspace(0.0, 1e-6, 41)]))
    else:
        br = u
    return -2.0 + 5.0 * br  # domain [-2, 3]


def points(br, B, rng):
    lo, hi = br[0], br[-1]
    nb = 8 * (len(br) - 1)
    special = np.concatenate([br, lo + (hi - lo) * np.arange(nb + 1) / nb, np.nextafter(br, -np.inf),
                              np.nextafter(br, np.inf), [lo - 0.3, hi + 0.2, lo - 1e-300, hi + 1e-12]])
    m = len(special) + 257
    x = rng.uniform(lo, hi, (m, B))
    cols = rng.integers(0, B, len(special))
    x[np.arange(len(special)), cols] = special
    return x


def local_scale(br, x, degree, order, cmax):
    idx = np.clip(np.searchsorted(br, x, side="right") - 1, 0, len(br) - 2)
    h = br[idx + 1] - br[idx]
    return cmax * (degree / h) ** order


@pytest.mark.parametrize("kind", ["quadratic", "cluster"])
@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("periodic", [False, True])
def test_graded_mesh_locate(D, oracle_mod, kind, degree, periodic):
    O = oracle_mod
    nc = 200
    br = mesh(kind, nc)
    bs = D.NonUniformBSplines(degree, periodic, br)
    obs = O.BSplines(degree, periodic, breaks=br)
    rng = np.random.default_rng(degree * 7 + (kind == "cluster") + 2 * periodic)
    B = 24
    x = points(br, B, rng)
    if periodic:
        # the evaluator wraps into the period; keep the points inside so derivatives compare too
        x = np.clip(x, br[0], np.nextafter(br[-1], -np.inf))
    coefs = rng.standard_normal((bs.size, B))
    if periodic:
        coefs[bs.size - degree:] = coefs[:degree]
    cmax = np.abs(coefs).max()
    xg, cg = torch.from_numpy(x).cuda(), torch.from_numpy(coefs).cuda()
    out = torch.empty_like(xg)
    rules = [(O.EX_PERIODIC, O.EX_PERIODIC)] if periodic else [(O.EX_NULL, O.EX_NULL), (O.EX_CONSTANT, O.EX_CONSTANT)]
    for ex_lo, ex_hi in rules:
        ev = D.SplineEvaluator(bs, ex_lo, ex_hi)
        ev(out, xg, cg)
        ref = O.evaluate(obs, x, coefs, ex_lo=ex_lo, ex_hi=ex_hi)
        got = out.cpu().numpy()
        assert np.all(np.abs(got - ref) <= 1e-12 * (np.abs(ref) + cmax)), np.abs(got - ref).max()
    # derivatives take no extrapolation rule; far outside the domain the end cells' polynomial
    # extension cancels catastrophically, so they are compared on the domain (ends included)
    ev = D.SplineEvaluator(bs)
    xin = np.clip(x, br[0], br[-1])
    xg = torch.from_numpy(xin).cuda()
    for order in range(1, min(degree, 2) + 1):
        ev.deriv(order, out, xg, cg)
        ref = O.evaluate(obs, xin, coefs, order=order)
        got = out.cpu().numpy()
        tol = 1e-12 * (np.abs(ref) + local_scale(br, xin, degree, order, cmax))
        assert np.all(np.abs(got - ref) <= tol), (order, np.abs(got - ref).max())
