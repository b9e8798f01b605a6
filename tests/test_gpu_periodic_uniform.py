"""Periodic splines on uniform meshes against the oracle: coefficients and evaluated values
(values and first derivatives) within 1e-12, for every degree, for sizes whose Greville points
are exact in binary (powers of two) and inexact (the assembled matrix is then circulant only up to
round-off), for small and large batches, through ddcb_build and the fused ddcb_build_eval."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


CASES = [(d, n, B) for d in (1, 2, 3, 4, 5) for n, B in ((128, 37), (1000, 301), (1024, 2600), (3000, 64))]


@pytest.mark.parametrize("case", CASES, ids=[f"d{c[0]}_n{c[1]}_B{c[2]}" for c in CASES])
def test_periodic_uniform_matches_oracle(case, oracle_mod):
    import ddc_b200 as D

    O = oracle_mod
    d, n, B = case
    bs = D.UniformBSplines(d, True, 0.0, 2.0, n)
    obs = O.BSplines(d, True, rmin=0.0, rmax=2.0, ncells=n)
    b = D.SplineBuilder(bs)
    ev = D.SplineEvaluator(bs)
    ob = O.Builder(obs, b.interpolation_points, O.PERIODIC, O.PERIODIC)
    rng = np.random.default_rng(d * 1000 + n)
    x = b.interpolation_points
    k = rng.integers(1, 9, B)
    vals = np.cos(np.pi * k[None, :] * x[:, None] + rng.random(B)[None, :] * 6.28) + 0.1 * rng.standard_normal((n, B))
    ref = ob(vals)
    coefs = torch.full((bs.size, B), float("nan"), dtype=torch.float64, device="cuda")
    b(coefs, cuda(vals))
    torch.cuda.synchronize()
    assert relerr(coefs.cpu().numpy(), ref) <= 1e-12
    m = 77
    xe = rng.random((m, B)) * 2.0
    c2 = torch.full_like(coefs, float("nan"))
    y = torch.full((m, B), float("nan"), dtype=torch.float64, device="cuda")
    for order in (0, 1):
        b.build_and_evaluate(ev, c2, cuda(vals), cuda(xe), y, order=order)
        torch.cuda.synchronize()
        assert relerr(c2.cpu().numpy(), ref) <= 1e-12
        yref = O.evaluate(obs, xe, ref, order=None if order == 0 else 1)
        # a derivative differences neighbouring coefficients (times n / length): its error is
        # measured against the coefficients' scale times that factor
        scale = np.abs(yref).max() if order == 0 else max(np.abs(yref).max(), np.abs(ref).max() * n / 2.0)
        assert np.abs(y.cpu().numpy() - yref).max() <= 1e-12 * scale
