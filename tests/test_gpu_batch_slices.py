"""A batch of 65536 lines built in one call and the same lines built in slices of 1024 give
identical coefficients: every line's arithmetic is independent of the batch size and of the tile
it lands in. One slice is also checked against the oracle (<= 1e-12, or 10*cond(A)*eps)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

B = 1 << 16
SLICE = 1024


def breaks(nc):
    rng = np.random.default_rng(nc)
    br = np.arange(nc + 1) / nc
    br[1:-1] += (rng.random(nc - 1) - 0.5) * 0.6 / nc
    return br


@pytest.mark.parametrize("case", ["periodic_cubic_1024", "quintic_hermite_1024", "quartic_greville_700"])
def test_whole_batch_matches_sliced_batch(case, oracle_mod):
    import ddc_b200 as D

    O = oracle_mod
    if case == "periodic_cubic_1024":
        bs, obs, lo = D.UniformBSplines(3, True, 0.0, 1.0, 1024), O.BSplines(3, True, rmin=0.0, rmax=1.0, ncells=1024), 0
    elif case == "quintic_hermite_1024":
        br = breaks(1024)
        bs, obs, lo = D.NonUniformBSplines(5, False, br), O.BSplines(5, False, breaks=br), 1
    else:
        br = breaks(700)
        bs, obs, lo = D.NonUniformBSplines(4, False, br), O.BSplines(4, False, breaks=br), 3
    b = D.SplineBuilder(bs, None, lo, lo)
    gen = torch.Generator(device="cuda").manual_seed(3)
    vals = torch.randn((b.npoints, B), dtype=torch.float64, device="cuda", generator=gen)
    nd = b.s_nbv_xmin if lo == 1 else 0
    dlo = torch.randn((nd, B), dtype=torch.float64, device="cuda", generator=gen) if nd else None
    dhi = torch.randn((nd, B), dtype=torch.float64, device="cuda", generator=gen) if nd else None
    full = torch.full((bs.size, B), float("nan"), dtype=torch.float64, device="cuda")
    b(full, vals, dlo, dhi)
    sliced = torch.full_like(full, float("nan"))
    for s0 in range(0, B, SLICE):
        sl = slice(s0, s0 + SLICE)
        b(sliced[:, sl], vals[:, sl], None if dlo is None else dlo[:, sl], None if dhi is None else dhi[:, sl])
    torch.cuda.synchronize()
    assert torch.equal(full, sliced)
    pts = b.interpolation_points
    ob = O.Builder(obs, pts, lo, lo)
    cols = slice(B - 37, B)
    ref = ob(vals[:, cols].cpu().numpy(), None if dlo is None else dlo[:, cols].cpu().numpy(),
             None if dhi is None else dhi[:, cols].cpu().numpy())
    got = full[:, cols].cpu().numpy()
    tol = max(1e-12, 10 * np.linalg.cond(ob.matrix()) * np.finfo(float).eps)
    assert np.abs(got - ref).max() <= tol * np.abs(ref).max()
