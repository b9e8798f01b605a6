"""3D builder and N-dimensional evaluator (SplineBuilder3D, SplineEvaluator3D, SplineEvaluatorND) on
the CUDA path vs the oracle, through the C-ABI.

Tolerance: max-norm relative error <= 1e-12 for coefficients, values and integrals, or
10 cond(A1) cond(A2) cond(A3) eps when that is larger (the condition number of the tensor-product
system; two backward-stable FP64 solves agree to about that); derivatives of order k take the same
bound times the k-th power of the largest inverse cell width ratio (they amplify coefficient
differences by 1/h per order), capped at 1e-10.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

H, G, P, HH = 1, 3, 0, 2


def relerr(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def make_dim(D, O, spec, rng):
    deg, closure, uniform, nc = spec
    periodic = closure == P
    if uniform:
        bs = D.UniformBSplines(deg, periodic, 0.0, 1.0, nc)
        obs = O.BSplines(deg, periodic, rmin=0.0, rmax=1.0, ncells=nc)
    else:
        br = np.linspace(0.0, 1.0, nc + 1)
        br[1:-1] += rng.uniform(-0.25, 0.25, nc - 1) / nc
        bs = D.NonUniformBSplines(deg, periodic, br)
        obs = O.BSplines(deg, periodic, breaks=br)
    pts = D.greville_points(bs, closure, closure)
    return bs, obs, D.SplineBuilder(bs, pts, closure, closure), O.Builder(obs, pts, closure, closure), pts, closure


CASES = [
    # three dimensions (degree, closure, uniform, ncells) and the batch
    ([(3, P, True, 12), (3, H, True, 10), (3, H, True, 11)], 3),      # advection-like: periodic x Hermite x Hermite
    ([(5, H, False, 9), (4, H, True, 10), (2, H, False, 8)], 2),      # all 27 inputs read
    ([(2, G, False, 10), (5, P, False, 9), (4, HH, True, 12)], 4),    # Greville, periodic non-uniform, homogeneous Hermite
    ([(1, G, True, 7), (3, G, False, 13), (5, H, True, 10)], 33),     # more than one warp of batch entries
]


def inputs_for(dims, B, rng):
    """vals and the derivative arrays the closures read, named as the reference's arguments."""
    kinds = []
    for (_, _, b, _, pts, cl) in dims:
        lo = b.s_nbv_xmin if cl == H else 0
        hi = b.s_nbv_xmax if cl == H else 0
        kinds.append({0: pts.size, 1: lo, 2: hi})
    lab = {1: "min", 2: "max"}
    vals = rng.standard_normal((kinds[0][0], kinds[1][0], kinds[2][0], B))
    derivs = {}
    for k1 in range(3):
        for k2 in range(3):
            for k3 in range(3):
                ks = (k1, k2, k3)
                if ks == (0, 0, 0) or any(kinds[d][k] == 0 for d, k in enumerate(ks)):
                    continue
                parts = [f"{lab[k]}{d + 1}" for d, k in enumerate(ks) if k]
                key = ("derivs_" if len(parts) == 1 else "mixed_derivs_") + "_".join(parts)
                derivs[key] = rng.standard_normal(tuple(kinds[d][k] for d, k in enumerate(ks)) + (B,))
    return vals, derivs


@pytest.mark.parametrize("case", range(len(CASES)))
def test_build3d_evalnd(oracle_mod, case):
    import ddc_b200 as D

    O = oracle_mod
    rng = np.random.default_rng(300 + case)
    specs, B = CASES[case]
    dims = [make_dim(D, O, s, rng) for s in specs]
    vals, derivs = inputs_for(dims, B, rng)
    ref = O.build3d(dims[0][3], dims[1][3], dims[2][3], vals, derivs)
    cond = np.prod([np.linalg.cond(d[3].matrix()) for d in dims])
    tol = max(1e-12, 10 * cond * np.finfo(float).eps)
    b3 = D.SplineBuilder3D(dims[0][2], dims[1][2], dims[2][2])
    coefs = torch.full(ref.shape, np.nan, dtype=torch.float64, device="cuda")
    b3(coefs, cuda(vals), **{k: cuda(v) for k, v in derivs.items()})
    got = coefs.cpu().numpy()
    assert relerr(got, ref) <= tol
    # with a caller workspace: identical
    ws = torch.empty(b3.workspace_bytes(B) // 8 + 1, dtype=torch.float64, device="cuda")
    c2 = torch.zeros_like(coefs)
    b3(c2, cuda(vals), workspace=ws, **{k: cuda(v) for k, v in derivs.items()})
    assert torch.equal(c2, coefs)
    # evaluation on the oracle's coefficients (isolates the evaluator): values with boundary handling
    exs = [(2, 1), (1, 2), (2, 2)]
    E = [D.SplineEvaluator(d[0], *ex) for d, ex in zip(dims, exs)]
    ev = D.SplineEvaluator3D(*E)
    m = 60
    x = rng.uniform(-0.15, 1.15, (m, B, 3))
    x[: m // 2, :, :] = np.clip(x[: m // 2], 0.0, 1.0)  # half the points inside the domain
    out = torch.zeros((m, B), dtype=torch.float64, device="cuda")
    cref = cuda(ref)
    ev(out, cuda(x), cref)
    bss = [d[1] for d in dims]
    oex = [(0, 0) if d[0].periodic else ex for d, ex in zip(dims, exs)]
    want = O.evaluatend(bss, x, ref, ex=oex)
    assert relerr(out.cpu().numpy(), want) <= 1e-12
    # derivatives (no boundary handling), in range
    xin = rng.uniform(0.0, 1.0, (m, B, 3))
    for orders in ((1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 1), (2, 0, 1)):
        if any(o > d[0].degree for o, d in zip(orders, dims)):
            continue
        ev.deriv(orders, out, cuda(xin), cref)
        want = O.evaluatend(bss, xin, ref, orders=orders)
        assert relerr(out.cpu().numpy(), want) <= 1e-11
    integ = torch.zeros(B, dtype=torch.float64, device="cuda")
    ev.integrate(integ, cref)
    want = np.einsum("ijkb,i,j,k->b", ref, *[d[1].integrals() for d in dims])
    assert np.abs(integ.cpu().numpy() - want).max() / np.abs(ref).max() <= 1e-12


def test_evalnd_matches_1d_and_2d(oracle_mod):
    """N = 1 and N = 2 give the 1D and 2D evaluators' results (values with every rule, and a
    derivative)."""
    import ddc_b200 as D

    rng = np.random.default_rng(17)
    b1 = D.NonUniformBSplines(4, False, np.sort(np.r_[0.0, rng.uniform(0.05, 0.95, 14), 1.0]))
    b2 = D.UniformBSplines(3, True, -1.0, 2.0, 20)
    B, m = 37, 90
    c1 = cuda(rng.standard_normal((b1.size, B)))
    e1 = D.SplineEvaluator(b1, D.Extrapolation.CONSTANT, D.Extrapolation.NULL)
    x = cuda(rng.uniform(-0.2, 1.2, (m, B)))
    y1 = torch.empty((m, B), dtype=torch.float64, device="cuda")
    e1(y1, x, c1)
    yn = torch.empty_like(y1)
    D.SplineEvaluatorND(e1)(yn, x[..., None].contiguous(), c1)
    assert relerr(yn.cpu(), y1.cpu()) <= 1e-13  # the 1D kernel divides by knot differences, ND uses the span table
    e2 = D.SplineEvaluator(b2)
    c2 = cuda(rng.standard_normal((b1.size, b2.size, B)))
    xy = np.stack([rng.uniform(-0.3, 1.3, (m, B)), rng.uniform(-2.0, 3.0, (m, B))], axis=-1)
    for rules in ((D.Extrapolation.CONSTANT, D.Extrapolation.CONSTANT), (D.Extrapolation.NULL, D.Extrapolation.CONSTANT)):
        ea = D.SplineEvaluator(b1, *rules)
        y2 = torch.empty((m, B), dtype=torch.float64, device="cuda")
        D.SplineEvaluator2D(ea, e2)(y2, cuda(xy), c2)
        yn2 = torch.empty_like(y2)
        D.SplineEvaluatorND(ea, e2)(yn2, cuda(xy), c2)
        assert relerr(yn2.cpu(), y2.cpu()) <= 1e-14
    xin = np.stack([rng.uniform(0.0, 1.0, (m, B)), rng.uniform(-1.0, 2.0, (m, B))], axis=-1)
    y2 = torch.empty((m, B), dtype=torch.float64, device="cuda")
    D.SplineEvaluator2D(e1, e2).deriv_1_and_2(y2, cuda(xin), c2)
    yn2 = torch.empty_like(y2)
    D.SplineEvaluatorND(e1, e2).deriv((1, 1), yn2, cuda(xin), c2)
    assert relerr(yn2.cpu(), y2.cpu()) <= 1e-14


def test_evalnd_4d(oracle_mod):
    """A 4D coefficient grid (periodic, Hermite-sized, non-uniform dimensions) against the oracle."""
    import ddc_b200 as D

    O = oracle_mod
    rng = np.random.default_rng(23)
    specs = [(1, True, True, 5), (2, False, False, 6), (3, False, True, 4), (5, True, False, 7)]
    bs, obs = [], []
    for deg, per, uni, nc in specs:
        if uni:
            bs.append(D.UniformBSplines(deg, per, 0.0, 1.0, nc))
            obs.append(O.BSplines(deg, per, rmin=0.0, rmax=1.0, ncells=nc))
        else:
            br = np.linspace(0.0, 1.0, nc + 1)
            br[1:-1] += rng.uniform(-0.2, 0.2, nc - 1) / nc
            bs.append(D.NonUniformBSplines(deg, per, br))
            obs.append(O.BSplines(deg, per, breaks=br))
    B, m = 5, 40
    c = rng.standard_normal(tuple(b.size for b in bs) + (B,))
    E = [D.SplineEvaluator(b, 1, 1) for b in bs]
    ev = D.SplineEvaluatorND(*E)
    x = rng.uniform(-0.1, 1.1, (m, B, 4))
    out = torch.zeros((m, B), dtype=torch.float64, device="cuda")
    ev(out, cuda(x), cuda(c))
    want = O.evaluatend(obs, x, c, ex=[(0, 0) if b.periodic else (1, 1) for b in bs])
    assert relerr(out.cpu().numpy(), want) <= 1e-12
    xin = rng.uniform(0.0, 1.0, (m, B, 4))
    ev.deriv((1, 2, 0, 3), out, cuda(xin), cuda(c))
    want = O.evaluatend(obs, xin, c, orders=(1, 2, 0, 3))
    assert relerr(out.cpu().numpy(), want) <= 1e-11
    integ = torch.zeros(B, dtype=torch.float64, device="cuda")
    ev.integrate(integ, cuda(c))
    want = np.einsum("ijklb,i,j,k,l->b", c, *[o.integrals() for o in obs])
    assert np.abs(integ.cpu().numpy() - want).max() / np.abs(c).max() <= 1e-12
