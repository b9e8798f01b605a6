"""2D tensor-product builder / evaluator vs the CPU oracle (SplineBuilder2D, SplineEvaluator2D).

Tolerance: max-norm relative error <= 1e-12 for coefficients, values, derivatives and integrals
(measured on B200: at most 6e-15 for coefficients, 8e-15 for values and 1e-14 for first and mixed
derivatives on these cases, whose tensor-product condition numbers reach 2e3). The named 512 x 512 x
64-field case runs at full size in FP64 and in FP32 with FP64 refinement."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def basis_pair(D, O, spec, rng):
    deg, periodic, uniform, nc = spec
    if uniform:
        return D.UniformBSplines(deg, periodic, 0.0, 1.0, nc), O.BSplines(deg, periodic, rmin=0.0, rmax=1.0, ncells=nc)
    br = np.linspace(0.0, 1.0, nc + 1)
    br[1:-1] += rng.uniform(-0.25, 0.25, nc - 1) / nc
    return D.NonUniformBSplines(deg, periodic, br), O.BSplines(deg, periodic, breaks=br)


CASES = [
    # (dim1 spec, closure1, dim2 spec, closure2, nbatch)
    ((3, True, True, 40), (0, 0), (3, False, True, 36), (1, 1), 5),     # the characteristics-advection pair
    ((5, False, False, 24), (1, 3), (4, True, False, 30), (0, 0), 3),
    ((2, False, True, 20), (1, 1), (5, False, False, 22), (1, 1), 2),
    ((4, False, True, 25), (3, 3), (3, False, False, 27), (2, 2), 4),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_build2d_eval2d(oracle_mod, case):
    import ddc_b200 as D

    O = oracle_mod
    rng = np.random.default_rng(100 + case)
    spec1, (lo1, hi1), spec2, (lo2, hi2), B = CASES[case]
    b1, o1 = basis_pair(D, O, spec1, rng)
    b2, o2 = basis_pair(D, O, spec2, rng)
    p1, p2 = D.greville_points(b1, lo1, hi1), D.greville_points(b2, lo2, hi2)
    B1, B2 = D.SplineBuilder(b1, p1, lo1, hi1), D.SplineBuilder(b2, p2, lo2, hi2)
    OB1, OB2 = O.Builder(o1, p1, lo1, hi1), O.Builder(o2, p2, lo2, hi2)
    nl1, nh1, nl2, nh2 = B1.s_nbv_xmin, B1.s_nbv_xmax, B2.s_nbv_xmin, B2.s_nbv_xmax
    vals = rng.standard_normal((p1.size, p2.size, B))
    dmin1 = rng.standard_normal((nl1, p2.size, B)) if lo1 == 1 else None
    dmax1 = rng.standard_normal((nh1, p2.size, B)) if hi1 == 1 else None
    dmin2 = rng.standard_normal((p1.size, nl2, B)) if lo2 == 1 else None
    dmax2 = rng.standard_normal((p1.size, nh2, B)) if hi2 == 1 else None
    mixed = [rng.standard_normal((a, c, B)) if (ca == 1 and cb == 1) else None
             for (a, ca), (c, cb) in [((nl1, lo1), (nl2, lo2)), ((nh1, hi1), (nl2, lo2)), ((nl1, lo1), (nh2, hi2)),
                                      ((nh1, hi1), (nh2, hi2))]]
    ref = O.build2d(OB1, OB2, vals, dmin1, dmax1, dmin2, dmax2, mixed)
    coefs = torch.zeros((b1.size, b2.size, B), dtype=torch.float64, device="cuda")
    g = lambda a: None if a is None else cuda(a)
    D.SplineBuilder2D(B1, B2)(coefs, cuda(vals), g(dmin1), g(dmax1), g(dmin2), g(dmax2), *[g(m) for m in mixed])
    got = coefs.cpu().numpy()
    assert relerr(got, ref) <= 1e-12
    # evaluation (values with boundary handling, then derivatives in range)
    E1, E2 = D.SplineEvaluator(b1, 2, 2), D.SplineEvaluator(b2, 2, 2)
    ev = D.SplineEvaluator2D(E1, E2)
    m = 200
    x1 = rng.uniform(-0.2, 1.2, (m, B))
    x2 = rng.uniform(-0.2, 1.2, (m, B))
    xy = np.stack([x1, x2], axis=-1)
    out = torch.zeros((m, B), dtype=torch.float64, device="cuda")
    ev(out, cuda(xy), coefs)
    want = O.evaluate2d(o1, o2, x1, x2, ref, ex=(2, 2, 2, 2))
    assert relerr(out.cpu().numpy(), want) <= 1e-12
    x1 = rng.uniform(0.0, 1.0, (m, B))
    x2 = rng.uniform(0.0, 1.0, (m, B))
    xy = np.stack([x1, x2], axis=-1)
    for (a, c), fn in [((1, 0), ev.deriv_dim_1), ((0, 1), ev.deriv_dim_2), ((1, 1), ev.deriv_1_and_2)]:
        fn(out, cuda(xy), coefs)
        want = O.evaluate2d(o1, o2, x1, x2, ref, orders=(a, c))
        assert relerr(out.cpu().numpy(), want) <= 1e-12
    integ = torch.zeros(B, dtype=torch.float64, device="cuda")
    ev.integrate(integ, coefs)
    want = np.einsum("ijb,i,j->b", ref, o1.integrals(), o2.integrals())
    scale = np.abs(ref).max()
    assert np.abs(integ.cpu().numpy() - want).max() / scale <= 1e-12


def test_build2d_explicit_workspace(oracle_mod):
    """The caller-provided workspace path gives the same coefficients as the stream-ordered one."""
    import ddc_b200 as D

    rng = np.random.default_rng(5)
    b1 = D.UniformBSplines(3, True, 0.0, 1.0, 64)
    b2 = D.UniformBSplines(3, False, 0.0, 1.0, 64)
    B1 = D.SplineBuilder(b1, None, 0, 0)
    B2 = D.SplineBuilder(b2, None, 1, 1)
    b2d = D.SplineBuilder2D(B1, B2)
    B = 40
    vals = cuda(rng.standard_normal((B1.npoints, B2.npoints, B)))
    dmin2 = cuda(rng.standard_normal((B1.npoints, 1, B)))
    dmax2 = cuda(rng.standard_normal((B1.npoints, 1, B)))
    c1 = torch.zeros((b1.size, b2.size, B), dtype=torch.float64, device="cuda")
    c2 = torch.zeros_like(c1)
    b2d(c1, vals, None, None, dmin2, dmax2)
    ws = torch.empty(b2d.workspace_bytes(B) // 8 + 1, dtype=torch.float64, device="cuda")
    b2d(c2, vals, None, None, dmin2, dmax2, workspace=ws)
    assert torch.equal(c1, c2)
    # captured in a CUDA graph (the derivative-slab passes fork onto a second stream and join back
    # inside the capture) and replayed on new inputs: the same as the eager build
    c3 = torch.zeros_like(c1)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        b2d(c3, vals, None, None, dmin2, dmax2, workspace=ws)  # warm-up outside the capture
    torch.cuda.current_stream().wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        b2d(c3, vals, None, None, dmin2, dmax2, workspace=ws)
    vals.copy_(cuda(rng.standard_normal((B1.npoints, B2.npoints, B))))
    g.replay()
    b2d(c1, vals, None, None, dmin2, dmax2, workspace=ws)
    torch.cuda.synchronize()
    assert torch.equal(c1, c3)


@pytest.mark.parametrize("precision,rounds", [("fp64", 2), ("fp32_refine", 1), ("fp32_refine", 2)])
def test_config3_full_size(oracle_mod, precision, rounds):
    """Periodic cubic x Hermite cubic on 512 x 512 cells, 64 fields (sin(2 pi x) cos(pi y) a_b plus
    noise), built on the GPU and evaluated at the semi-Lagrangian feet (x - v dt, y), against the
    oracle's FP64 build and evaluation of the same inputs. Measured: FP64 6e-15 / 4e-15
    (coefficients / values); FP32 + 1 refinement round 7e-14 / 3e-14; 2 rounds 6e-15 / 4e-15."""
    import ddc_b200 as D
    from ddc_b200 import workloads as W

    O = oracle_mod
    w = W.config3()
    bx, by = D.UniformBSplines(3, True, 0.0, 1.0, 512), D.UniformBSplines(3, False, 0.0, 1.0, 512)
    obx, oby = O.BSplines(3, True, rmin=0.0, rmax=1.0, ncells=512), O.BSplines(3, False, rmin=0.0, rmax=1.0, ncells=512)
    px, py = D.greville_points(bx, 0, 0), D.greville_points(by, 1, 1)
    ref = O.build2d(O.Builder(obx, px, 0, 0), O.Builder(oby, py, 1, 1), w["vals"], None, None, w["dmin2"], w["dmax2"])
    xy = w["coords"]
    want = O.evaluate2d(obx, oby, xy[..., 0].reshape(-1, 64), xy[..., 1].reshape(-1, 64), ref, ex=(0, 0, 1, 1))
    Bx = D.SplineBuilder(bx, None, 0, 0, precision=precision, refine_rounds=rounds)
    By = D.SplineBuilder(by, None, 1, 1, precision=precision, refine_rounds=rounds)
    c = torch.zeros((bx.size, by.size, 64), dtype=torch.float64, device="cuda")
    D.SplineBuilder2D(Bx, By)(c, cuda(w["vals"]), derivs_min2=cuda(w["dmin2"]), derivs_max2=cuda(w["dmax2"]))
    y = torch.zeros((512 * 513, 64), dtype=torch.float64, device="cuda")
    D.SplineEvaluator2D(D.SplineEvaluator(bx), D.SplineEvaluator(by))(y, cuda(xy), c)
    ec, ey = relerr(c.cpu().numpy(), ref), relerr(y.cpu().numpy(), want)
    print(f"PARITY config3 {precision} rounds={rounds} coefs={ec:.2e} values={ey:.2e}")
    assert ec <= 1e-12
    assert ey <= 1e-12
