"""The FP32 + FP64-refinement builder (precision "fp32_refine") against the FP64 oracle.

Error metric: max-norm relative error of the coefficients, as in the FP64 tests. Bound: 1e-12 after
the default two refinement rounds (BASELINE's bound for the refined FP32 path), or 10*cond(A)*eps
for the few ill-conditioned systems. One round stops short of FP64 accuracy on the quintic system,
which shows that the refinement, not the FP32 solve, sets the final error.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

P, H, HH, G = 0, 1, 2, 3


def relerr(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def D():
    import ddc_b200

    ddc_b200.load_library()
    return ddc_b200


def breaks_of(nc, seed):
    rng = np.random.default_rng(seed)
    h = 1.0 / nc
    br = np.arange(nc + 1) * h
    br[1:-1] += (rng.random(nc - 1) - 0.5) * 0.6 * h
    return np.sort(br)


CASES = [
    # degree, uniform, periodic, ncells, lower, upper
    (3, True, True, 1024, P, P),
    (3, True, True, 1000, P, P),
    (3, True, False, 512, H, H),
    (5, False, False, 1024, H, H),
    (4, False, False, 300, G, H),
    (2, False, True, 101, P, P),
    (1, True, False, 40, G, G),
    (5, True, True, 64, P, P),
    (3, False, False, 77, HH, G),
]


def build_pair(D, O, case, seed):
    degree, uniform, periodic, nc, lo, hi = case
    if uniform:
        bs = D.UniformBSplines(degree, periodic, 0.0, 1.0, nc)
        obs = O.BSplines(degree, periodic, rmin=0.0, rmax=1.0, ncells=nc)
    else:
        br = breaks_of(nc, seed)
        bs = D.NonUniformBSplines(degree, periodic, br)
        obs = O.BSplines(degree, periodic, breaks=br)
    return bs, obs


@pytest.mark.parametrize("case", CASES, ids=[f"d{c[0]}{'u' if c[1] else 'n'}{'p' if c[2] else 'b'}{c[3]}_{c[4]}{c[5]}" for c in CASES])
def test_refined_build_matches_fp64_oracle(D, oracle_mod, case):
    O = oracle_mod
    bs, obs = build_pair(D, O, case, 17)
    lo, hi = case[4], case[5]
    ref_b = D.SplineBuilder(bs, None, lo, hi)
    ob = O.Builder(obs, ref_b.interpolation_points, lo, hi)
    rng = np.random.default_rng(3)
    B = 203
    x = ref_b.interpolation_points
    k = rng.integers(1, 9, B)
    ph = rng.random(B) * 2 * np.pi
    vals = np.cos(2 * np.pi * k[None, :] * x[:, None] + ph[None, :])
    dlo = rng.standard_normal((ref_b.s_nbv_xmin, B)) if lo == H else None
    dhi = rng.standard_normal((ref_b.s_nbv_xmax, B)) if hi == H else None
    ref = ob(vals, dlo, dhi)
    cond = np.linalg.cond(ob.matrix())
    tol = max(1e-12, 10 * cond * np.finfo(float).eps)
    errs = {}
    for rounds in (2, 3):
        b = D.SplineBuilder(bs, None, lo, hi, precision="fp32_refine", refine_rounds=rounds)
        coefs = torch.full((bs.size, B), float("nan"), dtype=torch.float64, device="cuda")
        b(coefs, cuda(vals), None if dlo is None else cuda(dlo), None if dhi is None else cuda(dhi))
        torch.cuda.synchronize()
        errs[rounds] = relerr(coefs.cpu().numpy(), ref)
    assert errs[2] <= tol, errs
    assert errs[3] <= tol, errs


def test_refinement_rounds_reduce_the_error(D, oracle_mod):
    """One round leaves about (cond * 2^-24)^2 relative error; two reach FP64 level (C2 shape)."""
    from ddc_b200 import workloads

    O = oracle_mod
    br = workloads.config2_breaks()
    bs = D.NonUniformBSplines(5, False, br)
    obs = O.BSplines(5, False, breaks=br)
    pts = D.greville_points(bs, H, H)
    w = workloads.config2(B=387, points=pts)
    ref = O.Builder(obs, pts, H, H)(w["vals"], w["dlo"], w["dhi"])
    errs = []
    for rounds in (1, 2, 3):
        b = D.SplineBuilder(bs, pts, H, H, precision="fp32_refine", refine_rounds=rounds)
        coefs = torch.zeros((bs.size, 387), dtype=torch.float64, device="cuda")
        b(coefs, cuda(w["vals"]), cuda(w["dlo"]), cuda(w["dhi"]))
        torch.cuda.synchronize()
        errs.append(relerr(coefs.cpu().numpy(), ref))
    assert errs[0] < 1e-8, errs
    assert errs[1] <= 1e-12 and errs[2] <= 1e-12, errs


def test_refined_2d_build(D, oracle_mod):
    """The 2D builder (periodic cubic x Hermite cubic, 128 x 128, 6 fields) in refinement mode."""
    O = oracle_mod
    n = 128
    bx, by = D.UniformBSplines(3, True, 0.0, 1.0, n), D.UniformBSplines(3, False, 0.0, 1.0, n)
    obx, oby = O.BSplines(3, True, rmin=0.0, rmax=1.0, ncells=n), O.BSplines(3, False, rmin=0.0, rmax=1.0, ncells=n)
    Bx = D.SplineBuilder(bx, None, P, P, precision="fp32_refine")
    By = D.SplineBuilder(by, None, H, H, precision="fp32_refine")
    rng = np.random.default_rng(9)
    nb = 6
    vals = rng.standard_normal((Bx.npoints, By.npoints, nb))
    dmin2 = rng.standard_normal((Bx.npoints, 1, nb))
    dmax2 = rng.standard_normal((Bx.npoints, 1, nb))
    ox = O.Builder(obx, Bx.interpolation_points, P, P)
    oy = O.Builder(oby, By.interpolation_points, H, H)
    ref = O.build2d(ox, oy, vals, derivs_min2=dmin2, derivs_max2=dmax2)
    b2 = D.SplineBuilder2D(Bx, By)
    coefs = torch.zeros((bx.size, by.size, nb), dtype=torch.float64, device="cuda")
    b2(coefs, cuda(vals), derivs_min2=cuda(dmin2), derivs_max2=cuda(dmax2))
    torch.cuda.synchronize()
    assert relerr(coefs.cpu().numpy(), ref) <= 1e-12


@pytest.mark.parametrize("rounds", [1, 2])
def test_config5_forward_full_size(D, oracle_mod, rounds):
    """The differentiation workload's forward pass at its named size: periodic uniform cubic, 1024
    cells, 65536 lines, FP32 solves with FP64 refinement, build then evaluation at 1024 random
    points per line (the fused kernel, or the two kernels), against the oracle's FP64 build and
    evaluation of the same inputs: <= 1e-12 (coefficients and values)."""
    from tests.test_gpu_adjoint import config5_inputs

    O = oracle_mod
    B = 1 << 16
    vals, coords, _ = config5_inputs(B)
    bs = D.UniformBSplines(3, True, 0.0, 1.0, 1024)
    obs = O.BSplines(3, True, rmin=0.0, rmax=1.0, ncells=1024)
    pts = D.greville_points(bs, P, P)
    ref = O.Builder(obs, pts, P, P)(vals)
    want = O.evaluate(obs, coords, ref, ex_lo=0, ex_hi=0)
    b = D.SplineBuilder(bs, None, P, P, precision="fp32_refine", refine_rounds=rounds)
    e = D.SplineEvaluator(bs)
    c = torch.empty((bs.size, B), dtype=torch.float64, device="cuda")
    y = torch.empty((1024, B), dtype=torch.float64, device="cuda")
    b.build_and_evaluate(e, c, cuda(vals), cuda(coords), y)
    ec, ey = relerr(c.cpu().numpy(), ref), relerr(y.cpu().numpy(), want)
    print(f"PARITY config5 fp32_refine rounds={rounds} coefs={ec:.2e} values={ey:.2e}")
    assert ec <= 1e-12
    assert ey <= 1e-12


def test_refinement_convergence_status(D):
    """The device-side check of refined solves (ddcb_builder_device_status): the default bound
    (estimated relative error <= 1e-12) holds after the default two rounds on the quintic Hermite
    system; a bound no solve can meet (1e-30, standing in for a capped iteration) reports
    DDCB_ERR_NOT_CONVERGED once, and the query clears the flag."""
    from ddc_b200._lib import DdcbError

    br = breaks_of(256, 9)
    bs = D.NonUniformBSplines(5, False, br)
    rng = np.random.default_rng(4)
    B = 64
    b = D.SplineBuilder(bs, None, H, H, precision="fp32_refine", refine_rounds=2)
    vals = cuda(rng.standard_normal((b.npoints, B)))
    dlo, dhi = cuda(rng.standard_normal((2, B))), cuda(rng.standard_normal((2, B)))
    c = torch.empty((bs.size, B), dtype=torch.float64, device="cuda")
    b(c, vals, dlo, dhi)
    b.device_status()  # converged: no exception
    strict = D.SplineBuilder(bs, None, H, H, precision="fp32_refine", refine_rounds=1, refine_tolerance=1e-30)
    strict(c, vals, dlo, dhi)
    with pytest.raises(DdcbError) as err:
        strict.device_status()
    assert err.value.status == 6  # DDCB_ERR_NOT_CONVERGED
    strict.device_status()  # cleared
    # FP64 builders never set the flag
    b64 = D.SplineBuilder(bs, None, H, H)
    b64(c, vals, dlo, dhi)
    b64.device_status()
