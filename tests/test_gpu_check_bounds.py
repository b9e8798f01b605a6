"""The bounds-checked build (libddcb_check.so, DDCB_CHECK_BOUNDS=1): every computed array index of
the kernels checked on the device. The same workloads -- 1D non-uniform Hermite build, values with
extrapolation, first derivatives and integrals; the fused periodic build + evaluate and its adjoint;
the advection step; a 2D and a 3D build with their evaluators; an uneven batch -- run in two fresh
processes, one per library. On these valid inputs no kernel may record an out-of-range index
(ddcb_last_device_error reports none), and the checked build's outputs must equal the default
build's bit for bit (the checks clamp only indices that are out of range), except the adjoint's
sample cotangents, whose atomic sums may differ in the last bits between any two runs."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_workloads(out_path):
    """Runs in the child process: every workload, then ddcb_last_device_error; saves the outputs."""
    import torch

    import ddc_b200 as D
    from ddc_b200 import workloads as W

    rng = np.random.default_rng(7)
    cu = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    res = {"checked": np.array([int(D.bounds_checked())])}
    # 1D non-uniform quintic, Hermite closures
    br = W.config2_breaks(96)
    bs = D.NonUniformBSplines(5, False, br)
    b = D.SplineBuilder(bs, None, D.SplineBuilderClosure.HERMITE, D.SplineBuilderClosure.HERMITE)
    B = 37
    vals = rng.standard_normal((b.npoints, B))
    dlo, dhi = rng.standard_normal((b.s_nbv_xmin, B)), rng.standard_normal((b.s_nbv_xmax, B))
    c = torch.zeros((bs.size, B), dtype=torch.float64, device="cuda")
    b(c, cu(vals), cu(dlo), cu(dhi))
    for ex in ((D.Extrapolation.NULL, D.Extrapolation.CONSTANT), (D.Extrapolation.CONSTANT, D.Extrapolation.NULL)):
        e = D.SplineEvaluator(bs, *ex)
        x = cu(rng.uniform(-0.2, 1.2, (150, B)))
        y = torch.zeros((150, B), dtype=torch.float64, device="cuda")
        e(y, x, c)
        res[f"v{int(ex[0])}"] = y.cpu().numpy()
        e.deriv(1, y, x, c)
        res[f"d{int(ex[0])}"] = y.cpu().numpy()
    integ = torch.zeros(B, dtype=torch.float64, device="cuda")
    D.SplineEvaluator(bs).integrate(integ, c)
    res["c1d"], res["i1d"] = c.cpu().numpy(), integ.cpu().numpy()
    # periodic uniform cubic: fused build + evaluate, its adjoint, the advection step
    bs = D.UniformBSplines(3, True, 0.0, 1.0, 200)
    b, e = D.SplineBuilder(bs), D.SplineEvaluator(bs)
    B = 300
    v, x, g = cu(rng.standard_normal((200, B))), cu(rng.uniform(-1, 2, (200, B))), cu(rng.standard_normal((200, B)))
    c = torch.empty((bs.size, B), dtype=torch.float64, device="cuda")
    y = torch.empty((200, B), dtype=torch.float64, device="cuda")
    b.build_and_evaluate(e, c, v, x, y)
    gv, gx = torch.empty_like(v), torch.empty_like(x)
    b.build_and_evaluate_adjoint(e, x, c, g, gv, gx)
    res["fc"], res["fy"], res["gv"], res["gx"] = c.cpu().numpy(), y.cpu().numpy(), gv.cpu().numpy(), gx.cpu().numpy()
    ya = torch.empty_like(v)
    b.advect(e, ya, v, 0.37 / 200, velocity=1.0)
    res["adv"] = ya.cpu().numpy()
    # 2D: periodic cubic x Hermite cubic
    bx, by = D.UniformBSplines(3, True, 0.0, 1.0, 24), D.UniformBSplines(3, False, 0.0, 1.0, 20)
    Bx, By = D.SplineBuilder(bx, None, 0, 0), D.SplineBuilder(by, None, 1, 1)
    nf = 5
    v2 = rng.standard_normal((Bx.npoints, By.npoints, nf))
    d0, d1 = rng.standard_normal((Bx.npoints, 1, nf)), rng.standard_normal((Bx.npoints, 1, nf))
    c2 = torch.zeros((bx.size, by.size, nf), dtype=torch.float64, device="cuda")
    D.SplineBuilder2D(Bx, By)(c2, cu(v2), derivs_min2=cu(d0), derivs_max2=cu(d1))
    xy = rng.uniform(-0.1, 1.1, (64, nf, 2))
    y2 = torch.zeros((64, nf), dtype=torch.float64, device="cuda")
    D.SplineEvaluator2D(D.SplineEvaluator(bx), D.SplineEvaluator(by))(y2, cu(xy), c2)
    res["c2d"], res["y2d"] = c2.cpu().numpy(), y2.cpu().numpy()
    # 3D: periodic x Hermite x Greville, non-uniform in x3
    b1 = D.SplineBuilder(D.UniformBSplines(3, True, 0.0, 1.0, 10), None, 0, 0)
    b2 = D.SplineBuilder(D.UniformBSplines(4, False, 0.0, 1.0, 9), None, 1, 1)
    br3 = np.linspace(0.0, 1.0, 12)
    br3[1:-1] += rng.uniform(-0.02, 0.02, 10)
    b3 = D.SplineBuilder(D.NonUniformBSplines(2, False, br3), None, 3, 3)
    nb = 3
    v3 = rng.standard_normal((b1.npoints, b2.npoints, b3.npoints, nb))
    dm = rng.standard_normal((b1.npoints, b2.s_nbv_xmin, b3.npoints, nb))
    dM = rng.standard_normal((b1.npoints, b2.s_nbv_xmax, b3.npoints, nb))
    sizes = tuple(bb.bsplines.size for bb in (b1, b2, b3))
    c3 = torch.zeros(sizes + (nb,), dtype=torch.float64, device="cuda")
    D.SplineBuilder3D(b1, b2, b3)(c3, cu(v3), derivs_min2=cu(dm), derivs_max2=cu(dM))
    x3 = rng.uniform(-0.1, 1.1, (40, nb, 3))
    y3 = torch.zeros((40, nb), dtype=torch.float64, device="cuda")
    D.SplineEvaluator3D(*[D.SplineEvaluator(bb.bsplines) for bb in (b1, b2, b3)])(y3, cu(x3), c3)
    res["c3d"], res["y3d"] = c3.cpu().numpy(), y3.cpu().numpy()
    # an uneven batch
    probs = W.config4(count=64, nmax=700, seed=0xDDC0 + 77)
    w = W.config4_batch(D, probs)
    batch = D.UnevenBatch(w["builders"], w["evaluators"], w["nevals"])
    info = batch.info
    cb = torch.zeros((info.total_coefs,), dtype=torch.float64, device="cuda")
    yb = torch.zeros((info.total_evals,), dtype=torch.float64, device="cuda")
    batch(cu(w["vals"]), cu(w["dlo"]), cu(w["dhi"]), cb, cu(w["coords"]), yb)
    res["cb"], res["yb"] = cb.cpu().numpy(), yb.cpu().numpy()
    D.last_device_error()  # raises if a kernel recorded an out-of-range index
    np.savez(out_path, **res)


def run_child(out_path, checked):
    env = dict(os.environ)
    env.pop("DDCB_CHECK_BOUNDS", None)
    if checked:
        env["DDCB_CHECK_BOUNDS"] = "1"
    code = f"import sys; sys.path.insert(0, {ROOT!r}); import tests.test_gpu_check_bounds as t; t.run_workloads({out_path!r})"
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]


def test_checked_build_matches_default_build(tmp_path):
    if not os.path.exists(os.path.join(ROOT, "ddc_b200", "libddcb_check.so")):
        pytest.fail("libddcb_check.so is not built (python -m ddc_b200.build --check-bounds)")
    a, b = str(tmp_path / "default.npz"), str(tmp_path / "checked.npz")
    run_child(a, False)
    run_child(b, True)
    za, zb = np.load(a), np.load(b)
    assert int(za["checked"][0]) == 0 and int(zb["checked"][0]) == 1
    for k in za.files:
        if k == "checked":
            continue
        if k == "gv":
            # the adjoint scatter adds cotangents with shared-memory atomics, whose order (and so the
            # last bits of the sums) varies from run to run in either build
            assert np.abs(za[k] - zb[k]).max() <= 1e-13 * np.abs(za[k]).max(), k
            continue
        assert np.array_equal(za[k], zb[k], equal_nan=True), k
