"""The uneven batch (ddcb_batch_uneven_*): one graph launch of persistent kernels over problems of
different size, degree, closure and mesh, against the per-problem builder + evaluator calls (the
same arithmetic, so the results must be identical) and against the oracle on every problem (<= 1e-12,
or 10*cond(A)*eps for the ill-conditioned systems), in FP64 and in FP32 with FP64 refinement, under
the warp and the block schedules."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["fp64", "fp32_refine"])
def setup(request):
    import ddc_b200 as D
    from ddc_b200 import workloads as W

    D.load_library()
    probs = W.config4(count=257, nmax=1500, seed=0xDDC0 + 44)
    w = W.config4_batch(D, probs, precision=request.param)
    w["precision"] = request.param
    batch = D.UnevenBatch(w["builders"], w["evaluators"], w["nevals"])
    cu = lambda a: torch.from_numpy(a).cuda()
    dev = dict(vals=cu(w["vals"]), dlo=cu(w["dlo"]), dhi=cu(w["dhi"]), coords=cu(w["coords"]))
    info = batch.info
    dev["coefs"] = torch.full((info.total_coefs,), float("nan"), dtype=torch.float64, device="cuda")
    dev["out"] = torch.full((info.total_evals,), float("nan"), dtype=torch.float64, device="cuda")
    return D, W, probs, w, batch, dev


def run(batch, dev):
    batch(dev["vals"], dev["dlo"], dev["dhi"], dev["coefs"], dev["coords"], dev["out"])
    torch.cuda.synchronize()
    return dev["coefs"].cpu().numpy().copy(), dev["out"].cpu().numpy().copy()


def per_problem(w, off):
    """The same problems through the one-problem builder and evaluator calls."""
    coefs, outs = [], []
    for i, (b, e) in enumerate(zip(w["builders"], w["evaluators"])):
        v = torch.from_numpy(w["vals"][off["vals"][i]:off["vals"][i + 1]].copy()).cuda()[:, None]
        lo = w["dlo"][off["derivs_lo"][i]:off["derivs_lo"][i + 1]]
        hi = w["dhi"][off["derivs_hi"][i]:off["derivs_hi"][i + 1]]
        lo = torch.from_numpy(lo.copy()).cuda()[:, None] if lo.size else None
        hi = torch.from_numpy(hi.copy()).cuda()[:, None] if hi.size else None
        c = torch.empty((b.info.size, 1), dtype=torch.float64, device="cuda")
        b(c, v, lo, hi)
        x = torch.from_numpy(w["coords"][off["evals"][i]:off["evals"][i + 1]].copy()).cuda()[:, None]
        y = torch.empty_like(x)
        e(y, x, c)
        coefs.append(c[:, 0].cpu().numpy())
        outs.append(y[:, 0].cpu().numpy())
    return np.concatenate(coefs), np.concatenate(outs)


def test_batch_matches_per_problem_calls(setup):
    D, W, probs, w, batch, dev = setup
    off = batch.offsets()
    coefs, out = run(batch, dev)
    rc, ro = per_problem(w, off)
    assert np.isfinite(coefs).all() and np.isfinite(out).all()
    np.testing.assert_array_equal(coefs, rc)
    np.testing.assert_array_equal(out, ro)


def test_graph_replay_and_tuning_keep_results(setup):
    D, W, probs, w, batch, dev = setup
    c1, o1 = run(batch, dev)
    c2, o2 = run(batch, dev)  # replays the cached graph
    info = batch.tune(dev["vals"], dev["dlo"], dev["dhi"], dev["coefs"], dev["coords"], dev["out"], reps=1)
    assert info.tuned_us > 0 and info.threads in (128, 256, 512) and info.warp_schedule in (0, 1)
    c3, o3 = run(batch, dev)  # the graph of the tuned schedule
    for c, o in ((c2, o2), (c3, o3)):
        np.testing.assert_array_equal(c, c1)
        np.testing.assert_array_equal(o, o1)
    for b in w["builders"]:
        b.device_status()  # refined problems converged (FP64 ones never flag)


def test_batch_against_oracle_every_problem(setup, oracle_mod):
    O = oracle_mod
    D, W, probs, w, batch, dev = setup
    off = batch.offsets()
    coefs, out = run(batch, dev)
    clos = {"periodic": O.PERIODIC, "hermite": O.HERMITE, "greville": O.GREVILLE}
    worst_c = worst_y = 0.0
    for i in range(len(probs)):
        p, b = probs[i], w["builders"][i]
        per = p["closure"] == "periodic"
        obs = (O.BSplines(p["degree"], per, rmin=0.0, rmax=1.0, ncells=p["ncells"]) if p["uniform"]
               else O.BSplines(p["degree"], per, breaks=p["breaks"]))
        c = clos[p["closure"]]
        ob = O.Builder(obs, b.interpolation_points, c, c)
        lo = w["dlo"][off["derivs_lo"][i]:off["derivs_lo"][i + 1]]
        hi = w["dhi"][off["derivs_hi"][i]:off["derivs_hi"][i + 1]]
        herm = p["closure"] == "hermite"
        ref = ob(w["vals"][off["vals"][i]:off["vals"][i + 1]], lo.reshape(-1, 1) if herm else None,
                 hi.reshape(-1, 1) if herm else None)[:, 0]
        tol = max(1e-12, 10 * np.linalg.cond(ob.matrix()) * np.finfo(float).eps)
        got = coefs[off["coefs"][i]:off["coefs"][i + 1]]
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max(), (i, p["ncells"], p["degree"], p["closure"])
        x = w["coords"][off["evals"][i]:off["evals"][i + 1]]
        ev = O.evaluate(obs, x[:, None], ref[:, None])[:, 0]
        # values relative to max(|values|, |coefficients|): the B-splines sum to one, so a value's
        # error is at most the largest coefficient error
        scale = max(np.abs(ev).max(), np.abs(ref).max())
        assert np.abs(out[off["evals"][i]:off["evals"][i + 1]] - ev).max() <= tol * scale
        worst_c = max(worst_c, np.abs(got - ref).max() / np.abs(ref).max())
        worst_y = max(worst_y, np.abs(out[off["evals"][i]:off["evals"][i + 1]] - ev).max() / scale)
    print(f"PARITY uneven-257 {w['precision']} worst coefs={worst_c:.2e} values={worst_y:.2e}")


def test_long_lines_fall_back_to_narrower_tiles():
    """A 6000-cell periodic quintic line does not fit an 8-line tile; the builder and the evaluator
    take narrower tiles instead of failing."""
    import ddc_b200 as D

    n = 6000
    br = np.arange(n + 1) / n
    br[1:-1] += (np.random.default_rng(1).random(n - 1) - 0.5) * 0.6 / n
    bs = D.NonUniformBSplines(5, True, br)
    b = D.SplineBuilder(bs)
    e = D.SplineEvaluator(bs)
    B = 5
    vals = torch.from_numpy(np.cos(2 * np.pi * np.outer(b.interpolation_points, np.arange(1, B + 1)))).cuda()
    c = torch.empty((bs.size, B), dtype=torch.float64, device="cuda")
    b(c, vals)
    xs = torch.from_numpy(np.ascontiguousarray(np.tile(b.interpolation_points[:, None], (1, B)))).cuda()
    y = torch.empty_like(xs)
    e(y, xs, c)
    torch.cuda.synchronize()
    assert float((y - vals).abs().max()) <= 1e-10


@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
def test_config4_full_every_problem(oracle_mod, precision):
    """The uneven workload at its named size -- 4096 problems, 3.47 M points, degrees 1-5, three
    closures, uniform and perturbed meshes -- in one graph launch, every problem against the
    oracle's FP64 build and evaluation: <= 1e-12 relative per problem (coefficients; values
    relative to max(|values|, |coefficients|)), or 10 cond(A) eps for a problem whose matrix is
    ill-conditioned enough to need it."""
    import ddc_b200 as D
    from ddc_b200 import workloads as W

    O = oracle_mod
    D.load_library()
    probs = W.config4()
    w = W.config4_batch(D, probs, precision=precision)
    batch = D.UnevenBatch(w["builders"], w["evaluators"], w["nevals"])
    cu = lambda a: torch.from_numpy(a).cuda()
    info = batch.info
    coefs = torch.full((info.total_coefs,), float("nan"), dtype=torch.float64, device="cuda")
    out = torch.full((info.total_evals,), float("nan"), dtype=torch.float64, device="cuda")
    batch(cu(w["vals"]), cu(w["dlo"]), cu(w["dhi"]), coefs, cu(w["coords"]), out)
    coefs, out = coefs.cpu().numpy(), out.cpu().numpy()
    off = batch.offsets()
    clos = {"periodic": O.PERIODIC, "hermite": O.HERMITE, "greville": O.GREVILLE}
    worst_c = worst_y = 0.0
    for i, p in enumerate(probs):
        b = w["builders"][i]
        per = p["closure"] == "periodic"
        obs = (O.BSplines(p["degree"], per, rmin=0.0, rmax=1.0, ncells=p["ncells"]) if p["uniform"]
               else O.BSplines(p["degree"], per, breaks=p["breaks"]))
        c = clos[p["closure"]]
        ob = O.Builder(obs, b.interpolation_points, c, c)
        herm = p["closure"] == "hermite"
        lo = w["dlo"][off["derivs_lo"][i]:off["derivs_lo"][i + 1]]
        hi = w["dhi"][off["derivs_hi"][i]:off["derivs_hi"][i + 1]]
        ref = ob(w["vals"][off["vals"][i]:off["vals"][i + 1]], lo.reshape(-1, 1) if herm else None,
                 hi.reshape(-1, 1) if herm else None)[:, 0]
        x = w["coords"][off["evals"][i]:off["evals"][i + 1]]
        ev = O.evaluate(obs, x[:, None], ref[:, None])[:, 0]
        ec = np.abs(coefs[off["coefs"][i]:off["coefs"][i + 1]] - ref).max() / np.abs(ref).max()
        # the B-splines sum to one, so a value's error is at most the largest coefficient error:
        # values are compared relative to max(|values|, |coefficients|) (even-degree Hermite
        # closures give boundary coefficients hundreds of times the values they produce)
        ey = np.abs(out[off["evals"][i]:off["evals"][i + 1]] - ev).max() / max(np.abs(ev).max(), np.abs(ref).max())
        if max(ec, ey) > 1e-12:
            tol = 10 * np.linalg.cond(ob.matrix()) * np.finfo(float).eps
            assert max(ec, ey) <= tol, (i, p["ncells"], p["degree"], p["closure"], ec, ey, tol)
        worst_c, worst_y = max(worst_c, ec), max(worst_y, ey)
    print(f"PARITY config4 {precision} 4096 problems worst coefs={worst_c:.2e} values={worst_y:.2e}")
