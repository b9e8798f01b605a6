"""Adjoint kernels (ddcb_build_adjoint, ddcb_eval_adjoint, ddcb_build_eval_adjoint) and the
torch.autograd binding, against the oracle's FP64 matrices and central finite differences.

The builder is linear, coefs = M (vals, derivs); M is read off the oracle by building unit vectors,
so the builder adjoint must equal M^T (the transpose of the reference's FP64 interpolation map).
The evaluator's coefficient Jacobian E is read off the oracle the same way (unit coefficient
vectors), and the coordinate cotangent must equal g_out times the oracle's next derivative.
Tolerance: max-norm relative error <= 1e-12 (FP64 path), or 10*cond(A)*eps where the system is worse
conditioned. Finite differences (eps = 1e-6, FP64) use the GPU forward itself.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

P, H, HH, G = 0, 1, 2, 3
EX_NULL, EX_CONST = 1, 2


def relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def D():
    import ddc_b200

    ddc_b200.load_library()
    assert torch.cuda.is_available()
    return ddc_b200


def breaks_of(nc, seed):
    rng = np.random.default_rng(seed)
    h = 1.0 / nc
    br = np.arange(nc + 1) * h
    br[1:-1] += (rng.random(nc - 1) - 0.5) * 0.6 * h
    return np.sort(br)


def make_basis(D, O, degree, uniform, periodic, nc, seed=0):
    if uniform:
        return D.UniformBSplines(degree, periodic, 0.0, 1.0, nc), O.BSplines(degree, periodic, rmin=0.0, rmax=1.0, ncells=nc)
    br = breaks_of(nc, seed)
    return D.NonUniformBSplines(degree, periodic, br), O.BSplines(degree, periodic, breaks=br)


def oracle_build_map(O, ob, size):
    """M_v (size x np), M_lo (size x nbv_lo), M_hi (size x nbv_hi): the builder as a matrix."""
    npts, nlo, nhi = ob.npoints, ob.nbv_lo, ob.nbv_hi
    lo = np.zeros((nlo, npts)) if ob.lo == H else None
    hi = np.zeros((nhi, npts)) if ob.hi == H else None
    Mv = ob(np.eye(npts), lo, hi)
    Mlo = Mhi = None
    if ob.lo == H and nlo:
        Mlo = ob(np.zeros((npts, nlo)), np.eye(nlo), None if hi is None else np.zeros((nhi, nlo)))
    if ob.hi == H and nhi:
        Mhi = ob(np.zeros((npts, nhi)), None if lo is None else np.zeros((nlo, nhi)), np.eye(nhi))
    return Mv, Mlo, Mhi


def tol_of(ob):
    A = ob.matrix()
    return max(1e-12, 10 * np.linalg.cond(A) * np.finfo(float).eps)


BUILD_CASES = [
    # degree, uniform, periodic, ncells, lower, upper
    (3, True, True, 64, P, P),
    (3, True, True, 1024, P, P),
    (1, True, False, 20, G, G),
    (2, False, True, 30, P, P),
    (4, True, False, 40, G, H),
    (3, False, False, 33, HH, G),
    (5, False, False, 48, H, H),
    (5, False, False, 256, H, H),
    (4, False, True, 50, P, P),
    (5, True, True, 37, P, P),
]


@pytest.mark.parametrize("case", BUILD_CASES, ids=[f"d{c[0]}{'u' if c[1] else 'n'}{'p' if c[2] else 'b'}{c[3]}_{c[4]}{c[5]}" for c in BUILD_CASES])
def test_build_adjoint_is_transpose_of_interpolation_map(D, oracle_mod, case):
    O = oracle_mod
    degree, uniform, periodic, nc, lo, hi = case
    bs, obs = make_basis(D, O, degree, uniform, periodic, nc, seed=nc)
    b = D.SplineBuilder(bs, None, lo, hi)
    ob = O.Builder(obs, b.interpolation_points, lo, hi)
    size = b.info.size
    Mv, Mlo, Mhi = oracle_build_map(O, ob, size)
    B = 13
    rng = np.random.default_rng(7)
    gc = rng.standard_normal((size, B))
    g_vals = torch.full((b.npoints, B), float("nan"), dtype=torch.float64, device="cuda")
    g_lo = torch.full((b.s_nbv_xmin, B), float("nan"), dtype=torch.float64, device="cuda") if Mlo is not None else None
    g_hi = torch.full((b.s_nbv_xmax, B), float("nan"), dtype=torch.float64, device="cuda") if Mhi is not None else None
    b.adjoint(cuda(gc), g_vals, g_lo, g_hi)
    torch.cuda.synchronize()
    tol = tol_of(ob)
    assert relerr(g_vals.cpu().numpy(), Mv.T @ gc) <= tol
    if Mlo is not None:
        assert relerr(g_lo.cpu().numpy(), Mlo.T @ gc) <= tol
    if Mhi is not None:
        assert relerr(g_hi.cpu().numpy(), Mhi.T @ gc) <= tol


def eval_jacobian(O, obs, x, order, ex_lo, ex_hi):
    """E (m x size): d out / d coefs of one line at coordinates x (oracle, unit coefficient vectors)."""
    size = obs.size
    X = np.repeat(x[:, None], size, axis=1)
    return O.evaluate(obs, X, np.eye(size), order=order, ex_lo=ex_lo, ex_hi=ex_hi)


def wrapped(x, periodic):
    return x - np.floor(x) if periodic else x


EVAL_CASES = [
    # degree, uniform, periodic, ncells, ex_lo, ex_hi, order
    (3, True, True, 64, 0, 0, 0),
    (3, True, True, 64, 0, 0, 1),
    (5, False, False, 40, EX_NULL, EX_CONST, 0),
    (5, False, False, 40, EX_CONST, EX_NULL, 1),
    (1, True, False, 16, EX_CONST, EX_CONST, 0),
    (2, False, True, 25, 0, 0, 0),
    (4, True, False, 30, EX_NULL, EX_NULL, 0),
    (4, False, False, 30, EX_NULL, EX_NULL, 1),
    (1, False, True, 12, 0, 0, 1),
]


@pytest.mark.parametrize("case", EVAL_CASES, ids=[f"d{c[0]}{'u' if c[1] else 'n'}{'p' if c[2] else 'b'}_ex{c[4]}{c[5]}_o{c[6]}" for c in EVAL_CASES])
def test_eval_adjoint_matches_oracle_jacobian(D, oracle_mod, case):
    O = oracle_mod
    degree, uniform, periodic, nc, ex_lo, ex_hi, order = case
    bs, obs = make_basis(D, O, degree, uniform, periodic, nc, seed=3 * nc)
    ev = D.SplineEvaluator(bs, ex_lo or 1, ex_hi or 1)
    size = bs.size
    rng = np.random.default_rng(11)
    B, m = 9, 37
    x = rng.random((m, B)) * 1.2 - 0.1 if order == 0 else rng.random((m, B))
    coefs = rng.standard_normal((size, B))
    gy = rng.standard_normal((m, B))
    g_c = torch.full((size, B), float("nan"), dtype=torch.float64, device="cuda")
    g_x = torch.full((m, B), float("nan"), dtype=torch.float64, device="cuda")
    ev.adjoint(cuda(x), cuda(gy), g_c, cuda(coefs), g_x, order=order)
    torch.cuda.synchronize()
    g_c, g_x = g_c.cpu().numpy(), g_x.cpu().numpy()
    oex_lo = ex_lo if not periodic else 0
    oex_hi = ex_hi if not periodic else 0
    for j in range(B):
        E = eval_jacobian(O, obs, x[:, j], None if order == 0 else order, oex_lo, oex_hi)
        assert relerr(g_c[:, j], E.T @ gy[:, j]) <= 1e-12, f"line {j}"
        # dy/dx: the next derivative inside the domain, 0 where the extrapolation holds y fixed
        xi = wrapped(x[:, j], periodic)
        if degree >= order + 1:
            dnext = O.evaluate(obs, xi[:, None], coefs[:, j:j + 1], order=order + 1)[:, 0]
        else:
            dnext = np.zeros(m)
        if order == 0 and not periodic:
            dnext = np.where((xi < 0.0) | (xi > 1.0), 0.0, dnext)
        ref = gy[:, j] * dnext
        scale = max(np.abs(ref).max(), np.abs(gy[:, j]).max() * np.abs(coefs[:, j]).max() * nc)
        assert np.abs(g_x[:, j] - ref).max() <= 1e-12 * scale, f"line {j}"


FUSED_CASES = [
    (3, True, True, 1024, P, P, 0),
    (3, True, True, 200, P, P, 1),
    (5, False, False, 128, H, H, 1),
    (5, False, False, 128, H, H, 0),
    (4, True, False, 60, G, H, 0),
    (2, True, True, 50, P, P, 0),
]


@pytest.mark.parametrize("case", FUSED_CASES, ids=[f"d{c[0]}{'u' if c[1] else 'n'}{'p' if c[2] else 'b'}{c[3]}_{c[4]}{c[5]}_o{c[6]}" for c in FUSED_CASES])
def test_fused_build_eval_adjoint(D, oracle_mod, case):
    O = oracle_mod
    degree, uniform, periodic, nc, lo, hi, order = case
    bs, obs = make_basis(D, O, degree, uniform, periodic, nc, seed=5 * nc)
    b = D.SplineBuilder(bs, None, lo, hi)
    ev = D.SplineEvaluator(bs, 2, 2)
    ob = O.Builder(obs, b.interpolation_points, lo, hi)
    size = b.info.size
    Mv, Mlo, Mhi = oracle_build_map(O, ob, size)
    rng = np.random.default_rng(5)
    B, m = 17, 64
    x = rng.random((m, B))
    coefs = rng.standard_normal((size, B))
    gy = rng.standard_normal((m, B))
    g_vals = torch.full((b.npoints, B), float("nan"), dtype=torch.float64, device="cuda")
    g_x = torch.full((m, B), float("nan"), dtype=torch.float64, device="cuda")
    g_lo = torch.full((b.s_nbv_xmin, B), float("nan"), dtype=torch.float64, device="cuda") if Mlo is not None else None
    g_hi = torch.full((b.s_nbv_xmax, B), float("nan"), dtype=torch.float64, device="cuda") if Mhi is not None else None
    fused = b.build_and_evaluate_adjoint(ev, cuda(x), cuda(coefs), cuda(gy), g_vals, g_x, g_lo, g_hi, order=order)
    torch.cuda.synchronize()
    # two-call composition through the C-ABI
    g_c2 = torch.empty((size, B), dtype=torch.float64, device="cuda")
    g_x2 = torch.empty((m, B), dtype=torch.float64, device="cuda")
    ev.adjoint(cuda(x), cuda(gy), g_c2, cuda(coefs), g_x2, order=order)
    g_vals2 = torch.empty_like(g_vals)
    b.adjoint(g_c2, g_vals2)
    torch.cuda.synchronize()
    tol = tol_of(ob)
    gc_ref = np.stack([eval_jacobian(O, obs, x[:, j], None if order == 0 else order, 2, 2).T @ gy[:, j]
                       for j in range(B)], axis=1)
    assert relerr(g_vals.cpu().numpy(), Mv.T @ gc_ref) <= tol
    assert relerr(g_vals2.cpu().numpy(), Mv.T @ gc_ref) <= tol
    assert relerr(g_x.cpu().numpy(), g_x2.cpu().numpy()) <= 1e-13
    if Mlo is not None:
        assert relerr(g_lo.cpu().numpy(), Mlo.T @ gc_ref) <= tol
    if Mhi is not None:
        assert relerr(g_hi.cpu().numpy(), Mhi.T @ gc_ref) <= tol
    if (periodic and degree == 3) or (not periodic and degree == 5):
        assert fused


def config5_inputs(B, seed=0xDDC0 + 5):
    from ddc_b200 import workloads as W

    nc = 1024
    x = np.arange(nc) / nc
    k = np.floor(W.splitmix_uniform(seed, 1, B) * 8).astype(np.int64) + 1
    ph = W.splitmix_uniform(seed, 2, B) * 2 * np.pi
    vals = W.cos_family(x[:, None], k[None, :], ph[None, :])
    m = 1024
    coords = W.splitmix_uniform(seed, 3, m * B).reshape(m, B)
    u1 = W.splitmix_uniform(seed, 4, m * B)
    u2 = W.splitmix_uniform(seed, 5, m * B)
    w = (np.sqrt(-2.0 * np.log(np.maximum(u1, 1e-300))) * np.cos(2 * np.pi * u2)).reshape(m, B)
    return vals, coords, w


def test_autograd_finite_differences_config5_subset(D):
    """L = sum w_i s(x_i) on periodic cubic, 1024 cells: autograd gradients vs central differences
    (eps = 1e-6, FP64) on random entries of vals and coords, for a subset of 8 lines."""
    from ddc_b200.autograd import build_evaluate

    bs = D.UniformBSplines(3, True, 0.0, 1.0, 1024)
    b = D.SplineBuilder(bs)
    ev = D.SplineEvaluator(bs)
    vals, coords, w = config5_inputs(8)
    v = cuda(vals).requires_grad_(True)
    x = cuda(coords).requires_grad_(True)
    wt = cuda(w)
    L = (build_evaluate(v, x, b, ev) * wt).sum()
    L.backward()
    gv, gx = v.grad.cpu().numpy(), x.grad.cpu().numpy()

    def loss(vn, xn):
        with torch.no_grad():
            return float((build_evaluate(cuda(vn), cuda(xn), b, ev) * wt).sum())

    rng = np.random.default_rng(1)
    eps = 1e-6
    for _ in range(16):
        i, j = rng.integers(0, 1024), rng.integers(0, 8)
        vp, vm = vals.copy(), vals.copy()
        vp[i, j] += eps
        vm[i, j] -= eps
        fd = (loss(vp, coords) - loss(vm, coords)) / (2 * eps)
        assert abs(fd - gv[i, j]) <= 1e-6 * max(1.0, abs(gv[i, j])), (i, j, fd, gv[i, j])
    for _ in range(16):
        i, j = rng.integers(0, 1024), rng.integers(0, 8)
        xp, xm = coords.copy(), coords.copy()
        xp[i, j] += eps
        xm[i, j] -= eps
        fd = (loss(vals, xp) - loss(vals, xm)) / (2 * eps)
        assert abs(fd - gx[i, j]) <= 1e-5 * max(1.0, abs(gx[i, j])), (i, j, fd, gx[i, j])


def test_autograd_hermite_derivative_cotangents(D):
    """Hermite quintic: the cotangents of the boundary derivatives through autograd vs differences."""
    from ddc_b200.autograd import build_evaluate

    br = breaks_of(64, 2)
    bs = D.NonUniformBSplines(5, False, br)
    b = D.SplineBuilder(bs, None, H, H)
    ev = D.SplineEvaluator(bs, 2, 2)
    rng = np.random.default_rng(3)
    B, m = 4, 50
    vals = rng.standard_normal((b.npoints, B))
    dlo = rng.standard_normal((2, B))
    dhi = rng.standard_normal((2, B))
    coords = rng.random((m, B))
    w = cuda(rng.standard_normal((m, B)))
    tv, tlo, thi = (cuda(a).requires_grad_(True) for a in (vals, dlo, dhi))
    L = (build_evaluate(tv, cuda(coords), b, ev, 1, tlo, thi) * w).sum()
    L.backward()

    def loss(lo_, hi_):
        with torch.no_grad():
            return float((build_evaluate(cuda(vals), cuda(coords), b, ev, 1, cuda(lo_), cuda(hi_)) * w).sum())

    eps = 1e-6
    for arr, grad, which in ((dlo, tlo.grad, 0), (dhi, thi.grad, 1)):
        g = grad.cpu().numpy()
        for r in range(2):
            for j in range(B):
                p, mn = arr.copy(), arr.copy()
                p[r, j] += eps
                mn[r, j] -= eps
                fd = (loss(p, dhi) - loss(mn, dhi)) / (2 * eps) if which == 0 else \
                     (loss(dlo, p) - loss(dlo, mn)) / (2 * eps)
                assert abs(fd - g[r, j]) <= 1e-5 * max(1.0, abs(g[r, j])), (which, r, j, fd, g[r, j])


def test_adjoint_dot_product_identity_config5_full(D):
    """At the full config-5 size (1024 cells, 2^16 lines): <g_vals, dv> = <g_out, J dv>, where J dv is
    the forward build + evaluate of a random perturbation (the map vals -> out is linear)."""
    bs = D.UniformBSplines(3, True, 0.0, 1.0, 1024)
    b = D.SplineBuilder(bs)
    ev = D.SplineEvaluator(bs)
    B, m = 1 << 16, 1024
    gen = torch.Generator(device="cuda").manual_seed(5)
    x = torch.rand((m, B), dtype=torch.float64, device="cuda", generator=gen)
    gy = torch.randn((m, B), dtype=torch.float64, device="cuda", generator=gen)
    dv = torch.randn((1024, B), dtype=torch.float64, device="cuda", generator=gen)
    coefs = torch.empty((b.info.size, B), dtype=torch.float64, device="cuda")
    y = torch.empty((m, B), dtype=torch.float64, device="cuda")
    b.build_and_evaluate(ev, coefs, dv, x, y)
    g_vals = torch.empty((1024, B), dtype=torch.float64, device="cuda")
    g_x = torch.empty((m, B), dtype=torch.float64, device="cuda")
    assert b.build_and_evaluate_adjoint(ev, x, coefs, gy, g_vals, g_x)
    lhs = float((g_vals * dv).sum())
    rhs = float((gy * y).sum())
    scale = float((g_vals.abs() * dv.abs()).sum())
    assert abs(lhs - rhs) <= 1e-13 * scale, (lhs, rhs, scale)
    # g_x = g_out * s'(x), checked against the evaluator's derivative on a slice of lines
    d1 = torch.empty((m, 4096), dtype=torch.float64, device="cuda")
    ev.deriv(1, d1, x[:, :4096].contiguous(), coefs[:, :4096].contiguous())
    ref = gy[:, :4096] * d1
    assert float((g_x[:, :4096] - ref).abs().max()) <= 1e-12 * float(ref.abs().max())
