"""The no-allocation 2D build (ddcb_build2d_static_scratch) against the regular one (ddcb_build2d).

Some callers cannot let a library allocate device memory at call time and cannot pass a workspace
either (their device memory is owned by another allocator, or they run where allocation is not
allowed). For them ddcb_build2d_static_scratch takes its scratch from a fixed array inside the
library. This test calls it through the C-ABI twice in a row (the second call reuses the array
the first one left behind) and checks both results against ddcb_build2d with a stream-ordered
workspace, and that a request larger than the array is refused. The file name makes pytest
collect it last.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

VP = C.c_void_p


def _ptr(t):
    return VP(0 if t is None else t.data_ptr())


def test_static_scratch_build2d_matches_regular_build2d():
    import ddc_b200 as D
    from ddc_b200 import _lib

    L = _lib.load()
    rng = np.random.default_rng(2024)
    # a periodic cubic x Hermite cubic pair on 1024 x 1024 cells: 8.4 MB of scratch per field, so
    # the 10 fields run as three groups through the same scratch
    bx = D.UniformBSplines(3, True, 0.0, 1.0, 1024)
    by = D.UniformBSplines(3, False, 0.0, 1.0, 1024)
    Bx = D.SplineBuilder(bx, None, 0, 0)
    By = D.SplineBuilder(by, None, 1, 1)
    nb = 10
    vals = torch.from_numpy(rng.standard_normal((Bx.npoints, By.npoints, nb))).cuda()
    dmin2 = torch.from_numpy(rng.standard_normal((Bx.npoints, 1, nb))).cuda()
    dmax2 = torch.from_numpy(rng.standard_normal((Bx.npoints, 1, nb))).cuda()
    stream = VP(torch.cuda.current_stream().cuda_stream)

    build2d = L.ddcb_build2d
    build2d.restype = C.c_int
    build2d.argtypes = [VP] * 12 + [C.c_int64, VP, C.c_uint64, VP]
    static2d = L.ddcb_build2d_static_scratch
    static2d.restype = C.c_int
    static2d.argtypes = [VP] * 12 + [C.c_int64, VP]

    ref = torch.zeros((bx.size, by.size, nb), dtype=torch.float64, device="cuda")
    st = build2d(Bx._h, By._h, _ptr(ref), _ptr(vals), None, None, _ptr(dmin2), _ptr(dmax2), None, None, None, None,
                 nb, None, 0, stream)
    assert st == 0, L.ddcb_last_error_message()
    for call in range(2):
        got = torch.full_like(ref, float("nan"))
        st = static2d(Bx._h, By._h, _ptr(got), _ptr(vals), None, None, _ptr(dmin2), _ptr(dmax2), None, None, None, None,
                      nb, stream)
        assert st == 0, f"call {call}: " + L.ddcb_last_error_message().decode()
        torch.cuda.synchronize()
        err = (got - ref).abs().max().item() / ref.abs().max().item()
        assert err <= 1e-12, f"call {call}: relative difference {err:.3e}"


def test_static_scratch_build2d_rejects_oversized_requests():
    import ddc_b200 as D
    from ddc_b200 import _lib

    L = _lib.load()
    # one field of a 3000 x 3000 periodic grid already needs 3003 x 3000 x 8 bytes (72 MB > 48 MiB)
    bx = D.UniformBSplines(3, True, 0.0, 1.0, 3000)
    by = D.UniformBSplines(3, True, 0.0, 1.0, 3000)
    Bx = D.SplineBuilder(bx, None, 0, 0)
    By = D.SplineBuilder(by, None, 0, 0)
    static2d = L.ddcb_build2d_static_scratch
    static2d.restype = C.c_int
    static2d.argtypes = [VP] * 12 + [C.c_int64, VP]
    coefs = torch.zeros(8, dtype=torch.float64, device="cuda")  # never touched: the call is refused first
    vals = torch.zeros(8, dtype=torch.float64, device="cuda")
    st = static2d(Bx._h, By._h, _ptr(coefs), _ptr(vals), None, None, None, None, None, None, None, None, 1,
                  VP(torch.cuda.current_stream().cuda_stream))
    assert st == 5  # DDCB_ERR_UNSUPPORTED
    assert b"static scratch" in L.ddcb_last_error_message()


def test_static_scratch_build2d_hermite_both_dimensions():
    """Hermite closures in both dimensions (derivative slabs along each, the four mixed-derivative
    corner arrays) with a batch large enough that the dimension-2 slabs, sized by the whole batch,
    take a large part of the scratch: the static build equals the workspace build bit for bit (the
    same kernels on the same data), on two calls in a row."""
    import ddc_b200 as D
    from ddc_b200 import _lib

    L = _lib.load()
    rng = np.random.default_rng(7)
    bx = D.UniformBSplines(3, False, 0.0, 1.0, 300)
    by = D.NonUniformBSplines(5, False, np.sort(np.r_[0.0, rng.uniform(0.01, 0.99, 199), 1.0]))
    Bx = D.SplineBuilder(bx, None, 1, 1)
    By = D.SplineBuilder(by, None, 1, 1)
    nb = 150
    n1, n2 = Bx.npoints, By.npoints
    l1, h1, l2, h2 = Bx.s_nbv_xmin, Bx.s_nbv_xmax, By.s_nbv_xmin, By.s_nbv_xmax
    g = lambda *shape: torch.from_numpy(rng.standard_normal(shape)).cuda()
    vals = g(n1, n2, nb)
    d1lo, d1hi, d2lo, d2hi = g(l1, n2, nb), g(h1, n2, nb), g(n1, l2, nb), g(n1, h2, nb)
    m = [g(l1, l2, nb), g(h1, l2, nb), g(l1, h2, nb), g(h1, h2, nb)]
    stream = VP(torch.cuda.current_stream().cuda_stream)
    build2d = L.ddcb_build2d
    build2d.restype = C.c_int
    build2d.argtypes = [VP] * 12 + [C.c_int64, VP, C.c_uint64, VP]
    static2d = L.ddcb_build2d_static_scratch
    static2d.restype = C.c_int
    static2d.argtypes = [VP] * 12 + [C.c_int64, VP]
    args = [_ptr(vals), _ptr(d1lo), _ptr(d1hi), _ptr(d2lo), _ptr(d2hi)] + [_ptr(t) for t in m]
    ref = torch.zeros((bx.size, by.size, nb), dtype=torch.float64, device="cuda")
    st = build2d(Bx._h, By._h, _ptr(ref), *args, nb, None, 0, stream)
    assert st == 0, L.ddcb_last_error_message()
    for call in range(2):
        got = torch.full_like(ref, float("nan"))
        st = static2d(Bx._h, By._h, _ptr(got), *args, nb, stream)
        assert st == 0, f"call {call}: " + L.ddcb_last_error_message().decode()
        torch.cuda.synchronize()
        assert torch.equal(got, ref), f"call {call}"
