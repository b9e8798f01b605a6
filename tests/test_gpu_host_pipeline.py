"""The host pipeline (build + evaluate on host arrays, batch slices overlapped on three streams)
against the device path on the same data.

The pipeline runs the same kernels on slices of the batch, and a line's result does not depend on
the other lines of its launch, so the outputs must equal the device path's bit for bit: ragged
last slices, both host layouts, the optional coefficient copy-out, back-to-back runs that reuse
the device buffers before the host has synchronized, and pageable host memory.
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


def quintic_hermite(D):
    from ddc_b200 import workloads

    br = workloads.config2_breaks(256)
    bs = D.NonUniformBSplines(5, False, br)
    pts = D.greville_points(bs, 1, 1)
    return bs, D.SplineBuilder(bs, pts, 1, 1), D.SplineEvaluator(bs), pts


def device_reference(builder, ev, vals, x, dlo, dhi, order, dim):
    cu = lambda t: None if t is None else t.cuda()
    coefs_shape = list(vals.shape)
    coefs_shape[dim] = ev.bsplines.size
    coefs = torch.empty(coefs_shape, dtype=torch.float64, device="cuda")
    out = torch.empty(x.shape, dtype=torch.float64, device="cuda")
    builder.build_and_evaluate(ev, coefs, cu(vals), cu(x), out, cu(dlo), cu(dhi), order=order, dim=dim)
    torch.cuda.synchronize()
    return coefs.cpu(), out.cpu()


@pytest.mark.parametrize("B,slice_lines", [(3000, 1024), (1024, 1024), (7, 4), (1, 8)])
def test_rows_layout_matches_device_path(D, B, slice_lines):
    bs, builder, ev, pts = quintic_hermite(D)
    g = torch.Generator().manual_seed(B)
    m = 200
    vals = torch.randn((len(pts), B), dtype=torch.float64, generator=g).pin_memory()
    dlo = torch.randn((2, B), dtype=torch.float64, generator=g).pin_memory()
    dhi = torch.randn((2, B), dtype=torch.float64, generator=g).pin_memory()
    x = torch.rand((m, B), dtype=torch.float64, generator=g).pin_memory()
    ref_c, ref_y = device_reference(builder, ev, vals, x, dlo, dhi, 1, 0)
    pipe = D.HostPipeline(builder, ev, m, order=1, slice_lines=slice_lines)
    out = torch.full((m, B), float("nan"), dtype=torch.float64).pin_memory()
    coefs = torch.full((bs.size, B), float("nan"), dtype=torch.float64).pin_memory()
    pipe(vals, x, out, dlo, dhi, coefs)
    torch.cuda.synchronize()
    assert torch.equal(out, ref_y)
    assert torch.equal(coefs, ref_c)


def test_lines_layout_periodic_values(D):
    """(batch, x) host tensors (dim=1), periodic uniform cubic, values, coefficients copied out."""
    bs = D.UniformBSplines(3, True, 0.0, 1.0, 300)
    builder, ev = D.SplineBuilder(bs), D.SplineEvaluator(bs)
    B, m = 2500, 333
    g = torch.Generator().manual_seed(5)
    vals = torch.randn((B, builder.npoints), dtype=torch.float64, generator=g).pin_memory()
    x = (3 * torch.rand((B, m), dtype=torch.float64, generator=g) - 1).pin_memory()
    ref_c, ref_y = device_reference(builder, ev, vals, x, None, None, 0, 1)
    pipe = D.HostPipeline(builder, ev, m, order=0, slice_lines=1000)
    out = torch.empty((B, m), dtype=torch.float64).pin_memory()
    coefs = torch.empty((B, bs.size), dtype=torch.float64).pin_memory()
    pipe(vals, x, out, spline=coefs, dim=1)
    torch.cuda.synchronize()
    assert torch.equal(out, ref_y)
    assert torch.equal(coefs, ref_c)


def test_back_to_back_runs_and_pageable_memory(D):
    """Two runs queued without a host synchronization in between reuse the device buffer sets;
    the second run's inputs must not overwrite the first's before its kernels read them."""
    bs, builder, ev, pts = quintic_hermite(D)
    B, m = 4100, 64
    g = torch.Generator().manual_seed(11)
    runs = []
    for r in range(3):
        vals = torch.randn((len(pts), B), dtype=torch.float64, generator=g)
        dlo = torch.randn((2, B), dtype=torch.float64, generator=g)
        dhi = torch.randn((2, B), dtype=torch.float64, generator=g)
        x = torch.rand((m, B), dtype=torch.float64, generator=g)
        if r < 2:
            vals, dlo, dhi, x = (t.pin_memory() for t in (vals, dlo, dhi, x))
        runs.append((vals, dlo, dhi, x))
    refs = [device_reference(builder, ev, v, x, lo, hi, 1, 0)[1] for v, lo, hi, x in runs]
    pipe = D.HostPipeline(builder, ev, m, order=1, slice_lines=1000)
    outs = [torch.empty((m, B), dtype=torch.float64).pin_memory() for _ in runs]
    for (v, lo, hi, x), out in zip(runs, outs):
        pipe(v, x, out, lo, hi)
    torch.cuda.synchronize()
    for out, ref in zip(outs, refs):
        assert torch.equal(out, ref)


def test_argument_errors(D):
    bs, builder, ev, pts = quintic_hermite(D)
    pipe = D.HostPipeline(builder, ev, 16, order=1, slice_lines=64)
    B = 10
    vals = torch.zeros((len(pts), B), dtype=torch.float64)
    x = torch.zeros((16, B), dtype=torch.float64)
    out = torch.zeros((16, B), dtype=torch.float64)
    d = torch.zeros((2, B), dtype=torch.float64)
    with pytest.raises(TypeError):
        pipe(vals.cuda(), x, out, d, d)
    with pytest.raises(D.DdcbError):
        pipe(vals, x, out)  # the HERMITE closures need derivatives
    with pytest.raises(D.DdcbError):
        pipe(vals, torch.zeros((15, B), dtype=torch.float64), torch.zeros((15, B), dtype=torch.float64), d, d)
    # a batch in groups of rows (batch dimensions on both sides of the interest dimension) is
    # neither rows nor contiguous lines
    v3 = torch.zeros((2, len(pts), B // 2), dtype=torch.float64)
    x3 = torch.zeros((2, 16, B // 2), dtype=torch.float64)
    d3 = torch.zeros((2, 2, B // 2), dtype=torch.float64)
    with pytest.raises(D.DdcbError):
        pipe(v3, x3, x3.clone(), d3, d3, dim=1)
    with pytest.raises(D.DdcbError):
        D.HostPipeline(builder, ev, 16, order=6)
    with pytest.raises(D.DdcbError):
        D.HostPipeline(builder, ev, 16, slice_lines=0)
