"""torch.autograd binding of the batched build + evaluate step, backed by the adjoint kernels.

`BuildEvaluate.apply(vals, coords, builder, evaluator, order, derivs_xmin, derivs_xmax)` returns the
values (order 0) or first derivatives (order 1) at `coords` of the splines interpolating `vals`
(SplineBuilder::operator() followed by SplineEvaluator::operator() / deriv, one fused kernel when
one exists). Its backward runs ddcb_build_eval_adjoint: the transposed solve for the cotangents of
`vals` (and of the Hermite derivatives) and the spline derivative for those of `coords`. The
interpolation dimension is dimension 0 of every tensor; the other dimensions are batch dimensions.
"""
from __future__ import annotations

import torch

from .splines import SplineBuilder, SplineEvaluator


class BuildEvaluate(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vals, coords, builder: SplineBuilder, evaluator: SplineEvaluator, order: int = 0,
                derivs_xmin=None, derivs_xmax=None):
        vals = vals.contiguous()
        coords = coords.contiguous()
        batch = tuple(vals.shape[1:])
        coefs = torch.empty((builder.info.size,) + batch, dtype=torch.float64, device=vals.device)
        out = torch.empty_like(coords)
        builder.build_and_evaluate(evaluator, coefs, vals, coords, out,
                                   None if derivs_xmin is None else derivs_xmin.contiguous(),
                                   None if derivs_xmax is None else derivs_xmax.contiguous(), order=order)
        ctx.save_for_backward(coords, coefs)
        ctx.builder, ctx.evaluator, ctx.order = builder, evaluator, order
        ctx.shapes = (vals.shape, None if derivs_xmin is None else derivs_xmin.shape,
                      None if derivs_xmax is None else derivs_xmax.shape)
        return out

    @staticmethod
    def backward(ctx, g_out):
        coords, coefs = ctx.saved_tensors
        vshape, lo_shape, hi_shape = ctx.shapes
        need = ctx.needs_input_grad
        dev = coords.device
        g_vals = torch.empty(vshape, dtype=torch.float64, device=dev)
        g_coords = torch.empty_like(coords) if need[1] else None
        g_lo = torch.empty(lo_shape, dtype=torch.float64, device=dev) if (lo_shape is not None and need[5]) else None
        g_hi = torch.empty(hi_shape, dtype=torch.float64, device=dev) if (hi_shape is not None and need[6]) else None
        ctx.builder.build_and_evaluate_adjoint(ctx.evaluator, coords, coefs if need[1] else None, g_out.contiguous(),
                                               g_vals, g_coords, g_lo, g_hi, order=ctx.order)
        return (g_vals if need[0] else None), g_coords, None, None, None, g_lo, g_hi


def build_evaluate(vals, coords, builder: SplineBuilder, evaluator: SplineEvaluator, order: int = 0,
                   derivs_xmin=None, derivs_xmax=None):
    """Differentiable build + evaluate (see BuildEvaluate)."""
    return BuildEvaluate.apply(vals, coords, builder, evaluator, order, derivs_xmin, derivs_xmax)
