"""Differentiable gather and scatter: torch.autograd.Function over the node kernels.

The reference has no autograd; these functions change how the method is used, not its
arithmetic. With W_k(x) the B-spline weight of node k at position x:

    gather(f, x)_c,i  = sum_k W_k(x_i) f_k,c
    scatter(x, v)_k,c = sum_i W_k(x_i) v_c,i

are adjoint to each other (<scatter(x, v), f> = <v, gather(f, x)>), so

- gather, backward for the field: a scatter of the incoming gradient;
- scatter, backward for the deposited values: a gather of the incoming gradient;
- either, backward for the positions: the gather with the weight derivatives
  W_k'(x) (``mpf_gather_grad``), weighted by the cotangent (gather) or by the values
  (scatter), in position units (the 1 / cell factor included).

The derivative of a B-spline of degree p is B_{p-1}(. + 1/2) - B_{p-1}(. - 1/2)
(src/mpifield/splines.py:9,77). Where a bounded or clamped axis clamps a position the
weights do not move with it, and the position gradient there is zero.

A scatter skips markers whose values are all zero without reading their positions
(scatter_quadratic_3d_cuda.cu:32-38); the backward of such a scatter reads every
position, so a dead marker's position must be finite when its gradient is wanted.
"""

from __future__ import annotations

import torch

from mpifield_b200 import kernels as K
from mpifield_b200 import _lib
from mpifield_b200.sorting import _kind_of


def _geometry(grid) -> tuple:
    """A geometry tuple from a ``BlockGrid`` (its ``geometry``) or a tuple."""
    return tuple(grid.geometry) if hasattr(grid, "geometry") else tuple(grid)


def _rows(t: torch.Tensor) -> torch.Tensor:
    return t.view(1, -1) if t.dim() == 1 else t


class _Gather(torch.autograd.Function):
    @staticmethod
    def forward(ctx, field, positions, kind, degree, geometry):
        ncomp = field.shape[-1]
        result = torch.empty((ncomp, positions.shape[-1]), dtype=field.dtype, device=field.device)
        K.gather(kind, degree, positions, field, result, geometry)
        ctx.save_for_backward(field, positions)
        ctx.meta = (kind, degree, geometry)
        return result

    @staticmethod
    def backward(ctx, grad):
        field, positions = ctx.saved_tensors
        kind, degree, geometry = ctx.meta
        grad = grad.contiguous()
        d_field = d_pos = None
        if ctx.needs_input_grad[0]:
            d_field = torch.zeros_like(field)
            K.scatter(kind, degree, positions, grad, d_field, geometry)
        if ctx.needs_input_grad[1]:
            d_pos = K.gather_grad(kind, degree, positions, field, grad, geometry)
        return d_field, d_pos, None, None, None


class _Scatter(torch.autograd.Function):
    @staticmethod
    def forward(ctx, positions, values, kind, degree, geometry, shape):
        field = torch.zeros(shape, dtype=values.dtype, device=values.device)
        K.scatter(kind, degree, positions, values, field, geometry)
        ctx.save_for_backward(positions, values)
        ctx.meta = (kind, degree, geometry)
        return field

    @staticmethod
    def backward(ctx, grad):
        positions, values = ctx.saved_tensors
        kind, degree, geometry = ctx.meta
        grad = grad.contiguous()
        d_pos = d_values = None
        if ctx.needs_input_grad[1]:
            d_values = torch.empty_like(values)
            K.gather(kind, degree, positions, grad, d_values, geometry)
        if ctx.needs_input_grad[0]:
            d_pos = K.gather_grad(kind, degree, positions, grad, values, geometry)
        return d_pos, d_values, None, None, None, None


def gather(field: torch.Tensor, positions: torch.Tensor, weighting, grid) -> torch.Tensor:
    """``(ncomp, N)``: the field at the markers, differentiable in ``field`` and ``positions``.

    ``field`` is ``extent + (ncomp,)``, ``positions`` ``(ndim, N)``; ``weighting`` a built-in
    weighting (``LINEAR``, ``QUADRATIC``, ``CUBIC``, ``spline_weighting(p)``) or a
    ``(kind, degree)`` pair; ``grid`` a ``BlockGrid`` or a geometry tuple.
    """
    kind, degree = _kind_of(weighting)
    return _Gather.apply(field, positions, kind, degree, _geometry(grid))


def scatter(positions: torch.Tensor, values: torch.Tensor, weighting, grid) -> torch.Tensor:
    """A new field ``extent + (ncomp,)`` holding the deposit of ``values`` ``(ncomp, N)`` (or
    ``(N,)``), differentiable in ``positions`` and ``values``."""
    kind, degree = _kind_of(weighting)
    geometry = _geometry(grid)
    _, _, num, code, _ = _lib.geometry_arrays(geometry)
    values = _rows(values)
    shape = K._extent(num, code, degree) + (values.shape[0],)
    return _Scatter.apply(positions, values, kind, degree, geometry, shape)
