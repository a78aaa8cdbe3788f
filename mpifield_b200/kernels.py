"""The kernel callables of the B200 backend, with the arguments of mpifield's kernels.

mpifield's weightings call their kernels as (src/mpifield/weighting.py:22-38,
src/mpifield/edges.py:23-31)::

    scatter(positions, values, field, *geometry)               # adds into field
    gather(positions, field, result, *geometry)                 # overwrites result
    deposit_paths(start, end, charges, edges, *geometry)        # adds into edges

with ``geometry = (*lower, *cell_size, *num_nodes, *code)`` and, for the spline kernels,
a trailing ``degree``. The callables here take the same arguments as torch tensors on a
CUDA device (float64, or float32 for the single-precision variant) and launch the
sm_100a kernels of ``libmpifield_b200.so`` on torch's current stream, asynchronously.
`KERNELS` maps the reference's kernel names (src/mpifield/kernels/catalog.py:51-93) to
them; the linear 1D deposit also takes the reference's ``(N,)`` single-component arrays
and the linear 3D kernels its ``(nx * ny * nz, ncomp)`` row fields.

Marker arrays are ``(rows, N)`` with a unit column stride and any row stride
(``storage[:, :n]``); a copy is made only for other layouts (or another dtype), and a
non-contiguous output is written through a contiguous copy, as
``cunumpy.kernels.kernel_output`` does for the reference.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from mpifield_b200 import _lib


def _marker_rows(t: torch.Tensor, rows: int, name: str, dtype: torch.dtype) -> tuple[torch.Tensor, int]:
    """``t`` as ``(rows, N)`` with unit column stride, and its row stride in elements."""
    if t.dim() == 1:
        t = t.reshape(1, -1)
    if t.dim() != 2 or t.shape[0] != rows:
        raise ValueError(f"{name} must be ({rows}, N), got {tuple(t.shape)}")
    if t.dtype != dtype:
        t = t.to(dtype)
    if t.shape[1] > 1 and t.stride(1) != 1:
        t = t.contiguous()
    if t.shape[0] > 1 and t.stride(0) < t.shape[1]:
        t = t.contiguous()
    stride = t.stride(0) if t.shape[0] > 1 else t.shape[1]
    return t, int(stride)


class _Output:
    """A contiguous working copy of an output tensor, written back on exit if needed."""

    def __init__(self, target: torch.Tensor, dtype: torch.dtype, accumulate: bool):
        self.target = target
        self.direct = target.is_contiguous() and target.dtype == dtype
        if self.direct:
            self.work = target
        elif accumulate:
            self.work = target.to(dtype).contiguous()
        else:
            self.work = torch.empty(target.shape, dtype=dtype, device=target.device)

    def finish(self) -> None:
        if not self.direct:
            self.target.copy_(self.work)


def _extent(num, code, degree) -> tuple[int, ...]:
    return tuple(int(n) + (degree - 1 if int(c) == 2 else 0) for n, c in zip(num, code))


def _field_shape(field: torch.Tensor, extent: tuple[int, ...], name: str) -> torch.Tensor:
    """``field`` as ``extent + (ncomp,)``; a 1-D field or the linear 3D rows are reshaped."""
    ndim = len(extent)
    if field.dim() == ndim:
        field = field.unsqueeze(-1)
    elif ndim == 3 and field.dim() == 2 and field.shape[0] == extent[0] * extent[1] * extent[2]:
        field = field.view(*extent, field.shape[1]) if field.is_contiguous() else field.reshape(*extent, field.shape[1])
    if tuple(field.shape[:-1]) != extent or field.dim() != ndim + 1:
        raise ValueError(f"{name} on this grid is {extent} + (ncomp,), got {tuple(field.shape)}")
    return field


@dataclass(frozen=True)
class NodeKernel:
    """A gather or a scatter with the arithmetic of one reference stencil kind."""

    op: str  # "gather" or "scatter"
    kind: int
    ndim: int
    takes_degree: bool
    fixed_degree: int | None = None
    tuning: _lib.Tuning | None = None

    def __call__(self, *args) -> None:
        if self.takes_degree:
            *args, degree = args
            degree = int(degree)
        else:
            degree = int(self.fixed_degree)
        if self.op == "gather":
            positions, field, result, *geometry = args
            gather(self.kind, degree, positions, field, result, geometry, self.tuning)
        else:
            positions, values, field, *geometry = args
            scatter(self.kind, degree, positions, values, field, geometry, self.tuning)


def _tile_args(order, ndim: int, device):
    """The tile shape (ctypes array) and tile starts of a `sorting.TileOrder`, checked."""
    starts = order.tile_start
    if starts.device != device or starts.dtype != torch.int64 or not starts.is_contiguous():
        raise ValueError("order.tile_start must be a contiguous int64 tensor on the markers' device")
    if len(order.tile) != ndim or starts.numel() != order.num_tiles + 2:
        raise ValueError(f"a tile order of {len(order.tile)} axes and {starts.numel()} starts for a {ndim}D grid")
    return (C.c_int32 * ndim)(*(int(v) for v in order.tile)), starts.data_ptr()


def gather(kind: int, degree: int, positions: torch.Tensor, field: torch.Tensor, result: torch.Tensor,
           geometry, tuning: _lib.Tuning | None = None, order=None) -> None:
    """result(c, i) = sum_k W_k(x_i) field(k, c), overwriting ``result`` (ncomp, N).

    ``order``: the `sorting.TileOrder` whose rank order the markers are in, for
    ``mpf_gather_tiles`` (the same result, whatever the markers' order).
    """
    lower, cell, num, code, ndim = _lib.geometry_arrays(geometry)
    device = _lib.require_cuda(positions, field, result)
    dtype = field.dtype
    dcode = _lib.dtype_code(dtype)
    field = _field_shape(field, _extent(num, code, degree), "field")
    if not field.is_contiguous():
        field = field.contiguous()
    ncomp = field.shape[-1]
    pos, ps = _marker_rows(positions, ndim, "positions", dtype)
    n = pos.shape[1]
    if result.dim() == 1:
        result = result.view(1, -1)
    if tuple(result.shape) != (ncomp, n):
        raise ValueError(f"result must be ({ncomp}, {n}), got {tuple(result.shape)}")
    rows_ok = result.dtype == dtype and (n <= 1 or result.stride(1) == 1) and (ncomp == 1 or result.stride(0) >= n)
    out = result if rows_ok else torch.empty((ncomp, n), dtype=dtype, device=device)
    rs = out.stride(0) if ncomp > 1 else n
    tune = C.byref(tuning) if tuning is not None else None
    if order is None:
        status = _lib.library().mpf_gather(
            kind, degree, ndim, pos.data_ptr(), ps, n, field.data_ptr(), ncomp, out.data_ptr(), rs,
            lower, cell, num, code, dcode, tune, _lib.stream_of(device))
    else:
        tile, starts = _tile_args(order, ndim, device)
        status = _lib.library().mpf_gather_tiles(
            kind, degree, ndim, pos.data_ptr(), ps, n, field.data_ptr(), ncomp, out.data_ptr(), rs,
            lower, cell, num, code, tile, starts, dcode, tune, _lib.stream_of(device))
    _lib.check(status, "gather")
    if out is not result:
        result.copy_(out)


def scatter(kind: int, degree: int, positions: torch.Tensor, values: torch.Tensor, field: torch.Tensor,
            geometry, tuning: _lib.Tuning | None = None, order=None) -> None:
    """field(k, c) += sum_i W_k(x_i) values(c, i); dead markers (all values zero) skipped.

    ``order``: the `sorting.TileOrder` whose rank order the markers are in (positions and
    values permuted by ``order.order``), for ``mpf_scatter_tiles``; the result is the same
    up to the order of the floating-point adds, whatever the markers' order.
    """
    lower, cell, num, code, ndim = _lib.geometry_arrays(geometry)
    device = _lib.require_cuda(positions, values, field)
    dtype = field.dtype
    dcode = _lib.dtype_code(dtype)
    shaped = _field_shape(field, _extent(num, code, degree), "field")
    ncomp = shaped.shape[-1]
    pos, ps = _marker_rows(positions, ndim, "positions", dtype)
    vals, vs = _marker_rows(values, ncomp, "values", dtype)
    if vals.shape[1] != pos.shape[1]:
        raise ValueError(f"{pos.shape[1]} positions and {vals.shape[1]} values")
    out = _Output(shaped, dtype, accumulate=True)
    tune = C.byref(tuning) if tuning is not None else None
    if order is None:
        status = _lib.library().mpf_scatter(
            kind, degree, ndim, pos.data_ptr(), ps, vals.data_ptr(), vs, pos.shape[1], out.work.data_ptr(),
            ncomp, lower, cell, num, code, dcode, tune, _lib.stream_of(device))
    else:
        tile, starts = _tile_args(order, ndim, device)
        status = _lib.library().mpf_scatter_tiles(
            kind, degree, ndim, pos.data_ptr(), ps, vals.data_ptr(), vs, pos.shape[1], out.work.data_ptr(),
            ncomp, lower, cell, num, code, tile, starts, dcode, tune, _lib.stream_of(device))
    _lib.check(status, "scatter")
    out.finish()


def scatter_deterministic(kind: int, degree: int, positions: torch.Tensor, values: torch.Tensor,
                          field: torch.Tensor, geometry, workspace: torch.Tensor | None = None, order=None) -> None:
    """field(k, c) += sum_i W_k(x_i) values(c, i), the same bits for every run and marker
    order (``mpf_scatter_deterministic``: fixed-point integer sums); float64 only.

    ``order``: the `sorting.TileOrder` whose rank order the markers are in, for
    ``mpf_scatter_deterministic_tiles`` (the same bits).
    """
    lower, cell, num, code, ndim = _lib.geometry_arrays(geometry)
    device = _lib.require_cuda(positions, values, field)
    if field.dtype != torch.float64:
        raise TypeError("the deterministic scatter is float64 only")
    shaped = _field_shape(field, _extent(num, code, degree), "field")
    ncomp = shaped.shape[-1]
    pos, ps = _marker_rows(positions, ndim, "positions", torch.float64)
    vals, vs = _marker_rows(values, ncomp, "values", torch.float64)
    if vals.shape[1] != pos.shape[1]:
        raise ValueError(f"{pos.shape[1]} positions and {vals.shape[1]} values")
    size = C.c_size_t(0)
    _lib.check(_lib.library().mpf_scatter_deterministic_workspace_bytes(shaped.numel(), C.byref(size)),
               "scatter_deterministic_workspace_bytes")
    if workspace is None or workspace.numel() * workspace.element_size() < size.value:
        workspace = torch.empty(size.value, dtype=torch.uint8, device=device)
    out = _Output(shaped, torch.float64, accumulate=True)
    wbytes = workspace.numel() * workspace.element_size()
    if order is None:
        status = _lib.library().mpf_scatter_deterministic(
            kind, degree, ndim, pos.data_ptr(), ps, vals.data_ptr(), vs, pos.shape[1], out.work.data_ptr(), ncomp,
            lower, cell, num, code, workspace.data_ptr(), wbytes, _lib.stream_of(device))
    else:
        tile, starts = _tile_args(order, ndim, device)
        status = _lib.library().mpf_scatter_deterministic_tiles(
            kind, degree, ndim, pos.data_ptr(), ps, vals.data_ptr(), vs, pos.shape[1], out.work.data_ptr(), ncomp,
            lower, cell, num, code, tile, starts, workspace.data_ptr(), wbytes, _lib.stream_of(device))
    _lib.check(status, "scatter_deterministic")
    out.finish()


def gather_grad(kind: int, degree: int, positions: torch.Tensor, field: torch.Tensor,
                cotangent: torch.Tensor, geometry) -> torch.Tensor:
    """``(ndim, N)``: d/dx_d of sum_c cotangent(c, i) gather_c(x_i), the position gradient."""
    lower, cell, num, code, ndim = _lib.geometry_arrays(geometry)
    device = _lib.require_cuda(positions, field, cotangent)
    dtype = field.dtype
    field = _field_shape(field, _extent(num, code, degree), "field").contiguous()
    ncomp = field.shape[-1]
    pos, ps = _marker_rows(positions, ndim, "positions", dtype)
    cot, cs = _marker_rows(cotangent, ncomp, "cotangent", dtype)
    n = pos.shape[1]
    grad = torch.empty((ndim, n), dtype=dtype, device=device)
    status = _lib.library().mpf_gather_grad(
        kind, degree, ndim, pos.data_ptr(), ps, n, field.data_ptr(), ncomp, cot.data_ptr(), cs,
        grad.data_ptr(), n, lower, cell, num, code, _lib.dtype_code(dtype), _lib.stream_of(device))
    _lib.check(status, "gather_grad")
    return grad


@dataclass(frozen=True)
class PathKernel:
    """A path deposit: WHITNEY (kind LINEAR) or the spline edges (kind SPLINE + degree)."""

    kind: int
    ndim: int
    takes_degree: bool

    def __call__(self, *args) -> None:
        if self.takes_degree:
            *args, degree = args
            degree = int(degree)
        else:
            degree = 1
        start, end, charges, edges, *geometry = args
        deposit_paths(self.kind, degree, start, end, charges, edges, geometry)


@dataclass(frozen=True)
class EdgeGatherKernel:
    kind: int
    ndim: int
    takes_degree: bool

    def __call__(self, *args) -> None:
        if self.takes_degree:
            *args, degree = args
            degree = int(degree)
        else:
            degree = 1
        positions, edges, result, *geometry = args
        gather_edges(self.kind, degree, positions, edges, result, geometry)


def deposit_paths(kind: int, degree: int, start: torch.Tensor, end: torch.Tensor, charges: torch.Tensor,
                  edges: torch.Tensor, geometry, tuning: _lib.Tuning | None = None) -> None:
    """edges += the current of ``charges`` moving from ``start`` to ``end`` (ndim, N)."""
    lower, cell, num, code, ndim = _lib.geometry_arrays(geometry)
    device = _lib.require_cuda(start, end, charges, edges)
    dtype = edges.dtype
    s, ss = _marker_rows(start, ndim, "start", dtype)
    e, es = _marker_rows(end, ndim, "end", dtype)
    q = charges.reshape(-1).to(dtype).contiguous()
    if s.shape != e.shape or s.shape[1] != q.shape[0]:
        raise ValueError(f"paths from {tuple(s.shape)} to {tuple(e.shape)} for {q.shape[0]} charges")
    extent = _extent(num, code, degree)
    if tuple(edges.shape) != (*extent, ndim):
        raise ValueError(f"an edge field on this grid is {(*extent, ndim)}, got {tuple(edges.shape)}")
    out = _Output(edges, dtype, accumulate=True)
    status = _lib.library().mpf_deposit_paths(
        kind, degree, ndim, s.data_ptr(), ss, e.data_ptr(), es, q.data_ptr(), q.shape[0],
        out.work.data_ptr(), lower, cell, num, code, _lib.dtype_code(dtype),
        C.byref(tuning) if tuning is not None else None, _lib.stream_of(device))
    _lib.check(status, "deposit_paths")
    out.finish()


def gather_edges(kind: int, degree: int, positions: torch.Tensor, edges: torch.Tensor, result: torch.Tensor,
                 geometry) -> None:
    """result(a, i) = the field of the edge field along axis a at marker i."""
    lower, cell, num, code, ndim = _lib.geometry_arrays(geometry)
    device = _lib.require_cuda(positions, edges, result)
    dtype = edges.dtype
    pos, ps = _marker_rows(positions, ndim, "positions", dtype)
    n = pos.shape[1]
    extent = _extent(num, code, degree)
    if tuple(edges.shape) != (*extent, ndim):
        raise ValueError(f"an edge field on this grid is {(*extent, ndim)}, got {tuple(edges.shape)}")
    edges = edges.contiguous()
    out = _Output(result, dtype, accumulate=False)
    if tuple(out.work.shape) != (ndim, n):
        raise ValueError(f"result must be ({ndim}, {n}), got {tuple(result.shape)}")
    status = _lib.library().mpf_gather_edges(
        kind, degree, ndim, pos.data_ptr(), ps, n, edges.data_ptr(), out.work.data_ptr(), out.work.stride(0),
        lower, cell, num, code, _lib.dtype_code(dtype), _lib.stream_of(device))
    _lib.check(status, "gather_edges")
    out.finish()


def _catalog() -> dict:
    kernels = {}
    for n in (1, 2, 3):
        kernels[f"gather_linear_{n}d"] = NodeKernel("gather", _lib.LINEAR, n, False, 1)
        kernels[f"scatter_linear_{n}d"] = NodeKernel("scatter", _lib.LINEAR, n, False, 1)
        kernels[f"gather_quadratic_{n}d"] = NodeKernel("gather", _lib.QUADRATIC, n, False, 2)
        kernels[f"scatter_quadratic_{n}d"] = NodeKernel("scatter", _lib.QUADRATIC, n, False, 2)
        kernels[f"gather_spline_{n}d"] = NodeKernel("gather", _lib.SPLINE, n, True)
        kernels[f"scatter_spline_{n}d"] = NodeKernel("scatter", _lib.SPLINE, n, True)
        kernels[f"deposit_paths_{n}d"] = PathKernel(_lib.LINEAR, n, False)
        kernels[f"deposit_paths_spline_{n}d"] = PathKernel(_lib.SPLINE, n, True)
        kernels[f"gather_edges_{n}d"] = EdgeGatherKernel(_lib.LINEAR, n, False)
        kernels[f"gather_edges_spline_{n}d"] = EdgeGatherKernel(_lib.SPLINE, n, True)
    return kernels


#: The kernels by the reference's names.
KERNELS = _catalog()
