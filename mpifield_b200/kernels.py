"""The kernel callables of the B200 backend, with the arguments of mpifield's kernels.

mpifield's weightings call their kernels as (src/mpifield/weighting.py:22-38,
src/mpifield/edges.py:23-31)::

    scatter(positions, values, field, *geometry)               # adds into field
    gather(positions, field, result, *geometry)                 # overwrites result
    deposit_paths(start, end, charges, edges, *geometry)        # adds into edges

with ``geometry = (*lower, *cell_size, *num_nodes, *code)`` and, for the spline kernels,
a trailing ``degree``. The callables here take the same arguments as device arrays --
CuPy arrays as mpifield passes them, torch tensors, anything with
``__cuda_array_interface__`` or ``__dlpack__`` (`_arrays`) -- in float64, or float32 for
the single-precision variant, and launch the sm_100a kernels of ``libmpifield_b200.so``
asynchronously on the caller's stream (`_arrays.launch_stream`). `KERNELS` maps the
reference's kernel names (src/mpifield/kernels/catalog.py:51-93) to them, with the
signatures the reference's catalog documents: the linear 1D deposit also takes one
component as ``(N,)`` markers and an ``(nx,)`` grid, and the linear 3D kernels the grid
as rows ``(nx * ny * nz, ncomp)`` (src/mpifield/weighting.py:259-330); the launch
keywords the reference gives its CUDA kernels (``shared_mem``, ``n_threads``) are
accepted and left to this backend's own launch configuration.

Marker arrays are ``(rows, N)`` with a unit column stride and any row stride
(``storage[:, :n]``) and are passed as they are; another layout or element type is
copied first, and an output the C calls cannot write in place is written through a
contiguous copy, as ``cunumpy.kernels.kernel_output`` does for the reference.
"""

from __future__ import annotations

import contextlib
import ctypes as C
import functools
from dataclasses import dataclass

from mpifield_b200 import _lib
from mpifield_b200._arrays import DeviceArray, as_device_array, launch_stream, torch_on, use_stream

_DTYPES = {"f8": _lib.F64, "f4": _lib.F32}
#: Keywords of cunumpy kernel launches (src/mpifield/weighting.py:286-295): this
#: backend sizes its own launches, so they change nothing here.
_LAUNCH_KEYWORDS = frozenset({"shared_mem", "n_threads"})


def _dtype_code(a: DeviceArray, name: str) -> int:
    if a.dtype not in _DTYPES:
        raise TypeError(f"mpifield_b200 kernels take float64 or float32, {name} is {a.dtype}")
    return _DTYPES[a.dtype]


def _torch_dtype(code: str):
    import torch

    return {"f8": torch.float64, "f4": torch.float32}[code]


def _copied(a: DeviceArray, shape: tuple[int, ...], dtype: str, stream: int) -> DeviceArray:
    """A contiguous ``shape`` copy of ``a`` in ``dtype``, made on the launch stream."""
    with torch_on(stream):
        t = a.torch().reshape(shape).to(_torch_dtype(dtype)).contiguous()
    return as_device_array(t)


def _marker_rows(a: DeviceArray, rows: int, name: str, dtype: str, stream: int) -> tuple[DeviceArray, int]:
    """``a`` as ``(rows, N)`` with unit column stride, and its row stride in elements; a
    1-D array is one row. Copied only where the layout or element type needs it."""
    if a.ndim == 1:
        a = DeviceArray(a.ptr, (1, a.shape[0]), (a.shape[0], a.strides[0]), a.dtype, a.source, a.stream, a.device)
    if a.ndim != 2 or a.shape[0] != rows:
        raise ValueError(f"{name} must be ({rows}, N), got {a.shape}")
    n = a.shape[1]
    fits = a.dtype == dtype and (n <= 1 or a.strides[1] == 1) and (rows == 1 or a.strides[0] >= n)
    if not fits:
        a = _copied(a, (rows, n), dtype, stream)
    return a, (a.strides[0] if rows > 1 else n)


class _Output:
    """Where a call writes ``target``: the target itself when the C call takes its layout,
    else a contiguous copy (filled from the target for an accumulating call) that
    `finish` writes back, both on the launch stream."""

    def __init__(self, target: DeviceArray, dtype: str, accumulate: bool, stream: int, rows: int | None = None):
        self.target, self.stream = target, stream
        if rows is None:
            self.direct = target.is_contiguous() and target.dtype == dtype
        else:
            n = target.shape[-1]
            self.direct = (target.dtype == dtype and target.ndim == 2 and (n <= 1 or target.strides[1] == 1)
                           and (rows == 1 or target.strides[0] >= n))
        if self.direct:
            self.work = target
            return
        import torch

        with torch_on(stream):
            if accumulate:
                work = target.torch().to(_torch_dtype(dtype)).contiguous()
                if work.data_ptr() == target.ptr:
                    work = work.clone()
            else:
                work = torch.empty(target.shape, dtype=_torch_dtype(dtype), device=target.torch().device)
        self.work = as_device_array(work)

    @property
    def row_stride(self) -> int:
        return self.work.strides[0] if self.work.shape[0] > 1 else self.work.shape[-1]

    def finish(self) -> None:
        if not self.direct:
            with torch_on(self.stream):
                self.target.torch().copy_(self.work.torch())


def _extent(num, code, degree) -> tuple[int, ...]:
    return _extent_of(tuple(num), tuple(code), degree)


@functools.lru_cache(maxsize=1024)
def _extent_of(num: tuple, code: tuple, degree: int) -> tuple[int, ...]:
    return tuple(int(n) + (degree - 1 if int(c) == 2 else 0) for n, c in zip(num, code))


def _field(a: DeviceArray, extent: tuple[int, ...], name: str) -> DeviceArray:
    """``a`` as ``extent + (ncomp,)``: a field without the component axis is one
    component, and the linear 3D kernels' rows ``(nx * ny * nz, ncomp)`` are the grid."""
    ndim = len(extent)
    if a.ndim == ndim:
        a = DeviceArray(a.ptr, a.shape + (1,), a.strides + (1,), a.dtype, a.source, a.stream, a.device)
    elif ndim == 3 and a.ndim == 2 and a.shape[0] == extent[0] * extent[1] * extent[2]:
        if not a.is_contiguous():
            raise ValueError("the linear 3D kernels need a C-contiguous field")
        a = a.reshaped((*extent, a.shape[1]))
    if a.ndim != ndim + 1 or tuple(a.shape[:-1]) != extent:
        raise ValueError(f"{name} on this grid is {extent} + (ncomp,), got {a.shape}")
    return a


def _arrays(**named) -> tuple[dict[str, DeviceArray], int]:
    """Every named argument as a `DeviceArray` (None stays None), and the launch stream."""
    arrays = {k: (None if v is None else as_device_array(v, k)) for k, v in named.items()}
    present = [a for a in arrays.values() if a is not None]
    devices = {a.device for a in present if a.device is not None}
    if len(devices) > 1:
        raise ValueError(f"arrays on different devices: {sorted(devices)}")
    return arrays, launch_stream(*present)


def _tile_args(order, ndim: int):
    """The tile shape (ctypes array) and tile starts of a `sorting.TileOrder`, checked."""
    starts = as_device_array(order.tile_start, "order.tile_start")
    if starts.dtype != "i8" or not starts.is_contiguous():
        raise ValueError("order.tile_start must be a contiguous int64 array on the markers' device")
    if len(order.tile) != ndim or starts.size != order.num_tiles + 2:
        raise ValueError(f"a tile order of {len(order.tile)} axes and {starts.size} starts for a {ndim}D grid")
    return (C.c_int32 * ndim)(*(int(v) for v in order.tile)), starts.ptr


def _degree(takes_degree: bool, fixed: int | None, args: tuple) -> tuple[int, tuple]:
    if takes_degree:
        *rest, degree = args
        return int(degree), tuple(rest)
    return int(fixed), args


_NO_STREAM = contextlib.nullcontext()


def _launch_options(kernel: str, launch: dict):
    if not launch:
        return _NO_STREAM
    unknown = set(launch) - _LAUNCH_KEYWORDS - {"stream"}
    if unknown:
        raise TypeError(f"{kernel} got unexpected keyword arguments {sorted(unknown)}")
    stream = launch.get("stream")
    return use_stream(stream) if stream is not None else _NO_STREAM


@dataclass(frozen=True)
class NodeKernel:
    """A gather or a scatter with the arithmetic of one reference stencil kind."""

    op: str  # "gather" or "scatter"
    kind: int
    ndim: int
    takes_degree: bool
    fixed_degree: int | None = None
    tuning: _lib.Tuning | None = None

    def __call__(self, *args, **launch) -> None:
        degree, args = _degree(self.takes_degree, self.fixed_degree, args)
        with _launch_options(f"{self.op} kernel", launch):
            if self.op == "gather":
                positions, field, result, *geometry = args
                gather(self.kind, degree, positions, field, result, geometry, self.tuning)
            else:
                positions, values, field, *geometry = args
                scatter(self.kind, degree, positions, values, field, geometry, self.tuning)


def gather(kind: int, degree: int, positions, field, result, geometry, tuning: _lib.Tuning | None = None,
           order=None) -> None:
    """result(c, i) = sum_k W_k(x_i) field(k, c), overwriting ``result`` (ncomp, N).

    ``order``: the `sorting.TileOrder` whose rank order the markers are in, for
    ``mpf_gather_tiles`` (the same result, whatever the markers' order).
    """
    lower, cell, num, code, ndim = _lib.geometry_arrays(geometry)
    a, stream = _arrays(positions=positions, field=field, result=result)
    dtype = a["field"].dtype
    dcode = _dtype_code(a["field"], "field")
    f = _field(a["field"], _extent(num, code, degree), "field")
    if not f.is_contiguous():
        f = _copied(f, f.shape, dtype, stream)
    ncomp = f.shape[-1]
    pos, ps = _marker_rows(a["positions"], ndim, "positions", dtype, stream)
    n = pos.shape[1]
    res = a["result"]
    if res.ndim == 1:
        res = DeviceArray(res.ptr, (1, res.shape[0]), (res.shape[0], res.strides[0]), res.dtype, res.source,
                          res.stream, res.device)
    if res.shape != (ncomp, n):
        raise ValueError(f"result must be ({ncomp}, {n}), got {res.shape}")
    out = _Output(res, dtype, accumulate=False, stream=stream, rows=ncomp)
    tune = C.byref(tuning) if tuning is not None else None
    lib = _lib.library()
    if order is None:
        status = lib.mpf_gather(kind, degree, ndim, pos.ptr, ps, n, f.ptr, ncomp, out.work.ptr, out.row_stride,
                                lower, cell, num, code, dcode, tune, stream)
    else:
        tile, starts = _tile_args(order, ndim)
        status = lib.mpf_gather_tiles(kind, degree, ndim, pos.ptr, ps, n, f.ptr, ncomp, out.work.ptr,
                                      out.row_stride, lower, cell, num, code, tile, starts, dcode, tune, stream)
    _lib.check(status, "gather")
    out.finish()


def scatter(kind: int, degree: int, positions, values, field, geometry, tuning: _lib.Tuning | None = None,
            order=None) -> None:
    """field(k, c) += sum_i W_k(x_i) values(c, i); dead markers (all values zero) skipped.

    ``order``: the `sorting.TileOrder` whose rank order the markers are in (positions and
    values permuted by ``order.order``), for ``mpf_scatter_tiles``; the result is the same
    up to the order of the floating-point adds, whatever the markers' order.
    """
    lower, cell, num, code, ndim = _lib.geometry_arrays(geometry)
    a, stream = _arrays(positions=positions, values=values, field=field)
    dtype = a["field"].dtype
    dcode = _dtype_code(a["field"], "field")
    f = _field(a["field"], _extent(num, code, degree), "field")
    ncomp = f.shape[-1]
    pos, ps = _marker_rows(a["positions"], ndim, "positions", dtype, stream)
    vals, vs = _marker_rows(a["values"], ncomp, "values", dtype, stream)
    if vals.shape[1] != pos.shape[1]:
        raise ValueError(f"{pos.shape[1]} positions and {vals.shape[1]} values")
    out = _Output(f, dtype, accumulate=True, stream=stream)
    tune = C.byref(tuning) if tuning is not None else None
    lib = _lib.library()
    n = pos.shape[1]
    if order is None:
        status = lib.mpf_scatter(kind, degree, ndim, pos.ptr, ps, vals.ptr, vs, n, out.work.ptr, ncomp, lower, cell,
                                 num, code, dcode, tune, stream)
    else:
        tile, starts = _tile_args(order, ndim)
        status = lib.mpf_scatter_tiles(kind, degree, ndim, pos.ptr, ps, vals.ptr, vs, n, out.work.ptr, ncomp, lower,
                                       cell, num, code, tile, starts, dcode, tune, stream)
    _lib.check(status, "scatter")
    out.finish()


def scatter_deterministic(kind: int, degree: int, positions, values, field, geometry, workspace=None,
                          order=None) -> None:
    """field(k, c) += sum_i W_k(x_i) values(c, i), the same bits for every run and marker
    order (``mpf_scatter_deterministic``: fixed-point integer sums); float64 only.

    ``order``: the `sorting.TileOrder` whose rank order the markers are in, for
    ``mpf_scatter_deterministic_tiles`` (the same bits).
    """
    lower, cell, num, code, ndim = _lib.geometry_arrays(geometry)
    a, stream = _arrays(positions=positions, values=values, field=field, workspace=workspace)
    if a["field"].dtype != "f8":
        raise TypeError("the deterministic scatter is float64 only")
    f = _field(a["field"], _extent(num, code, degree), "field")
    ncomp = f.shape[-1]
    pos, ps = _marker_rows(a["positions"], ndim, "positions", "f8", stream)
    vals, vs = _marker_rows(a["values"], ncomp, "values", "f8", stream)
    if vals.shape[1] != pos.shape[1]:
        raise ValueError(f"{pos.shape[1]} positions and {vals.shape[1]} values")
    size = C.c_size_t(0)
    lib = _lib.library()
    _lib.check(lib.mpf_scatter_deterministic_workspace_bytes(f.size, C.byref(size)),
               "scatter_deterministic_workspace_bytes")
    ws = a["workspace"]
    if ws is None or ws.size * ws.itemsize < size.value:
        import torch

        with torch_on(stream):
            ws = as_device_array(torch.empty(size.value, dtype=torch.uint8, device=f.torch().device))
    out = _Output(f, "f8", accumulate=True, stream=stream)
    wbytes = ws.size * ws.itemsize
    n = pos.shape[1]
    if order is None:
        status = lib.mpf_scatter_deterministic(kind, degree, ndim, pos.ptr, ps, vals.ptr, vs, n, out.work.ptr, ncomp,
                                               lower, cell, num, code, ws.ptr, wbytes, stream)
    else:
        tile, starts = _tile_args(order, ndim)
        status = lib.mpf_scatter_deterministic_tiles(kind, degree, ndim, pos.ptr, ps, vals.ptr, vs, n, out.work.ptr,
                                                     ncomp, lower, cell, num, code, tile, starts, ws.ptr, wbytes,
                                                     stream)
    _lib.check(status, "scatter_deterministic")
    out.finish()


def gather_grad(kind: int, degree: int, positions, field, cotangent, geometry):
    """``(ndim, N)`` torch tensor: d/dx_d of sum_c cotangent(c, i) gather_c(x_i), the position gradient."""
    import torch

    lower, cell, num, code, ndim = _lib.geometry_arrays(geometry)
    a, stream = _arrays(positions=positions, field=field, cotangent=cotangent)
    dtype = a["field"].dtype
    f = _field(a["field"], _extent(num, code, degree), "field")
    if not f.is_contiguous():
        f = _copied(f, f.shape, dtype, stream)
    ncomp = f.shape[-1]
    pos, ps = _marker_rows(a["positions"], ndim, "positions", dtype, stream)
    cot, cs = _marker_rows(a["cotangent"], ncomp, "cotangent", dtype, stream)
    n = pos.shape[1]
    with torch_on(stream):
        grad = torch.empty((ndim, n), dtype=_torch_dtype(dtype), device=f.torch().device)
    status = _lib.library().mpf_gather_grad(
        kind, degree, ndim, pos.ptr, ps, n, f.ptr, ncomp, cot.ptr, cs, grad.data_ptr(), n, lower, cell, num, code,
        _dtype_code(f, "field"), stream)
    _lib.check(status, "gather_grad")
    return grad


@dataclass(frozen=True)
class PathKernel:
    """A path deposit: WHITNEY (kind LINEAR, degree 1) or the spline edges (kind SPLINE),
    whose degree is the last argument (``takes_degree``) or ``fixed_degree``."""

    kind: int
    ndim: int
    takes_degree: bool
    fixed_degree: int = 1

    def __call__(self, *args, **launch) -> None:
        degree, args = _degree(self.takes_degree, self.fixed_degree, args)
        start, end, charges, edges, *geometry = args
        with _launch_options("deposit_paths kernel", launch):
            deposit_paths(self.kind, degree, start, end, charges, edges, geometry)


@dataclass(frozen=True)
class EdgeGatherKernel:
    """An edge gather: the Whitney edge functions (kind LINEAR) or the spline edges, with
    the degree as for `PathKernel`."""

    kind: int
    ndim: int
    takes_degree: bool
    fixed_degree: int = 1

    def __call__(self, *args, **launch) -> None:
        degree, args = _degree(self.takes_degree, self.fixed_degree, args)
        positions, edges, result, *geometry = args
        with _launch_options("gather_edges kernel", launch):
            gather_edges(self.kind, degree, positions, edges, result, geometry)


def _edge_field(a: DeviceArray, num, code, degree, ndim) -> None:
    extent = _extent(num, code, degree)
    if a.shape != (*extent, ndim):
        raise ValueError(f"an edge field on this grid is {(*extent, ndim)}, got {a.shape}")


def deposit_paths(kind: int, degree: int, start, end, charges, edges, geometry,
                  tuning: _lib.Tuning | None = None) -> None:
    """edges += the current of ``charges`` moving from ``start`` to ``end`` (ndim, N)."""
    lower, cell, num, code, ndim = _lib.geometry_arrays(geometry)
    a, stream = _arrays(start=start, end=end, charges=charges, edges=edges)
    dtype = a["edges"].dtype
    s, ss = _marker_rows(a["start"], ndim, "start", dtype, stream)
    e, es = _marker_rows(a["end"], ndim, "end", dtype, stream)
    q = a["charges"]
    if q.ndim > 1:  # (1, N) or any array of N charges
        q = q.reshaped((q.size,)) if q.is_contiguous() else _copied(q, (q.size,), dtype, stream)
    q, _ = _marker_rows(q, 1, "charges", dtype, stream)
    if s.shape != e.shape or s.shape[1] != q.shape[1]:
        raise ValueError(f"paths from {s.shape} to {e.shape} for {q.shape[1]} charges")
    _edge_field(a["edges"], num, code, degree, ndim)
    out = _Output(a["edges"], dtype, accumulate=True, stream=stream)
    status = _lib.library().mpf_deposit_paths(
        kind, degree, ndim, s.ptr, ss, e.ptr, es, q.ptr, q.shape[1], out.work.ptr, lower, cell, num, code,
        _dtype_code(a["edges"], "edges"), C.byref(tuning) if tuning is not None else None, stream)
    _lib.check(status, "deposit_paths")
    out.finish()


def gather_edges(kind: int, degree: int, positions, edges, result, geometry) -> None:
    """result(a, i) = the field of the edge field along axis a at marker i."""
    lower, cell, num, code, ndim = _lib.geometry_arrays(geometry)
    a, stream = _arrays(positions=positions, edges=edges, result=result)
    dtype = a["edges"].dtype
    pos, ps = _marker_rows(a["positions"], ndim, "positions", dtype, stream)
    n = pos.shape[1]
    _edge_field(a["edges"], num, code, degree, ndim)
    ed = a["edges"] if a["edges"].is_contiguous() else _copied(a["edges"], a["edges"].shape, dtype, stream)
    if a["result"].shape != (ndim, n):
        raise ValueError(f"result must be ({ndim}, {n}), got {a['result'].shape}")
    out = _Output(a["result"], dtype, accumulate=False, stream=stream, rows=ndim)
    status = _lib.library().mpf_gather_edges(
        kind, degree, ndim, pos.ptr, ps, n, ed.ptr, out.work.ptr, out.row_stride, lower, cell, num, code,
        _dtype_code(ed, "edges"), stream)
    _lib.check(status, "gather_edges")
    out.finish()


def form_components(form: int, ndim: int) -> int:
    """The components of a ``form``-form in ``ndim`` dimensions: ndim choose form."""
    return {(1, 1): 1, (1, 2): 2, (2, 2): 1, (1, 3): 3, (2, 3): 3, (3, 3): 1}[(form, ndim)]


def gather_forms(degree: int, form: int, positions, field, result, geometry) -> None:
    """result(c, i) = the ``form``-form ``field`` (extent + (ncomp,)) at marker i, component c."""
    lower, cell, num, code, ndim = _lib.geometry_arrays(geometry)
    a, stream = _arrays(positions=positions, field=field, result=result)
    dtype = a["field"].dtype
    f = _field(a["field"], _extent(num, code, degree), "field")
    if not f.is_contiguous():
        f = _copied(f, f.shape, dtype, stream)
    ncomp = f.shape[-1]
    pos, ps = _marker_rows(a["positions"], ndim, "positions", dtype, stream)
    n = pos.shape[1]
    if a["result"].shape != (ncomp, n) and not (ncomp == 1 and a["result"].shape == (n,)):
        raise ValueError(f"result must be ({ncomp}, {n}), got {a['result'].shape}")
    res = a["result"]
    if res.ndim == 1:
        res = DeviceArray(res.ptr, (1, n), (n, res.strides[0]), res.dtype, res.source, res.stream, res.device)
    out = _Output(res, dtype, accumulate=False, stream=stream, rows=ncomp)
    status = _lib.library().mpf_gather_forms(degree, form, ndim, pos.ptr, ps, n, f.ptr, ncomp, out.work.ptr,
                                              out.row_stride, lower, cell, num, code, _dtype_code(f, "field"), stream)
    _lib.check(status, "gather_forms")
    out.finish()


def scatter_forms(degree: int, form: int, positions, values, field, geometry) -> None:
    """field(k, c) += the ``form``-form weights of markers' ``values`` (ncomp, N)."""
    lower, cell, num, code, ndim = _lib.geometry_arrays(geometry)
    a, stream = _arrays(positions=positions, values=values, field=field)
    dtype = a["field"].dtype
    f = _field(a["field"], _extent(num, code, degree), "field")
    ncomp = f.shape[-1]
    pos, ps = _marker_rows(a["positions"], ndim, "positions", dtype, stream)
    vals, vs = _marker_rows(a["values"], ncomp, "values", dtype, stream)
    if vals.shape[1] != pos.shape[1]:
        raise ValueError(f"{pos.shape[1]} positions and {vals.shape[1]} values")
    out = _Output(f, dtype, accumulate=True, stream=stream)
    status = _lib.library().mpf_scatter_forms(degree, form, ndim, pos.ptr, ps, vals.ptr, vs, pos.shape[1],
                                               out.work.ptr, ncomp, lower, cell, num, code, _dtype_code(f, "field"),
                                               stream)
    _lib.check(status, "scatter_forms")
    out.finish()


@dataclass(frozen=True)
class FormKernel:
    """A k-form gather or scatter: gather_forms_spline_{n}d / scatter_forms_spline_{n}d with
    ``degree`` and ``form`` as the last two arguments, or fixed (``fixed``: (degree, form))."""

    op: str
    ndim: int
    fixed: tuple | None = None

    def __call__(self, *args, **launch) -> None:
        if self.fixed is None:
            *args, degree, form = args
        else:
            degree, form = self.fixed
        with _launch_options(f"{self.op} forms kernel", launch):
            if self.op == "gather":
                positions, field, result, *geometry = args
                gather_forms(int(degree), int(form), positions, field, result, geometry)
            else:
                positions, values, field, *geometry = args
                scatter_forms(int(degree), int(form), positions, values, field, geometry)


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
        kernels[f"gather_forms_spline_{n}d"] = FormKernel("gather", n)
        kernels[f"scatter_forms_spline_{n}d"] = FormKernel("scatter", n)
    return kernels


#: The kernels by the reference's names.
KERNELS = _catalog()
