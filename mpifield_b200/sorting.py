"""Cell-tile sort of markers: keys, a stable order and the start of every tile.

Markers sorted by cell tile are what the shared-memory boxes of the gather and scatter
kernels need (each chunk of markers then touches one small box of the grid). The key of
a marker is the tile of its stencil's anchor node (the node LINEAR, QUADRATIC or the
spline stencil is anchored on), row-major over tiles of ``tile`` nodes per axis; a
marker whose values are all zero goes to the sentinel tile ``num_tiles`` without its
position being read (with ``within`` the key continues with the cell inside the tile).
The order is stable: equal keys keep the marker order, so the
result equals ``numpy.argsort(keys, kind="stable")`` bit for bit. The workspace is
allocated here by torch and passed to the C call, which allocates nothing.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from mpifield_b200 import _lib
from mpifield_b200._arrays import as_device_array, launch_stream, torch_on
from mpifield_b200.kernels import _marker_rows


@dataclass
class TileOrder:
    """The result of `sort_by_tile` and `resort_by_tile`."""

    keys: torch.Tensor | None  # (N,) int32 view of the uint32 keys, in marker order (sort_by_tile)
    order: torch.Tensor        # (N,) int32: the marker of every rank
    tile_start: torch.Tensor   # (num_tiles + 2,) int64: first rank of every tile, then N
    num_tiles: int
    tile: tuple = ()           # anchor nodes per tile, per axis
    sorted_keys: torch.Tensor | None = None  # (N,) int32 view of the keys in rank order (resort_by_tile)


def _kind_of(weighting) -> tuple[int, int]:
    """(kind, degree) of a built-in weighting, or of a ``(kind, degree)`` pair."""
    if isinstance(weighting, tuple):
        return int(weighting[0]), int(weighting[1])
    kernel = weighting.gather_kernel(1)
    return int(kernel.kind), int(kernel.fixed_degree)


def num_tiles(weighting, geometry, tile) -> int:
    kind, degree = _kind_of(weighting)
    _, _, num, code, ndim = _lib.geometry_arrays(geometry)
    t = (C.c_int32 * ndim)(*(int(v) for v in tile))
    out = C.c_int64(0)
    _lib.check(_lib.library().mpf_num_tiles(kind, degree, ndim, num, code, t, C.byref(out)), "num_tiles")
    return int(out.value)


def sort_workspace_bytes(n: int, ntiles: int) -> int:
    """Bytes of the sort's workspace for ``n`` markers and ``ntiles`` tiles."""
    size = C.c_size_t(0)
    _lib.check(_lib.library().mpf_sort_workspace_bytes(n, ntiles, C.byref(size)), "sort_workspace_bytes")
    return max(int(size.value), 256)


def _code_of(dtype: torch.dtype) -> str:
    _lib.dtype_code(dtype)  # float64 or float32 only
    return "f8" if dtype == torch.float64 else "f4"


def _empty(shape, dtype, device):
    return torch.empty(shape, dtype=dtype, device=device)


def sort_by_tile(positions: torch.Tensor, weighting, geometry, tile, values: torch.Tensor | None = None,
                 within: bool = False, alloc=None) -> TileOrder:
    """Sort markers by cell tile (see the module docstring).

    With ``within`` the key continues with the anchor cell inside the tile, so markers of
    one cell end up next to each other (tile-major, then cell-major): the order the
    gather and scatter kernels run fastest on. ``alloc(shape, dtype)`` supplies the
    keys, order, tile starts and workspace (default: new tensors on the device).
    """
    kind, degree = _kind_of(weighting)
    lower, cell, num, code, ndim = _lib.geometry_arrays(geometry)
    p = as_device_array(positions, "positions")
    v = None if values is None else as_device_array(values, "values")
    stream = launch_stream(*(a for a in (p, v) if a is not None))
    if p.dtype not in ("f8", "f4"):
        raise TypeError(f"positions must be float64 or float32, got {p.dtype}")
    pos, ps = _marker_rows(p, ndim, "positions", p.dtype, stream)
    n = pos.shape[1]
    ntiles = num_tiles((kind, degree), geometry, tile)
    t = (C.c_int32 * ndim)(*(int(v) for v in tile))
    device = pos.torch().device
    new = alloc or (lambda shape, dt: _empty(shape, dt, device))
    with torch_on(stream):
        workspace = new((sort_workspace_bytes(n, ntiles),), torch.uint8)
        keys = new((n,), torch.int32)
        order = new((n,), torch.int32)
        tile_start = new((ntiles + 2,), torch.int64)
    if v is not None:
        vals, vs = _marker_rows(v, v.shape[0] if v.ndim == 2 else 1, "values", p.dtype, stream)
        vptr, ncomp = vals.ptr, vals.shape[0]
    else:
        vptr, vs, ncomp = None, 0, 0
    status = _lib.library().mpf_sort_by_tile(
        kind, degree, ndim, pos.ptr, ps, vptr, vs, ncomp, n, lower, cell, num, code, t, int(bool(within)),
        keys.data_ptr(), order.data_ptr(), tile_start.data_ptr(), workspace.data_ptr(), workspace.numel(),
        _lib.F64 if p.dtype == "f8" else _lib.F32, stream)
    _lib.check(status, "sort_by_tile")
    return TileOrder(keys, order, tile_start, ntiles, tuple(int(v) for v in tile))


def resort_by_tile(positions, weighting, geometry, tile, values=None, within: bool = False,
                   previous: TileOrder | None = None, alloc=None) -> TileOrder:
    """Sort a marker store by cell tile, again: ``positions`` (and ``values``) are the store's
    arrays in their current order, ``previous`` the `TileOrder` this function returned for
    the store before its markers moved (after which the store's arrays were permuted by its
    ``order``), or None for the first sort. The result is the order `sort_by_tile` gives,
    bit for bit, with ``sorted_keys`` for the next call; with ``previous`` only the markers
    whose key changed are sorted (mpf_resort_by_tile). ``alloc`` as in `sort_by_tile`.
    """
    kind, degree = _kind_of(weighting)
    lower, cell, num, code, ndim = _lib.geometry_arrays(geometry)
    p = as_device_array(positions, "positions")
    v = None if values is None else as_device_array(values, "values")
    stream = launch_stream(*(a for a in (p, v) if a is not None))
    if p.dtype not in ("f8", "f4"):
        raise TypeError(f"positions must be float64 or float32, got {p.dtype}")
    pos, ps = _marker_rows(p, ndim, "positions", p.dtype, stream)
    n = pos.shape[1]
    ntiles = num_tiles((kind, degree), geometry, tile)
    t = (C.c_int32 * ndim)(*(int(x) for x in tile))
    if previous is not None:
        if previous.sorted_keys is None or previous.sorted_keys.numel() != n or tuple(previous.tile) != tuple(
                int(x) for x in tile):
            raise ValueError("previous must be the resort_by_tile result of this store (same markers and tile)")
    size = C.c_size_t(0)
    _lib.check(_lib.library().mpf_resort_workspace_bytes(kind, degree, ndim, num, code, t, int(bool(within)), n,
                                                       C.byref(size)), "resort_workspace_bytes")
    device = pos.torch().device
    new = alloc or (lambda shape, dt: _empty(shape, dt, device))
    with torch_on(stream):
        workspace = new((max(int(size.value), 256),), torch.uint8)
        order = new((n,), torch.int32)
        sorted_keys = new((n,), torch.int32)
        tile_start = new((ntiles + 2,), torch.int64)
    if v is not None:
        vals, vs = _marker_rows(v, v.shape[0] if v.ndim == 2 else 1, "values", p.dtype, stream)
        vptr, ncomp = vals.ptr, vals.shape[0]
    else:
        vptr, vs, ncomp = None, 0, 0
    prev = previous.sorted_keys.data_ptr() if previous is not None else None
    status = _lib.library().mpf_resort_by_tile(
        kind, degree, ndim, pos.ptr, ps, vptr, vs, ncomp, n, lower, cell, num, code, t, int(bool(within)), prev,
        sorted_keys.data_ptr(), order.data_ptr(), tile_start.data_ptr(), workspace.data_ptr(), workspace.numel(),
        _lib.F64 if p.dtype == "f8" else _lib.F32, stream)
    _lib.check(status, "resort_by_tile")
    return TileOrder(None, order, tile_start, ntiles, tuple(int(x) for x in tile), sorted_keys)


def permute(array: torch.Tensor, order: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """``array[:, order]`` for a marker array (rows, N), by the backend's permute kernel
    (into ``out``, a contiguous (rows, N) tensor, when given)."""
    device = _lib.require_cuda(array, order)
    squeeze = array.dim() == 1
    rows = 1 if squeeze else array.shape[0]
    stream = _lib.stream_of(device)
    src, ss = _marker_rows(as_device_array(array), rows, "array", _code_of(array.dtype), stream)
    n = src.shape[1]
    dst = torch.empty((rows, n), dtype=array.dtype, device=device) if out is None else out.view(rows, n)
    if not dst.is_contiguous() or dst.dtype != array.dtype:
        raise ValueError(f"out must be a contiguous ({rows}, {n}) {array.dtype} tensor")
    order = order.to(torch.int32).contiguous()
    status = _lib.library().mpf_permute_rows(dst.data_ptr(), n, src.ptr, ss, rows, order.data_ptr(), n,
                                            _lib.dtype_code(array.dtype), stream)
    _lib.check(status, "permute_rows")
    return dst[0] if squeeze else dst


def unpermute(array: torch.Tensor, order: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """The inverse of `permute`: ``out[:, order] = array`` (results back in marker order)."""
    device = _lib.require_cuda(array, order)
    squeeze = array.dim() == 1
    rows = 1 if squeeze else array.shape[0]
    stream = _lib.stream_of(device)
    src, ss = _marker_rows(as_device_array(array), rows, "array", _code_of(array.dtype), stream)
    n = src.shape[1]
    dst = out if out is not None else torch.empty((rows, n), dtype=array.dtype, device=device)
    if dst.dim() == 1:
        dst = dst.view(1, -1)
    if not dst.is_contiguous() or tuple(dst.shape) != (rows, n):
        raise ValueError(f"out must be a contiguous ({rows}, {n}) tensor")
    order = order.to(torch.int32).contiguous()
    status = _lib.library().mpf_unpermute_rows(dst.data_ptr(), n, src.ptr, ss, rows, order.data_ptr(), n,
                                              _lib.dtype_code(array.dtype), stream)
    _lib.check(status, "unpermute_rows")
    return dst[0] if squeeze else dst
