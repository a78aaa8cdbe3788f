"""The test oracle: NumPy-facing wrappers of the C restatement (TEST INFRASTRUCTURE).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this
module, as the checker; the product (``mpifield_b200``) never does.

- `gather`, `scatter`, `deposit_whitney`, `deposit_spline`, `gather_edges`,
  `gather_forms`, `scatter_forms`, `gather_grad`, `tile_keys`: the serial C restatement in ``mpf_oracle.c`` of the
  reference kernels (citations there).
- `divergence_block`, `gradient_block`: ``EdgeWeighting.divergence_block`` and
  ``gradient_block`` of src/mpifield/edges.py:217-259, restated on NumPy.
- `halo_fill`, `halo_fold`: the one-block periodic halo copy and accumulation of the
  external ``mpiarray`` 0.2.1 (called at src/mpifield/field.py:613,630), restated from
  the method cards at field.py:601-630 (axis by axis, the layers spanning the whole
  storage along the other axes; halos beyond a wall untouched on fill, dropped on fold).
- `node_volumes`: ``Field.node_volumes`` of field.py:563-588.
- `cpu_gather`, `cpu_scatter`, `cpu_deposit_*`: the OpenMP restatement of the Pyccel
  kernels in ``cpu_baseline.c``, the reported CPU baseline.
- `RefHost`: the reference's own ``.cu`` kernels compiled as serial C++
  (``oracle/_ref``), which pins the restatement.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
KINDS = {"linear": 0, "quadratic": 1, "spline": 2}

_lib = None


def library() -> C.CDLL:
    """The oracle library, built on first use if missing."""
    global _lib
    if _lib is None:
        from oracle.build_oracle import build_oracle

        path = build_oracle()
        _lib = C.CDLL(str(path))
        _declare(_lib)
    return _lib


_P = C.c_void_p
_I = C.c_int
_L = C.c_int64


def _declare(lib: C.CDLL) -> None:
    sig = {
        "og_gather": [_I, _I, _I, _P, _L, _L, _P, _L, _P, _L, _P, _P, _P, _P],
        "og_scatter": [_I, _I, _I, _P, _L, _P, _L, _L, _P, _L, _P, _P, _P, _P],
        "og_gather_grad": [_I, _I, _I, _P, _L, _L, _P, _L, _P, _L, _P, _L, _P, _P, _P, _P],
        "og_deposit_whitney": [_I, _P, _L, _P, _L, _P, _L, _P, _P, _P, _P, _P],
        "og_deposit_spline": [_I, _I, _P, _L, _P, _L, _P, _L, _P, _P, _P, _P, _P],
        "og_gather_edges": [_I, _I, _P, _L, _L, _P, _P, _L, _P, _P, _P, _P],
        "og_tile_keys": [_I, _I, _I, _P, _L, _P, _L, _L, _L, _P, _P, _P, _P, _P, _I, _P],
        "og_gather_forms": [_I, _I, _I, _P, _L, _L, _P, _L, _P, _L, _P, _P, _P, _P],
        "og_scatter_forms": [_I, _I, _I, _P, _L, _P, _L, _L, _P, _L, _P, _P, _P, _P],
        "cb_gather": [_I, _I, _I, _P, _L, _L, _P, _L, _P, _L, _P, _P, _P, _P, _I],
        "cb_scatter": [_I, _I, _I, _P, _L, _P, _L, _L, _P, _L, _P, _P, _P, _P, _I],
        "cb_deposit_whitney": [_I, _P, _L, _P, _L, _P, _L, _P, _P, _P, _P, _P, _I],
        "cb_deposit_spline": [_I, _I, _P, _L, _P, _L, _P, _L, _P, _P, _P, _P, _P],
    }
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _I if name.startswith("cb_") else None


# ------------------------------------------------------------------ helpers --


def split_geometry(geometry) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """``(*lower, *cell, *num, *code)`` as four arrays (float64, float64, int32, int32)."""
    ndim = len(geometry) // 4
    lower = np.ascontiguousarray(geometry[:ndim], dtype=np.float64)
    cell = np.ascontiguousarray(geometry[ndim : 2 * ndim], dtype=np.float64)
    num = np.ascontiguousarray(geometry[2 * ndim : 3 * ndim], dtype=np.int32)
    code = np.ascontiguousarray(geometry[3 * ndim :], dtype=np.int32)
    return lower, cell, num, code


def _rows(a: np.ndarray) -> tuple[np.ndarray, int]:
    """A 2D float64 array with unit column stride and its row stride in elements."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 1:
        a = a.reshape(1, -1)
    if a.strides[1] != 8 or a.strides[0] % 8:
        a = np.ascontiguousarray(a)
    stride = a.strides[0] // 8 if a.shape[0] > 1 else a.shape[1]
    return a, stride


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _kind(kind) -> int:
    return KINDS[kind] if isinstance(kind, str) else int(kind)


def field_extent(num, code, degree) -> tuple[int, ...]:
    """The node extent of an array along each axis (num + p - 1 on clamped axes)."""
    return tuple(int(n) + (degree - 1 if c == 2 else 0) for n, c in zip(num, code))


# ---------------------------------------------------------------- node kernels --


def gather(kind, degree: int, positions: np.ndarray, field: np.ndarray, geometry) -> np.ndarray:
    """``result (ncomp, N)`` of the reference gather with ``kind`` weights."""
    lower, cell, num, code = split_geometry(geometry)
    pos, ps = _rows(positions)
    field = np.ascontiguousarray(field, dtype=np.float64)
    ncomp = field.shape[-1]
    n = pos.shape[1]
    result = np.zeros((ncomp, n))
    library().og_gather(_kind(kind), degree, lower.size, _ptr(pos), ps, n, _ptr(field), ncomp,
                        _ptr(result), n, _ptr(lower), _ptr(cell), _ptr(num), _ptr(code))
    return result


def scatter(kind, degree: int, positions, values, field: np.ndarray, geometry) -> np.ndarray:
    """Add the reference deposit of ``values (ncomp, N)`` into ``field`` (in place); returns it."""
    lower, cell, num, code = split_geometry(geometry)
    pos, ps = _rows(positions)
    vals, vs = _rows(values)
    assert field.flags.c_contiguous and field.dtype == np.float64
    ncomp = field.shape[-1]
    library().og_scatter(_kind(kind), degree, lower.size, _ptr(pos), ps, _ptr(vals), vs,
                         pos.shape[1], _ptr(field), ncomp, _ptr(lower), _ptr(cell), _ptr(num),
                         _ptr(code))
    return field


def gather_grad(kind, degree: int, positions, field, cotangent, geometry) -> np.ndarray:
    """``(ndim, N)``: d/dx of sum_c cotangent_c * gather_c, the position gradient."""
    lower, cell, num, code = split_geometry(geometry)
    pos, ps = _rows(positions)
    cot, cs = _rows(cotangent)
    field = np.ascontiguousarray(field, dtype=np.float64)
    n = pos.shape[1]
    grad = np.zeros((lower.size, n))
    library().og_gather_grad(_kind(kind), degree, lower.size, _ptr(pos), ps, n, _ptr(field),
                             field.shape[-1], _ptr(cot), cs, _ptr(grad), n, _ptr(lower),
                             _ptr(cell), _ptr(num), _ptr(code))
    return grad


def deposit_whitney(start, end, charges, edges: np.ndarray, geometry) -> np.ndarray:
    """Add the WHITNEY current of the paths to ``edges`` (num + (ndim,)), in place."""
    lower, cell, num, code = split_geometry(geometry)
    s, ss = _rows(start)
    e, es = _rows(end)
    q = np.ascontiguousarray(charges, dtype=np.float64).reshape(-1)
    assert edges.flags.c_contiguous and edges.dtype == np.float64
    library().og_deposit_whitney(lower.size, _ptr(s), ss, _ptr(e), es, _ptr(q), q.size,
                                 _ptr(edges), _ptr(lower), _ptr(cell), _ptr(num), _ptr(code))
    return edges


def deposit_spline(degree: int, start, end, charges, edges: np.ndarray, geometry) -> np.ndarray:
    """Add the spline-edge current of degree 1-3 to ``edges``, in place."""
    lower, cell, num, code = split_geometry(geometry)
    s, ss = _rows(start)
    e, es = _rows(end)
    q = np.ascontiguousarray(charges, dtype=np.float64).reshape(-1)
    assert edges.flags.c_contiguous and edges.dtype == np.float64
    library().og_deposit_spline(lower.size, degree, _ptr(s), ss, _ptr(e), es, _ptr(q), q.size,
                                _ptr(edges), _ptr(lower), _ptr(cell), _ptr(num), _ptr(code))
    return edges


def gather_edges(degree: int, positions, edges, geometry) -> np.ndarray:
    """The field ``(ndim, N)`` of an edge field; degree 0 selects the Whitney functions."""
    lower, cell, num, code = split_geometry(geometry)
    pos, ps = _rows(positions)
    edges = np.ascontiguousarray(edges, dtype=np.float64)
    n = pos.shape[1]
    result = np.zeros((lower.size, n))
    library().og_gather_edges(lower.size, degree, _ptr(pos), ps, n, _ptr(edges), _ptr(result), n,
                              _ptr(lower), _ptr(cell), _ptr(num), _ptr(code))
    return result


def num_form_components(form: int, ndim: int) -> int:
    """The components of a ``form``-form in ``ndim`` dimensions (spline_forms.py:43-48)."""
    return {(1, 1): 1, (1, 2): 2, (2, 2): 1, (1, 3): 3, (2, 3): 3, (3, 3): 1}[(form, ndim)]


def gather_forms(degree: int, form: int, positions, field: np.ndarray, geometry) -> np.ndarray:
    """``result (ncomp, N)`` of the reference k-form gather (gather_forms_spline)."""
    lower, cell, num, code = split_geometry(geometry)
    pos, ps = _rows(positions)
    field = np.ascontiguousarray(field, dtype=np.float64)
    ncomp = field.shape[-1]
    n = pos.shape[1]
    result = np.zeros((ncomp, n))
    library().og_gather_forms(lower.size, degree, form, _ptr(pos), ps, n, _ptr(field), ncomp, _ptr(result), n,
                              _ptr(lower), _ptr(cell), _ptr(num), _ptr(code))
    return result


def scatter_forms(degree: int, form: int, positions, values, field: np.ndarray, geometry) -> np.ndarray:
    """Add the reference k-form deposit of ``values (ncomp, N)`` to ``field`` (in place); returns it."""
    lower, cell, num, code = split_geometry(geometry)
    pos, ps = _rows(positions)
    vals, vs = _rows(values)
    assert field.flags.c_contiguous and field.dtype == np.float64
    library().og_scatter_forms(lower.size, degree, form, _ptr(pos), ps, _ptr(vals), vs, pos.shape[1], _ptr(field),
                               field.shape[-1], _ptr(lower), _ptr(cell), _ptr(num), _ptr(code))
    return field


def tile_keys(kind, degree: int, positions, geometry, tile, values=None, within: bool = False) -> np.ndarray:
    """The cell-tile key of every marker (uint32); dead markers get the sentinel key."""
    lower, cell, num, code = split_geometry(geometry)
    pos, ps = _rows(positions)
    tile = np.ascontiguousarray(tile, dtype=np.int32)
    n = pos.shape[1]
    keys = np.zeros(n, dtype=np.uint32)
    if values is None:
        vptr, vs, ncomp = None, 0, 0
    else:
        vals, vs = _rows(values)
        vptr, ncomp = _ptr(vals), vals.shape[0]
    library().og_tile_keys(_kind(kind), degree, lower.size, _ptr(pos), ps, vptr, vs, ncomp, n,
                           _ptr(lower), _ptr(cell), _ptr(num), _ptr(code), _ptr(tile), int(bool(within)),
                           _ptr(keys))
    return keys


def sort_by_tile(keys: np.ndarray) -> np.ndarray:
    """The stable order of the keys (the permutation the sort must produce)."""
    return np.argsort(keys, kind="stable").astype(np.int32)


# ---------------------------------------------------------- edge incidence --


def gradient_block(nodes: np.ndarray, periodic) -> np.ndarray:
    """``G phi``: the difference of a node field along every edge (edges.py:217-237)."""
    ndim = nodes.ndim
    result = np.zeros((*nodes.shape, ndim))
    for axis, wraps in enumerate(periodic):
        if wraps:
            result[..., axis] = np.roll(nodes, -1, axis=axis) - nodes
        else:
            lo = [slice(None)] * ndim
            hi = [slice(None)] * ndim
            lo[axis] = slice(0, -1)
            hi[axis] = slice(1, None)
            result[(*lo, axis)] = nodes[tuple(hi)] - nodes[tuple(lo)]
    return result


def divergence_block(edges: np.ndarray, periodic) -> np.ndarray:
    """``G^T j``: the transpose of `gradient_block` (edges.py:239-259)."""
    ndim = edges.ndim - 1
    result = np.zeros(edges.shape[:-1])
    for axis, wraps in enumerate(periodic):
        flow = edges[..., axis]
        if wraps:
            result += np.roll(flow, 1, axis=axis) - flow
        else:
            lo = [slice(None)] * ndim
            hi = [slice(None)] * ndim
            lo[axis] = slice(0, -1)
            hi[axis] = slice(1, None)
            result[tuple(lo)] -= flow[tuple(lo)]
            result[tuple(hi)] += flow[tuple(lo)]
    return result


# ---------------------------------------------------------------------- halos --


def halo_fill(stored: np.ndarray, halo: int, periodic) -> np.ndarray:
    """Fill the halo nodes of one block from the wrapped interior, axis by axis (in place).

    ``stored`` is ``(n_0 + 2h, ..., ncomp)``. On a periodic axis the low halo takes
    the last ``h`` owned nodes and the high halo the first ``h``; the layers span the
    whole storage along the other axes, so corners are filled too. At a wall the halos
    are left unchanged.
    """
    h = halo
    for axis, wraps in enumerate(periodic):
        if not wraps or h == 0:
            continue
        n = stored.shape[axis] - 2 * h
        src_hi = [slice(None)] * stored.ndim
        dst_lo = [slice(None)] * stored.ndim
        src_hi[axis] = slice(n, n + h)
        dst_lo[axis] = slice(0, h)
        stored[tuple(dst_lo)] = stored[tuple(src_hi)]
        src_lo = [slice(None)] * stored.ndim
        dst_hi = [slice(None)] * stored.ndim
        src_lo[axis] = slice(h, 2 * h)
        dst_hi[axis] = slice(n + h, n + 2 * h)
        stored[tuple(dst_hi)] = stored[tuple(src_lo)]
    return stored


def halo_fold(stored: np.ndarray, halo: int, periodic) -> np.ndarray:
    """Add the halo nodes onto their wrapped owners and clear them, axis by axis (in place).

    On a periodic axis the high halo adds onto the first ``h`` owned nodes and the low
    halo onto the last ``h``; at a wall the halo values are dropped (zeroed).
    """
    h = halo
    if h == 0:
        return stored
    for axis, wraps in enumerate(periodic):
        n = stored.shape[axis] - 2 * h
        lo = [slice(None)] * stored.ndim
        hi = [slice(None)] * stored.ndim
        lo[axis] = slice(0, h)
        hi[axis] = slice(n + h, n + 2 * h)
        if wraps:
            first = [slice(None)] * stored.ndim
            last = [slice(None)] * stored.ndim
            first[axis] = slice(h, 2 * h)
            last[axis] = slice(n, n + h)
            stored[tuple(first)] += stored[tuple(hi)]
            stored[tuple(last)] += stored[tuple(lo)]
        stored[tuple(lo)] = 0.0
        stored[tuple(hi)] = 0.0
    return stored


def node_volumes(num, cell, periodic) -> np.ndarray:
    """The volume each node collects: prod(h), halved per bounded end node (field.py:563-588)."""
    result = np.ones(tuple(int(n) for n in num))
    for axis, (n, h, wraps) in enumerate(zip(num, cell, periodic)):
        factor = np.full(int(n), float(h))
        if not wraps:
            factor[0] *= 0.5
            factor[-1] *= 0.5
        shape = [1] * len(num)
        shape[axis] = int(n)
        result = result * factor.reshape(shape)
    return result


# ------------------------------------------------------------- CPU baseline --


def cpu_gather(kind, degree, positions, field, geometry, threads=0) -> np.ndarray:
    """The Pyccel-structured OpenMP gather (the CPU baseline)."""
    lower, cell, num, code = split_geometry(geometry)
    pos, ps = _rows(positions)
    field = np.ascontiguousarray(field, dtype=np.float64)
    n = pos.shape[1]
    result = np.zeros((field.shape[-1], n))
    library().cb_gather(_kind(kind), degree, lower.size, _ptr(pos), ps, n, _ptr(field),
                        field.shape[-1], _ptr(result), n, _ptr(lower), _ptr(cell), _ptr(num),
                        _ptr(code), threads)
    return result


def cpu_scatter(kind, degree, positions, values, field, geometry, threads=0) -> int:
    """The Pyccel-structured OpenMP scatter into ``field``; returns the threads used."""
    lower, cell, num, code = split_geometry(geometry)
    pos, ps = _rows(positions)
    vals, vs = _rows(values)
    return library().cb_scatter(_kind(kind), degree, lower.size, _ptr(pos), ps, _ptr(vals), vs,
                                pos.shape[1], _ptr(field), field.shape[-1], _ptr(lower),
                                _ptr(cell), _ptr(num), _ptr(code), threads)


def cpu_deposit(degree, start, end, charges, edges, geometry, threads=0) -> int:
    """The Pyccel-structured path deposit (Whitney for degree 1 per-thread, spline serial)."""
    lower, cell, num, code = split_geometry(geometry)
    s, ss = _rows(start)
    e, es = _rows(end)
    q = np.ascontiguousarray(charges, dtype=np.float64).reshape(-1)
    if degree == 1:
        return library().cb_deposit_whitney(lower.size, _ptr(s), ss, _ptr(e), es, _ptr(q), q.size,
                                            _ptr(edges), _ptr(lower), _ptr(cell), _ptr(num),
                                            _ptr(code), threads)
    return library().cb_deposit_spline(lower.size, degree, _ptr(s), ss, _ptr(e), es, _ptr(q),
                                       q.size, _ptr(edges), _ptr(lower), _ptr(cell), _ptr(num),
                                       _ptr(code))


# ----------------------------------------------------- the reference, compiled --


class RefHost:
    """The reference's ``.cu`` kernels compiled as serial host C++ (``oracle/_ref``)."""

    def __init__(self) -> None:
        path = HERE / "_ref" / "libref_host.so"
        if not path.exists():
            from oracle.build_oracle import build_ref_host

            built = build_ref_host()
            if built is None:
                raise FileNotFoundError("oracle/_ref/libref_host.so is not built")
        self.lib = C.CDLL(str(path))

    def available(self, name: str) -> bool:
        return hasattr(self.lib, f"ref_{name}")

    def call(self, name: str, n_threads: int, *args) -> None:
        """Run kernel ``name`` for ``n_threads``; arrays are float64 NumPy arrays."""
        from oracle.build_oracle import kernel_parameters

        params = kernel_parameters(name)
        if len(params) != len(args):
            raise TypeError(f"{name} takes {len(params)} arguments, got {len(args)}")
        cargs: list = [C.c_longlong(n_threads)]
        keep = []
        for (kind, _, ndim), value in zip(params, args, strict=True):
            if kind == "array":
                assert isinstance(value, np.ndarray) and value.dtype == np.float64
                assert value.ndim == ndim, (name, value.shape, ndim)
                shape = (C.c_longlong * ndim)(*value.shape)
                strides = (C.c_longlong * ndim)(*(s // 8 for s in value.strides))
                keep += [shape, strides]
                cargs += [C.c_void_p(value.ctypes.data), shape, strides]
            elif kind == "double":
                cargs.append(C.c_double(float(value)))
            else:
                cargs.append(C.c_int(int(value)))
        getattr(self.lib, f"ref_{name}")(*cargs)
