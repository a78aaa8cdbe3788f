"""mpifield's own plug-in classes driving this backend's kernels (CPU, no GPU needed).

The reference's ``weighting.py`` and ``edges.py`` are loaded from the mpifield sources
(``MPF_REFERENCE_SRC``, else the ``reference/src`` folder beside this repository; the
test is skipped where neither exists) with every kernel module they import replaced by
this backend's kernel of the same name (`mpifield_b200.KERNELS`): the reference then
builds its own LINEAR, QUADRATIC, CUBIC, WHITNEY, QUADRATIC_EDGES and CUBIC_EDGES from
our kernels, exactly as a user would plug the backend in. The stub of ``cunumpy`` hands
the kernels "device arrays" as CuPy does: objects with ``__cuda_array_interface__``,
whose memory here is host memory. The C library is replaced by a recorder that checks
each call's arguments and runs the oracle (the C restatement of the reference kernels)
on the same pointers, so the whole host side -- the reference's own call (including its
special LINEAR signatures: one component ``(N,)`` in 1D, the grid as rows in 3D,
src/mpifield/weighting.py:259-330), our array adapter, the C-ABI arguments -- is checked
against the oracle called directly.
"""

from __future__ import annotations

import contextlib
import ctypes as C
import importlib.util
import os
import sys
import types
from pathlib import Path

import numpy as np
import pytest

import mpifield_b200 as mf
from mpifield_b200 import _lib
from oracle import oracle as O
from tests.helpers import RTOL_F64, rel_err

ROOT = Path(__file__).resolve().parents[1]
SRC = Path(os.environ.get("MPF_REFERENCE_SRC", ROOT.parent / "reference" / "src"))

pytestmark = pytest.mark.skipif(not (SRC / "mpifield" / "weighting.py").exists(),
                                reason="the mpifield sources are not here")


class FakeDeviceArray:
    """A CuPy-like array: ``__cuda_array_interface__`` (version 3) over host memory."""

    def __init__(self, array: np.ndarray):
        self.a = array

    @property
    def __cuda_array_interface__(self):
        return {"shape": self.a.shape, "typestr": self.a.dtype.str, "data": (self.a.ctypes.data, False),
                "strides": self.a.strides, "version": 3, "stream": None}

    shape = property(lambda self: self.a.shape)
    ndim = property(lambda self: self.a.ndim)
    dtype = property(lambda self: self.a.dtype)
    flags = property(lambda self: self.a.flags)

    def __getitem__(self, key):
        return FakeDeviceArray(self.a[key])

    def reshape(self, *shape):
        view = self.a.reshape(*shape)
        assert np.shares_memory(view, self.a)
        return FakeDeviceArray(view)


def _cunumpy_stub():
    xp = types.ModuleType("cunumpy")
    kernels = types.ModuleType("cunumpy.kernels")

    def as_kernel_array(x, like=None, dtype=float, strided=False):
        if isinstance(x, FakeDeviceArray):
            return x
        a = np.asarray(x, dtype=np.float64)
        return FakeDeviceArray(a if strided else np.ascontiguousarray(a))

    @contextlib.contextmanager
    def kernel_output(target, like=None, dtype=float, strided=False):
        a = target.a
        rows_ok = a.flags.c_contiguous or (strided and a.ndim == 2 and a.strides[-1] == a.itemsize)
        if rows_ok:
            yield target
            return
        work = np.ascontiguousarray(a)
        yield FakeDeviceArray(work)
        a[...] = work

    kernels.as_kernel_array = as_kernel_array
    kernels.kernel_output = kernel_output
    xp.kernels = kernels
    xp.is_gpu = lambda a: isinstance(a, FakeDeviceArray)
    xp.cuda = types.SimpleNamespace(shared_memory_fits=lambda n: True)
    return xp


class _AnyAttribute(types.ModuleType):
    def __getattr__(self, name):
        return None


def _load(name: str, path: Path):
    spec = importlib.util.spec_from_file_location(name, path)
    module = importlib.util.module_from_spec(spec)
    sys.modules[name] = module
    spec.loader.exec_module(module)
    return module


@pytest.fixture(scope="module")
def reference():
    saved = dict(sys.modules)
    stub = types.ModuleType("methodcard")
    stub.method = lambda *args, **kwargs: (lambda f: f)
    sys.modules["methodcard"] = stub
    sys.modules["cunumpy"] = _cunumpy_stub()
    for name, path in (("mpifield", SRC / "mpifield"), ("mpifield.kernels", SRC / "mpifield" / "kernels")):
        package = types.ModuleType(name)
        package.__path__ = [str(path)]
        sys.modules[name] = package
    sys.modules["mpifield._method_checks"] = _AnyAttribute("mpifield._method_checks")
    for name, kernel in mf.KERNELS.items():
        module = types.ModuleType(f"mpifield.kernels.{name}")
        module.kernel = kernel  # the reference's kernel of this name is ours
        sys.modules[module.__name__] = module
    numpy_1d = types.ModuleType("mpifield.kernels.scatter_linear_1d.scatter_linear_1d_numpy")
    numpy_1d.scatter_linear_1d = None  # not reached: the shared-memory path always fits here
    sys.modules[numpy_1d.__name__] = numpy_1d
    rows_3d = types.ModuleType("mpifield.kernels.scatter_rows_3d")
    rows_3d.kernel = None  # reached for NumPy arrays only
    sys.modules[rows_3d.__name__] = rows_3d
    _load("mpifield._types", SRC / "mpifield" / "_types.py")
    weighting = _load("mpifield.weighting", SRC / "mpifield" / "weighting.py")
    edges = _load("mpifield.edges", SRC / "mpifield" / "edges.py")
    splines = _load("mpifield.splines", SRC / "mpifield" / "splines.py")
    yield types.SimpleNamespace(weighting=weighting, edges=edges, splines=splines,
                                types=sys.modules["mpifield._types"])
    sys.modules.clear()
    sys.modules.update(saved)


class OracleLibrary:
    """Stands in for libmpifield_b200.so: checks the arguments of a call and runs the
    oracle on the same (host) memory."""

    def __init__(self):
        self.calls = []
        self.oracle = O.library()

    def _record(self, name, args):
        self.calls.append((name, args))

    def mpf_gather(self, kind, degree, ndim, pos, ps, n, field, ncomp, out, rs, lower, cell, num, code, dtype,
                   tuning, stream):
        self._record("gather", (kind, degree, ndim, ps, n, ncomp, rs, dtype, stream))
        assert dtype == _lib.F64 and stream == 0
        self.oracle.og_gather(kind, degree, ndim, pos, ps, n, field, ncomp, out, rs, C.addressof(lower),
                              C.addressof(cell), C.addressof(num), C.addressof(code))
        return 0

    def mpf_scatter(self, kind, degree, ndim, pos, ps, vals, vs, n, field, ncomp, lower, cell, num, code, dtype,
                    tuning, stream):
        self._record("scatter", (kind, degree, ndim, ps, vs, n, ncomp, dtype, stream))
        assert dtype == _lib.F64 and stream == 0
        self.oracle.og_scatter(kind, degree, ndim, pos, ps, vals, vs, n, field, ncomp, C.addressof(lower),
                               C.addressof(cell), C.addressof(num), C.addressof(code))
        return 0

    def mpf_deposit_paths(self, kind, degree, ndim, s, ss, e, es, q, n, edges, lower, cell, num, code, dtype, tuning,
                          stream):
        self._record("deposit_paths", (kind, degree, ndim, ss, es, n, dtype, stream))
        geometry = (C.addressof(lower), C.addressof(cell), C.addressof(num), C.addressof(code))
        if kind == _lib.LINEAR:
            self.oracle.og_deposit_whitney(ndim, s, ss, e, es, q, n, edges, *geometry)
        else:
            self.oracle.og_deposit_spline(ndim, degree, s, ss, e, es, q, n, edges, *geometry)
        return 0

    def mpf_gather_forms(self, degree, form, ndim, pos, ps, n, field, ncomp, out, rs, lower, cell, num, code, dtype,
                         stream):
        self._record("gather_forms", (degree, form, ndim, ps, n, ncomp, rs, dtype, stream))
        self.oracle.og_gather_forms(ndim, degree, form, pos, ps, n, field, ncomp, out, rs, C.addressof(lower),
                                    C.addressof(cell), C.addressof(num), C.addressof(code))
        return 0

    def mpf_scatter_forms(self, degree, form, ndim, pos, ps, vals, vs, n, field, ncomp, lower, cell, num, code,
                          dtype, stream):
        self._record("scatter_forms", (degree, form, ndim, ps, vs, n, ncomp, dtype, stream))
        self.oracle.og_scatter_forms(ndim, degree, form, pos, ps, vals, vs, n, field, ncomp, C.addressof(lower),
                                     C.addressof(cell), C.addressof(num), C.addressof(code))
        return 0

    def mpf_gather_edges(self, kind, degree, ndim, pos, ps, n, edges, out, rs, lower, cell, num, code, dtype,
                         stream):
        self._record("gather_edges", (kind, degree, ndim, ps, n, rs, dtype, stream))
        self.oracle.og_gather_edges(ndim, 0 if kind == _lib.LINEAR else degree, pos, ps, n, edges, out, rs,
                                    C.addressof(lower), C.addressof(cell), C.addressof(num), C.addressof(code))
        return 0


@pytest.fixture
def recorder(monkeypatch):
    fake = OracleLibrary()
    monkeypatch.setattr(_lib, "library", lambda: fake)
    return fake


def _grid(ref, ndim, periodic, clamped=False):
    shape = (9, 7, 6)[:ndim]
    lower = (0.0, -1.0, 2.0)[:ndim]
    cell = (0.25, 0.5, 0.1)[:ndim]
    flags = (periodic,) * ndim
    ends = ((clamped,) + (False,) * (ndim - 1)) if clamped else None
    if clamped:
        flags = (False,) + (periodic,) * (ndim - 1)
    return ref.types.BlockGrid.from_geometry(lower, cell, shape, flags, ends)


def _markers(rng, grid, n, rows):
    lo = np.asarray(grid.bounds.lower_bound)
    hi = np.asarray(grid.bounds.upper_bound)
    pad = 0.6 * np.asarray(grid.grid_spacing)
    pos = rng.uniform(lo - pad, hi + pad, (n, lo.size)).T
    # rows with a gap, as the reference's storage[:, :n]
    store = np.zeros((rows, n + 5))
    store[:, :n] = rng.uniform(0.5, 1.5, (rows, n))
    return np.ascontiguousarray(pos), store[:, :n]


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("name,kind,degree", [("LINEAR", "linear", 1), ("QUADRATIC", "quadratic", 2),
                                              ("CUBIC", "spline", 3)])
def test_the_reference_weightings_on_our_kernels(reference, recorder, ndim, name, kind, degree):
    rng = np.random.default_rng(ndim * 10 + degree)
    weighting = getattr(reference.weighting, name)
    for periodic in (False, True):
        grid = _grid(reference, ndim, periodic)
        ncomp = 2
        pos, values = _markers(rng, grid, 300, ncomp)
        shape = tuple(int(n) for n in grid.num_gridpoints)
        field = np.zeros(shape + (ncomp,))
        weighting.scatter_block(FakeDeviceArray(pos), FakeDeviceArray(values), FakeDeviceArray(field), grid)
        expected = O.scatter(kind, degree, pos, np.ascontiguousarray(values), np.zeros_like(field), grid.geometry)
        assert rel_err(field, expected) <= RTOL_F64
        source = rng.normal(size=shape + (ncomp,))
        result = np.zeros((ncomp, 300))
        weighting.gather_block(FakeDeviceArray(pos), FakeDeviceArray(source), FakeDeviceArray(result), grid)
        assert rel_err(result, O.gather(kind, degree, pos, source, grid.geometry)) <= RTOL_F64
    ops = {c[0] for c in recorder.calls}
    assert ops == {"scatter", "gather"}
    if name == "LINEAR" and ndim == 1:
        # the reference deposits one component at a time into (nx,) columns
        assert [c[1][6] for c in recorder.calls if c[0] == "scatter"] == [1, 1, 1, 1]


def test_a_users_weighting_made_of_our_kernels(reference, recorder):
    ref = reference.weighting
    mine = ref.Weighting("b200-quadratic",
                         scatter={n: mf.KERNELS[f"scatter_quadratic_{n}d"] for n in (1, 2, 3)},
                         gather={n: mf.KERNELS[f"gather_quadratic_{n}d"] for n in (1, 2, 3)}, halo=2, degree=2)
    rng = np.random.default_rng(3)
    grid = _grid(reference, 3, True)
    pos, values = _markers(rng, grid, 500, 2)
    field = np.zeros((9, 7, 6, 2))
    mine.scatter_block(FakeDeviceArray(pos), FakeDeviceArray(values), FakeDeviceArray(field), grid)
    expected = O.scatter("quadratic", 2, pos, np.ascontiguousarray(values), np.zeros_like(field), grid.geometry)
    assert rel_err(field, expected) <= RTOL_F64
    # the marker rows with their gap were passed as they are: row stride n + 5
    assert recorder.calls[-1][1][4] == 505


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("name,degree", [("WHITNEY", 1), ("QUADRATIC_EDGES", 2), ("CUBIC_EDGES", 3)])
def test_the_reference_edge_weightings_on_our_kernels(reference, recorder, ndim, name, degree):
    rng = np.random.default_rng(40 + ndim + degree)
    ew = getattr(reference.edges, name)
    grid = _grid(reference, ndim, True)
    shape = tuple(int(n) for n in grid.num_gridpoints)
    start, _ = _markers(rng, grid, 200, 1)
    end = start + rng.uniform(-0.9, 0.9, start.shape) * np.asarray(grid.grid_spacing)[:, None]
    q = rng.uniform(0.5, 1.5, 200)
    edges = np.zeros(shape + (ndim,))
    ew.deposit_paths_block(FakeDeviceArray(start), FakeDeviceArray(end), FakeDeviceArray(q),
                           FakeDeviceArray(edges), grid)
    expected = np.zeros_like(edges)
    if degree == 1:
        O.deposit_whitney(start, end, q, expected, grid.geometry)
    else:
        O.deposit_spline(degree, start, end, q, expected, grid.geometry)
    assert rel_err(edges, expected) <= RTOL_F64
    field = rng.normal(size=edges.shape)
    result = np.zeros((ndim, 200))
    ew.gather_block(FakeDeviceArray(start), FakeDeviceArray(field), FakeDeviceArray(result), grid)
    assert rel_err(result, O.gather_edges(0 if degree == 1 else degree, start, field, grid.geometry)) <= RTOL_F64


def test_our_block_types_accept_interface_arrays(recorder):
    # this package's own Weighting / EdgeWeighting on the same CuPy-like arrays
    rng = np.random.default_rng(8)
    grid = mf.BlockGrid.from_geometry((0.0, 0.0), (0.1, 0.2), (8, 6), (True, False))
    pos = np.ascontiguousarray(rng.uniform(0.0, 0.9, (2, 100)))
    field = np.zeros((8, 6, 1))
    mf.QUADRATIC.scatter_block(FakeDeviceArray(pos), FakeDeviceArray(np.ones(100)), FakeDeviceArray(field), grid)
    expected = O.scatter("quadratic", 2, pos, np.ones((1, 100)), np.zeros_like(field), grid.geometry)
    assert rel_err(field, expected) <= RTOL_F64


@pytest.mark.parametrize("degree", [1, 2, 3])
def test_the_reference_faces_and_cells_on_our_kernels(reference, recorder, degree):
    # mpifield's own Splines (src/mpifield/splines.py:185-205) built from our form kernels
    rng = np.random.default_rng(60 + degree)
    sp = reference.splines.SPLINES[degree]
    grid = _grid(reference, 3, True)
    pos, values = _markers(rng, grid, 300, 3)
    faces = np.zeros((9, 7, 6, 3))
    sp.faces.scatter_block(FakeDeviceArray(pos), FakeDeviceArray(values), FakeDeviceArray(faces), grid)
    expected = O.scatter_forms(degree, 2, pos, np.ascontiguousarray(values), np.zeros_like(faces), grid.geometry)
    assert rel_err(faces, expected) <= RTOL_F64
    for ndim in (1, 2, 3):
        g = _grid(reference, ndim, False)
        p, _ = _markers(rng, g, 200, 1)
        shape = tuple(int(n) for n in g.num_gridpoints)
        cells = rng.normal(size=shape + (1,))
        result = np.zeros((1, 200))
        sp.cells.gather_block(FakeDeviceArray(p), FakeDeviceArray(cells), FakeDeviceArray(result), g)
        assert rel_err(result, O.gather_forms(degree, ndim, p, cells, g.geometry)) <= RTOL_F64
    assert {c[0] for c in recorder.calls} == {"scatter_forms", "gather_forms"}
