"""The C ABI library and the host-side logic (CPU only: no kernel runs here).

The library loads and exports every entry point include/*.h declares; calls whose
arguments are invalid return their status before any device work; the Python layer
mirrors the reference's plug-in types and their errors (src/mpifield/weighting.py,
edges.py, splines.py, _types.py, field.py).
"""

from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import mpifield_b200 as mf
from mpifield_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols() -> set[str]:
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        names |= set(re.findall(r"MPF_API\s+[\w\s\*]+?\b(mpf_\w+)\s*\(", header.read_text()))
    return names


def test_the_library_exports_every_declared_entry_point():
    lib = _lib.library()
    declared = declared_symbols()
    assert {"mpf_gather", "mpf_scatter", "mpf_deposit_paths", "mpf_sort_by_tile"} <= declared
    for name in declared:
        assert hasattr(lib, name), name
    assert declared == set(_lib.symbols()) | (declared - set(_lib.symbols()))
    assert set(_lib.symbols()) <= declared
    assert lib.mpf_version() == 10000
    assert lib.mpf_status_string(_lib.ERR_ARGUMENT) == b"invalid argument"


def _geom(ndim=3, num=8, code=1):
    lower = (C.c_double * ndim)(*[0.0] * ndim)
    cell = (C.c_double * ndim)(*[0.1] * ndim)
    nums = (C.c_int32 * ndim)(*[num] * ndim)
    codes = (C.c_int32 * ndim)(*[code] * ndim)
    return lower, cell, nums, codes


def test_invalid_arguments_return_a_status_before_any_device_work():
    lib = _lib.library()
    lower, cell, num, code = _geom()
    fake = 1 << 20  # never dereferenced: every call below fails its checks first
    # a dimension out of range
    assert lib.mpf_gather(1, 2, 4, fake, 0, 10, fake, 1, fake, 0, lower, cell, num, code, 0, None, None) == _lib.ERR_ARGUMENT
    # LINEAR must be degree 1, QUADRATIC degree 2, splines 0..3
    assert lib.mpf_gather(0, 2, 3, fake, 0, 10, fake, 1, fake, 0, lower, cell, num, code, 0, None, None) == _lib.ERR_ARGUMENT
    assert lib.mpf_scatter(2, 4, 3, fake, 0, fake, 0, 10, fake, 1, lower, cell, num, code, 0, None, None) == _lib.ERR_ARGUMENT
    # a row stride below n
    assert lib.mpf_gather(1, 2, 3, fake, 5, 10, fake, 1, fake, 0, lower, cell, num, code, 0, None, None) == _lib.ERR_SHAPE
    # a misaligned pointer
    assert lib.mpf_gather(1, 2, 3, fake + 3, 0, 10, fake, 1, fake, 0, lower, cell, num, code, 0, None, None) == _lib.ERR_ALIGNMENT
    # clamped axes are for spline stencils of degree >= 1 (weighting.py:91-97)
    l2, c2, n2, k2 = _geom(code=2)
    assert lib.mpf_gather(1, 2, 3, fake, 0, 10, fake, 1, fake, 0, l2, c2, n2, k2, 0, None, None) == _lib.ERR_UNSUPPORTED
    assert lib.mpf_gather(2, 0, 3, fake, 0, 10, fake, 1, fake, 0, l2, c2, n2, k2, 0, None, None) == _lib.ERR_UNSUPPORTED
    # a bounded axis needs two nodes
    l1, c1, n1, k1 = _geom(num=1, code=0)
    assert lib.mpf_gather(1, 2, 3, fake, 0, 10, fake, 1, fake, 0, l1, c1, n1, k1, 0, None, None) == _lib.ERR_ARGUMENT
    # a zero cell size
    zero = (C.c_double * 3)(0.0, 0.1, 0.1)
    assert lib.mpf_gather(1, 2, 3, fake, 0, 10, fake, 1, fake, 0, lower, zero, num, code, 0, None, None) == _lib.ERR_ARGUMENT
    # WHITNEY is degree 1; spline edges 1..3
    assert lib.mpf_deposit_paths(0, 2, 3, fake, 0, fake, 0, fake, 10, fake, lower, cell, num, code, 0, None, None) == _lib.ERR_ARGUMENT
    assert lib.mpf_deposit_paths(2, 0, 3, fake, 0, fake, 0, fake, 10, fake, lower, cell, num, code, 0, None, None) == _lib.ERR_ARGUMENT
    # a dtype other than f64 / f32
    assert lib.mpf_gather(1, 2, 3, fake, 0, 10, fake, 1, fake, 0, lower, cell, num, code, 7, None, None) == _lib.ERR_ARGUMENT
    # halos wider than the owned block
    stored = (C.c_int32 * 1)(3)
    per = (C.c_int32 * 1)(1)
    assert lib.mpf_halo_fold(fake, 1, stored, 1, 2, per, 0, None) == _lib.ERR_SHAPE
    # halo slabs: an axis outside the block, a slab past the storage, a misaligned buffer
    s2 = (C.c_int32 * 2)(6, 5)
    assert lib.mpf_halo_pack(fake, 2, s2, 1, 2, 2, 0, fake, 0, None) == _lib.ERR_ARGUMENT
    assert lib.mpf_halo_pack(fake, 2, s2, 1, 2, 1, 4, fake, 0, None) == _lib.ERR_SHAPE
    assert lib.mpf_halo_unpack(fake, 2, s2, 1, 2, 0, 0, fake + 4, 1, 0, None) == _lib.ERR_ALIGNMENT
    assert lib.mpf_halo_unpack(fake, 2, s2, 1, 0, 0, 0, fake, 1, 0, None) == _lib.ERR_ARGUMENT
    # the deterministic scatter: a workspace too small, misaligned
    size = C.c_size_t()
    assert lib.mpf_scatter_deterministic_workspace_bytes(8 * 8 * 8, C.byref(size)) == 0
    assert size.value >= 2 * 8 * 512
    assert lib.mpf_scatter_deterministic(1, 2, 3, fake, 0, fake, 0, 10, fake, 1, lower, cell, num, code, fake,
                                         16, None) == _lib.ERR_WORKSPACE
    assert lib.mpf_scatter_deterministic(1, 2, 3, fake, 0, fake, 0, 10, fake, 1, lower, cell, num, code, fake + 8,
                                         size.value, None) == _lib.ERR_ALIGNMENT
    # the re-sort: a workspace too small, the previous keys given as the output
    t3 = (C.c_int32 * 3)(4, 4, 4)
    size = C.c_size_t()
    assert lib.mpf_resort_workspace_bytes(1, 2, 3, num, code, t3, 1, 1000, C.byref(size)) == 0
    assert lib.mpf_resort_by_tile(1, 2, 3, fake, 0, None, 0, 0, 1000, lower, cell, num, code, t3, 1, None, fake, fake,
                                  fake, fake, 16, 0, None) == _lib.ERR_WORKSPACE
    assert lib.mpf_resort_by_tile(1, 2, 3, fake, 0, None, 0, 0, 1000, lower, cell, num, code, t3, 1, fake, fake, fake,
                                  fake, fake, size.value, 0, None) == _lib.ERR_ARGUMENT
    # a workspace too small
    t = (C.c_int32 * 3)(4, 4, 4)
    assert lib.mpf_sort_by_tile(1, 2, 3, fake, 0, None, 0, 0, 1000, lower, cell, num, code, t, 0, fake, fake, fake,
                                fake, 16, 0, None) == _lib.ERR_WORKSPACE


def test_the_sort_without_allocation_checks_everything_before_any_cuda_call():
    # no CUDA device here: a call that reached the device would return MPF_ERR_CUDA
    lib = _lib.library()
    lower, cell, num, code = _geom()
    t = (C.c_int32 * 3)(4, 4, 4)
    fake = 1 << 20  # never dereferenced
    most = 1 << 20  # MPF_NOALLOC_MAX_MARKERS

    def call(n=1000, kind=1, degree=2, ndim=3, pos=fake, within=0, dtype=0, order=fake):
        return lib.mpf_sort_by_tile_noalloc(kind, degree, ndim, pos, 0, None, 0, 0, n, lower, cell, num, code, t,
                                            within, fake, order, fake, dtype, None)

    assert call(n=most + 1) == _lib.ERR_WORKSPACE
    assert call(n=-1) == _lib.ERR_ARGUMENT
    assert call(kind=0) == _lib.ERR_ARGUMENT  # LINEAR is degree 1
    assert call(ndim=4) == _lib.ERR_ARGUMENT
    assert call(within=2) == _lib.ERR_ARGUMENT
    assert call(dtype=5) == _lib.ERR_ARGUMENT
    assert call(pos=fake + 3) == _lib.ERR_ALIGNMENT
    assert call(order=0) == _lib.ERR_ARGUMENT
    assert lib.mpf_last_error() == b"none"


def test_tile_counts_and_workspace_sizes():
    lib = _lib.library()
    num = (C.c_int32 * 3)(256, 256, 256)
    code = (C.c_int32 * 3)(1, 1, 1)
    tile = (C.c_int32 * 3)(8, 8, 8)
    out = C.c_int64()
    assert lib.mpf_num_tiles(1, 2, 3, num, code, tile, C.byref(out)) == 0
    assert out.value == 32 ** 3
    # a clamped axis of degree 3 holds num + 2 entries
    code2 = (C.c_int32 * 3)(2, 1, 1)
    assert lib.mpf_num_tiles(2, 3, 3, num, code2, tile, C.byref(out)) == 0
    assert out.value == 33 * 32 * 32
    size = C.c_size_t()
    assert lib.mpf_sort_workspace_bytes(1 << 20, 32768, C.byref(size)) == 0
    assert size.value >= 16 * (1 << 20)
    assert lib.mpf_sort_workspace_bytes(-1, 1, C.byref(size)) == _lib.ERR_ARGUMENT


def test_block_grid_from_geometry():
    # src/mpifield/tests/unit/test_weighting.py:191-199
    grid = mf.BlockGrid.from_geometry((0.0, 0.0), (0.5, 0.5), (3, 3), (True, False))
    assert grid.geometry == (0.0, 0.0, 0.5, 0.5, 3, 3, 1, 0)
    with pytest.raises(ValueError, match="differ in length"):
        mf.BlockGrid.from_geometry((0.0,), (0.5, 0.5), (3, 3))
    with pytest.raises(ValueError, match="either periodic or clamped"):
        mf.BlockGrid.from_geometry((0.0,), (0.5,), (3,), (True,), (True,))
    grid = mf.BlockGrid.from_geometry((0.0,), (0.5,), (3,), None, (True,))
    assert grid.geometry[-1] == 2


def test_weighting_checks_and_reprs():
    # test_weighting.py:67-79 and test_splines.py
    with pytest.raises(ValueError, match="halo must be >= 0"):
        mf.Weighting("bad", scatter={}, gather={}, halo=-1)
    with pytest.raises(ValueError, match="1, 2 or 3 dimensions, got 4"):
        mf.Weighting("bad", scatter={4: print}, gather={})
    with pytest.raises(ValueError, match="degree must be >= 0"):
        mf.Weighting("bad", scatter={}, gather={}, degree=-1)
    assert (mf.LINEAR.halo, mf.QUADRATIC.halo, mf.CUBIC.halo) == (1, 2, 2)
    assert (mf.LINEAR.degree, mf.QUADRATIC.degree, mf.CUBIC.degree) == (1, 2, 3)
    assert repr(mf.CUBIC) == ("Weighting('cubic': scatter 1D/2D/3D; gather 1D/2D/3D; halo 2, degree 3, "
                              "takes clamped axes)")
    assert repr(mf.QUADRATIC_EDGES) == ("EdgeWeighting('quadratic': gather 1D/2D/3D; deposit_paths 1D/2D/3D; "
                                        "halo 2, degree 2, takes clamped axes)")
    assert mf.CUBIC.dimensions() == (1, 2, 3)
    with pytest.raises(ValueError, match="degree must be >= 1"):
        mf.EdgeWeighting("bad", gather={}, deposit_paths={}, degree=0)
    with pytest.raises(ValueError, match=r"the bad edge weighting has no 2D deposit_paths kernel \(has none\)"):
        mf.EdgeWeighting("bad", gather={}, deposit_paths={}).deposit_paths_kernel(2)
    assert (mf.WHITNEY.degree, mf.QUADRATIC_EDGES.degree, mf.CUBIC_EDGES.degree) == (1, 2, 3)
    with pytest.raises(TypeError):
        mf.LINEAR.scatter[2] = print  # read-only mapping
    mine = mf.Weighting("mine", scatter={2: print}, gather={2: print})
    with pytest.raises(ValueError, match="no 3D scatter kernel"):
        mine.scatter_kernel(3)
    with pytest.raises(ValueError, match=r"no 1D gather kernel \(has 2D\)"):
        mine.gather_kernel(1)


def test_splines_pair_the_weightings():
    assert tuple(mf.SPLINES) == (1, 2, 3)
    assert mf.splines(1).nodes is mf.LINEAR and mf.splines(1).edges is mf.WHITNEY
    assert mf.splines(2).nodes is mf.QUADRATIC and mf.splines(2).edges is mf.QUADRATIC_EDGES
    assert mf.splines(3).nodes is mf.CUBIC and mf.splines(3).edges is mf.CUBIC_EDGES
    assert [mf.splines(p).halo for p in (1, 2, 3)] == [1, 2, 2]
    assert repr(mf.splines(1)) == ("Splines(degree 1: nodes='linear', edges='whitney', faces='linear faces', "
                                   "cells='linear cells')")
    assert mf.splines(1).forms()[:2] == (mf.LINEAR, mf.WHITNEY)
    assert mf.splines(2).faces.dimensions() == (3,) and mf.splines(2).cells.dimensions() == (1, 2, 3)
    assert all(w.clamps for w in mf.splines(1, clamped=True).forms())
    with pytest.raises(ValueError, match="no built-in splines of degree 5"):
        mf.splines(5)
    with pytest.raises(ValueError, match="an integer"):
        mf.splines(1.5)
    with pytest.raises(ValueError, match="has degree 1, not 2"):
        mf.Splines(2, mf.LINEAR)
    assert mf.splines(2, clamped=True).nodes.clamps


def test_clamped_grids_need_a_clamping_weighting():
    grid = mf.BlockGrid.from_geometry((0.0,), (0.5,), (3,), None, (True,))
    with pytest.raises(ValueError, match="does not take clamped axes"):
        mf.QUADRATIC.scatter_block(np.zeros((1, 1)), np.zeros((1, 1)), np.zeros((3, 1)), grid)


def test_the_kernels_refuse_cpu_tensors():
    import torch

    field = torch.zeros(8, 1, dtype=torch.float64)
    with pytest.raises(TypeError, match="no CPU fallback"):
        mf.KERNELS["gather_quadratic_1d"](torch.zeros(1, 4, dtype=torch.float64), field,
                                          torch.zeros(1, 4, dtype=torch.float64), 0.0, 0.1, 8, 1)


def test_the_catalog_has_the_reference_kernel_names():
    # src/mpifield/kernels/catalog.py:51-93 (the hot-path and edge-gather kernels)
    for n in (1, 2, 3):
        for name in ("gather_linear", "scatter_linear", "gather_quadratic", "scatter_quadratic", "gather_spline",
                     "scatter_spline", "deposit_paths", "deposit_paths_spline", "gather_edges",
                     "gather_edges_spline", "gather_forms_spline", "scatter_forms_spline"):
            assert f"{name}_{n}d" in mf.KERNELS
