"""The allocation-free sort entry point (mpf_sort_by_tile_noalloc), through the C ABI.

Some callers cannot call cudaMalloc: a host application that gives all device memory to
its own pool at start-up, a real-time loop that cannot afford an allocation's implicit
synchronisation. For them the library sorts in a fixed array of its own instead of a
caller's workspace. This test checks that two calls in a row (the array keeps the
previous call's contents) give exactly the keys, order and tile starts of
mpf_sort_by_tile with a workspace of its own. (Sizes above the array's limit and bad
arguments are refused before any CUDA call; tests/test_abi.py checks that without a
GPU.) It lives in a file of its own, collected last, so that a run stopping at the
first failure has run every other test first.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from mpifield_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_MARKERS = 1 << 20  # MPF_NOALLOC_MAX_MARKERS


def _geometry():
    lower = (C.c_double * 3)(0.0, -1.0, 0.5)
    cell = (C.c_double * 3)(1 / 64, 1 / 48, 1 / 40)
    num = (C.c_int32 * 3)(64, 96, 40)
    code = (C.c_int32 * 3)(1, 0, 1)
    tile = (C.c_int32 * 3)(8, 8, 4)
    return lower, cell, num, code, tile


def _sort(positions, values, within, noalloc):
    lib = _lib.library()
    lower, cell, num, code, tile = _geometry()
    n = positions.shape[1]
    ntiles = C.c_int64()
    _lib.check(lib.mpf_num_tiles(1, 2, 3, num, code, tile, C.byref(ntiles)), "num_tiles")
    keys = torch.empty(n, dtype=torch.int32, device="cuda")
    order = torch.empty(n, dtype=torch.int32, device="cuda")
    starts = torch.empty(ntiles.value + 2, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    args = (1, 2, 3, positions.data_ptr(), positions.stride(0), values.data_ptr(), values.stride(0), 1, n,
            lower, cell, num, code, tile, within, keys.data_ptr(), order.data_ptr(), starts.data_ptr())
    if noalloc:
        status = lib.mpf_sort_by_tile_noalloc(*args, _lib.F64, stream)
    else:
        size = C.c_size_t()
        _lib.check(lib.mpf_sort_workspace_bytes(n, ntiles.value, C.byref(size)), "workspace")
        workspace = torch.empty(size.value, dtype=torch.uint8, device="cuda")
        status = lib.mpf_sort_by_tile(*args, workspace.data_ptr(), size.value, _lib.F64, stream)
    _lib.check(status, "sort")
    torch.cuda.synchronize()
    return keys.cpu().numpy(), order.cpu().numpy(), starts.cpu().numpy()


def _markers(n, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    box = torch.tensor([[1.0], [2.0], [1.0]], dtype=torch.float64, device="cuda")
    low = torch.tensor([[0.0], [-1.0], [0.5]], dtype=torch.float64, device="cuda")
    positions = low + box * torch.rand((3, n), generator=g, dtype=torch.float64, device="cuda")
    values = torch.rand((1, n), generator=g, dtype=torch.float64, device="cuda") + 0.5
    values[0, ::7] = 0.0  # dead markers go last without their positions being read
    positions[:, ::7] = float("nan")
    return positions, values


def test_two_calls_in_a_row_match_the_sort_with_a_workspace():
    for n, seed, within in ((MAX_MARKERS, 1, 1), (300_001, 2, 0)):
        positions, values = _markers(n, seed)
        expected = _sort(positions, values, within, noalloc=False)
        got = _sort(positions, values, within, noalloc=True)
        for a, b in zip(got, expected):
            np.testing.assert_array_equal(a, b)
