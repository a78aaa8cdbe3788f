"""The store kept sorted across steps (mpf_resort_by_tile) equals the full sort, bit for bit.

A marker store is sorted once, its arrays permuted by the order, and then, step after
step, its markers move (by less than a cell, or anything at all) and it is re-sorted
against the keys of the previous sort. Every step's order, tile starts and sorted keys
must equal those of mpf_sort_by_tile on the same store (numpy.argsort(keys,
kind="stable") of the oracle's keys, bit for bit): with and without the cell inside
the tile in the key, dead markers (values zero) going to and leaving the sentinel tile,
markers crossing periodic seams, no marker moving, every marker moving, 1D to 3D.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import mpifield_b200 as mf
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = [
    # (ndim, grid, tile, kind, degree, within, shift in cells)
    (3, (40, 32, 48), (4, 4, 16), (1, 2), True, 0.4),
    (3, (40, 32, 48), (8, 8, 8), (1, 2), False, 0.4),
    (3, (24, 24, 24), (4, 4, 8), (0, 1), True, 3.0),
    (2, (64, 48), (8, 16), (2, 3), True, 0.3),
    (1, (300,), (16,), (2, 2), True, 0.6),
]


def _store(ndim, grid, n, rng):
    geom = tuple([0.0] * ndim + [1.0 / g for g in grid] + list(grid) + [1] * ndim)
    pos = rng.uniform(0.0, 1.0, (ndim, n))
    pos[:, : n // 5] = np.remainder(rng.normal(0.5, 0.05, (ndim, n // 5)), 1.0)  # a beam
    values = rng.uniform(0.5, 1.5, (1, n))
    values[0, ::11] = 0.0
    return geom, pos, values


def _full(kind_degree, pos, values, geom, tile, within):
    keys = O.tile_keys(["linear", "quadratic", "spline"][kind_degree[0]], kind_degree[1], pos, geom, tile,
                       values=values, within=within)
    order = O.sort_by_tile(keys)
    return keys, order


@pytest.mark.parametrize("case", range(len(CASES)))
def test_resorted_store_equals_the_full_sort(case):
    ndim, grid, tile, kd, within, shift = CASES[case]
    rng = np.random.default_rng(case)
    n = 300_001
    geom, pos, values = _store(ndim, grid, n, rng)
    cells = np.prod(tile) if within else 1
    p = torch.tensor(pos, device="cuda")
    v = torch.tensor(values, device="cuda")
    t = mf.resort_by_tile(p, kd, geom, tile, values=v, within=within)  # the first, full sort
    for step in range(4):
        # the store in its sorted order, then its markers move
        order = t.order.cpu().numpy()
        keys, expected = _full(kd, p.cpu().numpy(), v.cpu().numpy(), geom, tile, within)
        np.testing.assert_array_equal(order, expected)
        np.testing.assert_array_equal(t.sorted_keys.cpu().numpy().view(np.uint32), keys[expected])
        starts = np.searchsorted(keys[expected] // cells, np.arange(t.num_tiles + 2))
        np.testing.assert_array_equal(t.tile_start.cpu().numpy(), starts)
        p = mf.permute(p, t.order)
        v = mf.permute(v, t.order)
        h = torch.tensor([1.0 / g for g in grid], device="cuda", dtype=torch.float64)[:, None]
        move = (torch.rand(p.shape, device="cuda", dtype=torch.float64) * 2 - 1) * shift * h
        if step == 2:
            move.zero_()  # nobody moves
        p = torch.remainder(p + move, 1.0)
        if step == 1:  # some markers die, some come back to life
            v[0, ::7] = 0.0
            v[0, ::11] = 1.0
        t = mf.resort_by_tile(p, kd, geom, tile, values=v, within=within, previous=t)


def test_an_empty_store_and_a_wrong_previous():
    geom = (0.0, 0.0, 0.1, 0.1, 10, 10, 1, 1)
    empty = torch.zeros((2, 0), dtype=torch.float64, device="cuda")
    t = mf.resort_by_tile(empty, (1, 2), geom, (4, 4))
    assert t.order.numel() == 0 and int(t.tile_start[-1]) == 0
    p = torch.rand((2, 100), dtype=torch.float64, device="cuda")
    first = mf.resort_by_tile(p, (1, 2), geom, (4, 4))
    with pytest.raises(ValueError, match="previous"):
        mf.resort_by_tile(p[:, :50], (1, 2), geom, (4, 4), previous=first)
