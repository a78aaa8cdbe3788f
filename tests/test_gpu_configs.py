"""Oracle parity at the exact configurations the bench times, through the bench's own code.

- 3D QUADRATIC gather + scatter: 256^3 periodic, a 3-component Fourier field, N = 2^26
  markers (80% uniform, 20% beam), the store sorted by 4 x 4 x 64 cell tiles, the tile
  gather and the tile scatter with the store's tile starts (`bench.Step`). The sort is
  checked bit for bit against the oracle's keys and numpy's stable argsort, E on a random
  subset of 2^20 markers (the gather is independent per marker) and the density of all
  2^26 markers against the oracle, within 1e-12 of max; the float32 variant within its
  stated bound.
- The plain 2D step: 101 x 51 bounded, LINEAR, N = 100,000 from default_rng(0), E from
  numpy.gradient (`bench.plain_2d_case`).
- The path deposit: 128^3 periodic, 2^25 paths (`bench.path_case`); WHITNEY,
  QUADRATIC_EDGES and CUBIC_EDGES on a random subset of 2^20 paths, in the bench's random
  and tile-sorted orders, against the oracle.

The tolerance is the reference's own for its emulated CUDA kernels against NumPy
(src/mpifield/tests/kernels/test_cuda_emulated.py:160): 1e-12.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import bench
import mpifield_b200 as mf
from oracle import oracle as O
from tests.helpers import RTOL_F32, RTOL_F64, rel_err

pytestmark = pytest.mark.gpu

N_C2 = 1 << 26
SUBSET = 1 << 20


@pytest.fixture(scope="module")
def c2_store():
    device = torch.device("cuda", 0)
    step = bench.Step(N_C2, device, torch.float64)
    pos, w = bench.make_markers(N_C2, device, torch.float64, seed=1)
    tiles, ps, ws = step.sort(pos, w)
    step.gather_scatter(ps, ws)
    torch.cuda.synchronize()
    yield step, pos, tiles, ps, ws
    del step, pos, tiles, ps, ws
    torch.cuda.empty_cache()


def _subset(n, count, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.randperm(n, generator=g, device="cuda")[:count]


def test_c2_sort_is_the_stable_order_of_the_oracle_keys(c2_store):
    _, pos, tiles, _, _ = c2_store
    keys = O.tile_keys("quadratic", 2, pos.cpu().numpy(), bench.geometry(), bench.TILE, within=True)
    order = tiles.order.cpu().numpy()
    np.testing.assert_array_equal(order, O.sort_by_tile(keys))
    # tile starts: the first rank of every tile (the sentinel tile last)
    cells = int(np.prod(bench.TILE))
    sorted_tiles = keys[order] // cells
    starts = tiles.tile_start.cpu().numpy()
    expected = np.searchsorted(sorted_tiles, np.arange(starts.size))
    np.testing.assert_array_equal(starts, expected)


def test_c2_gather_matches_the_oracle(c2_store):
    step, _, _, ps, _ = c2_store
    idx = _subset(N_C2, SUBSET, 3)
    got = step.E[:, idx].cpu().numpy()
    expected = O.gather("quadratic", 2, ps[:, idx].cpu().numpy(), step.field.cpu().numpy(), bench.geometry())
    assert rel_err(got, expected) <= RTOL_F64


def test_c2_scatter_matches_the_oracle_on_every_marker(c2_store):
    step, _, _, ps, ws = c2_store
    expected = np.zeros((bench.GRID,) * 3 + (1,))
    O.scatter("quadratic", 2, ps.cpu().numpy(), ws.cpu().numpy(), expected, bench.geometry())
    got = step.density.cpu().numpy()
    assert rel_err(got, expected) <= RTOL_F64
    # the deposit keeps the total charge
    assert abs(got.sum() - float(ws.sum())) <= 1e-9 * float(ws.sum())


def test_c2_float32_variant_within_its_stated_bound(c2_store):
    step, _, _, ps, ws = c2_store
    p32, w32, f32 = ps.float(), ws.float(), step.field.float()
    E32 = torch.empty((3, N_C2), dtype=torch.float32, device=ps.device)
    D32 = torch.zeros(step.density.shape, dtype=torch.float32, device=ps.device)
    mf.kernels.gather(step.lib.QUADRATIC, 2, p32, f32, E32, step.geom, order=step.order)
    mf.kernels.scatter(step.lib.QUADRATIC, 2, p32, w32, D32, step.geom, order=step.order)
    idx = _subset(N_C2, SUBSET, 4)
    expected_e = O.gather("quadratic", 2, ps[:, idx].cpu().numpy(), step.field.cpu().numpy(), bench.geometry())
    assert rel_err(E32[:, idx].double().cpu().numpy(), expected_e) <= RTOL_F32
    assert rel_err(D32.double().cpu().numpy(), step.density.cpu().numpy()) <= RTOL_F32


def test_c1_plain_2d_matches_the_oracle():
    geom, pos, E = bench.plain_2d_case()
    n = pos.shape[1]
    p = torch.tensor(pos, device="cuda")
    field = torch.tensor(E, device="cuda")
    ones = torch.ones((1, n), dtype=torch.float64, device="cuda")
    rho = torch.zeros((101, 51, 1), dtype=torch.float64, device="cuda")
    out = torch.empty((2, n), dtype=torch.float64, device="cuda")
    mf.KERNELS["scatter_linear_2d"](p, ones, rho, *geom)
    mf.KERNELS["gather_linear_2d"](p, field, out, *geom)
    expected_rho = O.scatter("linear", 1, pos, np.ones((1, n)), np.zeros((101, 51, 1)), geom)
    expected_e = O.gather("linear", 1, pos, E, geom)
    assert rel_err(rho.cpu().numpy(), expected_rho) <= RTOL_F64
    assert rel_err(out.cpu().numpy(), expected_e) <= RTOL_F64
    assert abs(float(rho.sum()) - n) <= 1e-9 * n


@pytest.fixture(scope="module")
def c3_paths():
    start, end, q, grid = bench.path_case("cuda", 1 << 25)
    idx = _subset(start.shape[1], SUBSET, 5)
    # the bench's sorted order: by the start's cell tile
    order = mf.sort_by_tile(start, mf.LINEAR, grid.geometry, bench.TILE, within=True).order
    sorted_pick = torch.zeros(start.shape[1], dtype=torch.bool, device="cuda")
    sorted_pick[idx] = True
    keep = sorted_pick[order.long()]
    s_idx = order.long()[keep]
    yield start, end, q, grid, idx, s_idx
    del start, end, q
    torch.cuda.empty_cache()


@pytest.mark.parametrize("degree", [1, 2, 3])
def test_c3_path_deposit_matches_the_oracle(c3_paths, degree):
    start, end, q, grid, idx, s_idx = c3_paths
    ew = mf.splines(degree).edges
    expected = np.zeros((128, 128, 128, 3))
    s, e, c = (t[:, idx].cpu().numpy() for t in (start, end, q))
    if degree == 1:
        O.deposit_whitney(s, e, c, expected, grid.geometry)
    else:
        O.deposit_spline(degree, s, e, c, expected, grid.geometry)
    for pick in (idx, s_idx):  # random order, then the tile-sorted order of the bench
        edges = torch.zeros((128, 128, 128, 3), dtype=torch.float64, device="cuda")
        ew.deposit_paths_block(start[:, pick], end[:, pick], q[0, pick], edges, grid)
        assert rel_err(edges.cpu().numpy(), expected) <= RTOL_F64
