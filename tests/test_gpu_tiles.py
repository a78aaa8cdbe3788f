"""GPU parity of the tile scatter and gather (mpf_scatter_tiles, mpf_gather_tiles) with the oracle.

Markers sorted by cell tile (mpf_sort_by_tile) and permuted into rank order are
scattered with the sort's tile starts; FP64 results agree with the oracle's scatter of
the same markers within RTOL_F64 of max |oracle| (atomic order only). Covered: every
weighting of at most 27 stencil points in 1D-3D on periodic grids, tile shapes from
one node to boxes too large for shared memory (the launch then takes the segment
scatter), tiles sorted with and without the cell inside the tile, dead markers in the
sentinel tile, dense cells split across CTAs, a store whose tile starts do not belong
to its positions (every marker outside its rank's tile adds to global memory), bounded
and clamped axes (the segment scatter), several components, FP32, and at 2^24 markers
the size-independent property: the tile scatter equals mpf_scatter on the same store. The
tile gather equals mpf_gather bit for bit (the same sums in the same order) on the same
shapes, tiles and stores, and the oracle within RTOL_F64.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import mpifield_b200 as mf
from mpifield_b200 import _lib
from mpifield_b200.kernels import gather, scatter
from oracle import oracle as O
from tests.helpers import KIND_NAMES, RTOL_F32, RTOL_F64, rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _store(rng, shape, codes, n, kind, degree, tile, within=True, dead=0.0, ncomp=1, dtype=torch.float64,
           positions=None):
    ndim = len(shape)
    lower = rng.uniform(-1.0, 1.0, ndim)
    cell = rng.uniform(0.1, 0.6, ndim)
    geom = (*lower, *cell, *shape, *codes)
    if positions is None:
        upper = lower + cell * np.array(shape)
        positions = rng.uniform(lower - 0.3 * cell, upper + 0.3 * cell, (n, ndim)).T.copy()
    values = rng.uniform(0.5, 1.5, (ncomp, positions.shape[1]))
    if dead:
        values[:, rng.uniform(size=positions.shape[1]) < dead] = 0.0
    pos = torch.tensor(positions, dtype=dtype, device=DEV)
    val = torch.tensor(values, dtype=dtype, device=DEV)
    order = mf.sort_by_tile(pos, (KIND_NAMES[kind], degree), geom, tile, values=val, within=within)
    ps = mf.permute(pos, order.order).contiguous()
    vs = mf.permute(val, order.order).contiguous()
    ext = tuple(s + (degree - 1 if c == 2 else 0) for s, c in zip(shape, codes))
    return geom, ps, vs, order, ext


def _scatter(kind, degree, ps, vs, ext, geom, order=None, tuning=None):
    field = torch.zeros((*ext, vs.shape[0]), dtype=ps.dtype, device=DEV)
    scatter(KIND_NAMES[kind], degree, ps, vs, field, geom, tuning, order=order)
    return field


def _oracle(kind, degree, ps, vs, ext, geom):
    pos, val = ps.double().cpu().numpy(), vs.double().cpu().numpy()
    return O.scatter(kind, degree, pos, val, np.zeros((*ext, val.shape[0])), geom)


KINDS = [("linear", 1), ("quadratic", 2), ("spline", 0), ("spline", 1), ("spline", 2), ("spline", 3)]


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("kind,degree", KINDS, ids=[f"{k}{d}" for k, d in KINDS])
def test_periodic_kinds_equal_the_oracle(ndim, kind, degree):
    if ndim == 3 and degree == 3:
        pytest.skip("64 stencil points: the transposed scatter, covered by the node tests")
    rng = np.random.default_rng(10 * ndim + degree)
    shape = (40, 24, 18)[:ndim]
    tile = (8, 6, 5)[:ndim]
    geom, ps, vs, order, ext = _store(rng, shape, (1,) * ndim, 20000, kind, degree, tile)
    got = _scatter(kind, degree, ps, vs, ext, geom, order).cpu().numpy()
    assert rel_err(got, _oracle(kind, degree, ps, vs, ext, geom)) < RTOL_F64
    assert _lib.device_errors() == 0


@pytest.mark.parametrize("tile", [(1, 1, 1), (2, 3, 4), (8, 8, 8), (8, 8, 16), (16, 16, 8), (24, 20, 18),
                                  (64, 64, 64)],
                         ids=lambda t: "x".join(map(str, t)))
@pytest.mark.parametrize("within", [True, False], ids=["cells", "tiles"])
def test_tile_shapes(tile, within):
    # 24 x 20 x 18 covers the grid in one tile; 64^3 does not fit shared memory (segment scatter)
    rng = np.random.default_rng(sum(tile) + within)
    geom, ps, vs, order, ext = _store(rng, (24, 20, 18), (1, 1, 1), 60000, "quadratic", 2, tile, within)
    got = _scatter("quadratic", 2, ps, vs, ext, geom, order).cpu().numpy()
    assert rel_err(got, _oracle("quadratic", 2, ps, vs, ext, geom)) < RTOL_F64


@pytest.mark.parametrize("kind", ["quadratic", "spline"])
@pytest.mark.parametrize("tile", [(8, 8, 8), (8, 8, 16), (4, 4, 64)], ids=lambda t: "x".join(map(str, t)))
def test_compile_time_tile_shapes(kind, tile):
    # the 3D degree-2 kernels with the tile shape as constants: uniform cells, a beam of
    # dense cells, dead markers, rows of the last axis that end inside a thread's markers,
    # empty cells inside a row (runs that end two cells apart)
    rng = np.random.default_rng(sum(tile) + len(kind))
    shape, cell, lower = (48, 40, 64), np.array([0.3, 0.2, 0.25]), np.array([-0.1, 0.2, -0.3])
    span = cell * np.array(shape)
    uniform = rng.uniform(0.0, 1.0, (150000, 3)) * span
    beam = rng.normal(0.5, 0.02, (50000, 3)) * span
    positions = (np.concatenate([uniform, beam]) + lower).T.copy()
    values = rng.uniform(0.5, 1.5, (1, positions.shape[1]))
    values[:, rng.uniform(size=positions.shape[1]) < 0.05] = 0.0
    geom = (*lower, *cell, *shape, 1, 1, 1)
    pos, val = torch.tensor(positions, device=DEV), torch.tensor(values, device=DEV)
    order = mf.sort_by_tile(pos, (KIND_NAMES[kind], 2), geom, tile, values=val, within=True)
    ps, vs = mf.permute(pos, order.order).contiguous(), mf.permute(val, order.order).contiguous()
    got = _scatter(kind, 2, ps, vs, shape, geom, order).cpu().numpy()
    assert rel_err(got, _oracle(kind, 2, ps, vs, shape, geom)) < RTOL_F64


@pytest.mark.parametrize("shape", [(6, 5, 4), (12, 10, 8)], ids=["box_wider_than_grid", "one_tile"])
def test_one_tile_covers_the_grid(shape):
    # the box (tile + 2 nodes per axis) wraps onto itself: its nodes alias on the grid
    rng = np.random.default_rng(sum(shape))
    geom, ps, vs, order, ext = _store(rng, shape, (1, 1, 1), 20000, "quadratic", 2, shape)
    got = _scatter("quadratic", 2, ps, vs, ext, geom, order).cpu().numpy()
    assert rel_err(got, _oracle("quadratic", 2, ps, vs, ext, geom)) < RTOL_F64


def test_dead_markers_sit_in_the_sentinel_tile():
    rng = np.random.default_rng(3)
    geom, ps, vs, order, ext = _store(rng, (32, 32, 32), (1, 1, 1), 50000, "quadratic", 2, (8, 8, 8), dead=0.3)
    starts = order.tile_start.cpu().numpy()
    assert starts[order.num_tiles] < starts[order.num_tiles + 1]  # dead markers exist
    got = _scatter("quadratic", 2, ps, vs, ext, geom, order).cpu().numpy()
    assert rel_err(got, _oracle("quadratic", 2, ps, vs, ext, geom)) < RTOL_F64


def test_dense_cells_split_across_ctas():
    # a beam: 300k markers in a few cells of one tile (the tile's ranks cut into many
    # CTA shares), plus a thin uniform background
    rng = np.random.default_rng(4)
    beam = rng.normal(0.0, 0.01, (3, 300000)) + np.array([[0.5], [0.45], [0.4]])
    background = rng.uniform(0.0, 1.0, (3, 5000))
    positions = np.concatenate([beam, background], axis=1)
    rng2 = np.random.default_rng(5)
    geom = (0.0, 0.0, 0.0, 1 / 32, 1 / 32, 1 / 32, 32, 32, 32, 1, 1, 1)
    pos = torch.tensor(positions, device=DEV)
    val = torch.tensor(rng2.uniform(0.5, 1.5, (1, positions.shape[1])), device=DEV)
    order = mf.sort_by_tile(pos, mf.QUADRATIC, geom, (8, 8, 8), within=True)
    ps, vs = mf.permute(pos, order.order).contiguous(), mf.permute(val, order.order).contiguous()
    got = _scatter("quadratic", 2, ps, vs, (32, 32, 32), geom, order).cpu().numpy()
    assert rel_err(got, _oracle("quadratic", 2, ps, vs, (32, 32, 32), geom)) < RTOL_F64


def test_tile_starts_of_another_store_still_give_the_scatter():
    # tile starts from one store, positions of another (random order): markers outside
    # their rank's tile go to global memory, the result is unchanged
    rng = np.random.default_rng(6)
    geom, ps, vs, order, ext = _store(rng, (30, 26, 22), (1, 1, 1), 40000, "quadratic", 2, (8, 8, 8))
    perm = torch.randperm(ps.shape[1], generator=torch.Generator().manual_seed(0)).to(DEV)
    ps2, vs2 = ps[:, perm].contiguous(), vs[:, perm].contiguous()
    got = _scatter("quadratic", 2, ps2, vs2, ext, geom, order).cpu().numpy()
    assert rel_err(got, _oracle("quadratic", 2, ps2, vs2, ext, geom)) < RTOL_F64


@pytest.mark.parametrize("codes", [(0, 0, 0), (1, 0, 1), (2, 1, 1)], ids=["bounded", "mixed", "clamped"])
def test_other_boundaries_take_the_segment_scatter(codes):
    rng = np.random.default_rng(7)
    geom, ps, vs, order, ext = _store(rng, (20, 18, 16), codes, 30000, "spline", 2, (8, 8, 8))
    got = _scatter("spline", 2, ps, vs, ext, geom, order).cpu().numpy()
    assert rel_err(got, _oracle("spline", 2, ps, vs, ext, geom)) < RTOL_F64


def test_several_components_and_small_stores():
    rng = np.random.default_rng(8)
    geom, ps, vs, order, ext = _store(rng, (16, 16, 16), (1, 1, 1), 3000, "quadratic", 2, (4, 4, 4), ncomp=3)
    got = _scatter("quadratic", 2, ps, vs, ext, geom, order).cpu().numpy()
    assert rel_err(got, _oracle("quadratic", 2, ps, vs, ext, geom)) < RTOL_F64
    for n in (1, 37, 255, 257):
        geom, ps, vs, order, ext = _store(rng, (16, 16, 16), (1, 1, 1), n, "quadratic", 2, (8, 8, 8))
        got = _scatter("quadratic", 2, ps, vs, ext, geom, order).cpu().numpy()
        assert rel_err(got, _oracle("quadratic", 2, ps, vs, ext, geom)) < RTOL_F64


def test_variant_one_ignores_the_tiles():
    rng = np.random.default_rng(9)
    geom, ps, vs, order, ext = _store(rng, (24, 24, 24), (1, 1, 1), 40000, "quadratic", 2, (8, 8, 8))
    tiles = _scatter("quadratic", 2, ps, vs, ext, geom, order)
    segments = _scatter("quadratic", 2, ps, vs, ext, geom, order, _lib.tuning_struct(_lib.PATH_STAGED, variant=1))
    assert rel_err(tiles.cpu().numpy(), segments.cpu().numpy()) < RTOL_F64


def test_float32_is_within_the_stated_bound():
    rng = np.random.default_rng(11)
    geom, ps, vs, order, ext = _store(rng, (32, 32, 32), (1, 1, 1), 60000, "quadratic", 2, (8, 8, 8),
                                      dtype=torch.float32)
    got = _scatter("quadratic", 2, ps, vs, ext, geom, order).double().cpu().numpy()
    assert rel_err(got, _oracle("quadratic", 2, ps, vs, ext, geom)) < RTOL_F32


def test_the_tile_scatter_equals_the_scatter_at_2_24_markers():
    n, grid = 1 << 24, 160
    g = torch.Generator(device=DEV).manual_seed(12)
    geom = (0.0, 0.0, 0.0, 1 / grid, 1 / grid, 1 / grid, grid, grid, grid, 1, 1, 1)
    pos = torch.rand((3, n), generator=g, dtype=torch.float64, device=DEV)
    val = torch.rand((1, n), generator=g, dtype=torch.float64, device=DEV) + 0.5
    order = mf.sort_by_tile(pos, mf.QUADRATIC, geom, (8, 8, 8), within=True)
    ps, vs = mf.permute(pos, order.order).contiguous(), mf.permute(val, order.order).contiguous()
    del pos, val
    ext = (grid, grid, grid)
    tiles = _scatter("quadratic", 2, ps, vs, ext, geom, order)
    plain = _scatter("quadratic", 2, ps, vs, ext, geom)
    assert (tiles - plain).abs().max().item() <= RTOL_F64 * plain.abs().max().item()
    # mass: every marker's weights sum to one
    assert abs(tiles.sum().item() - vs.sum().item()) <= 1e-10 * vs.sum().item()
    assert _lib.device_errors() == 0


def test_bad_tile_orders_are_refused():
    rng = np.random.default_rng(13)
    geom, ps, vs, order, ext = _store(rng, (16, 16, 16), (1, 1, 1), 1000, "quadratic", 2, (8, 8, 8))
    field = torch.zeros((*ext, 1), dtype=torch.float64, device=DEV)
    bad = mf.TileOrder(order.keys, order.order, order.tile_start[:-1], order.num_tiles, order.tile)
    with pytest.raises(ValueError):
        scatter(KIND_NAMES["quadratic"], 2, ps, vs, field, geom, order=bad)
    bad = mf.TileOrder(order.keys, order.order, order.tile_start, order.num_tiles, (8, 8))
    with pytest.raises(ValueError):
        scatter(KIND_NAMES["quadratic"], 2, ps, vs, field, geom, order=bad)


# ------------------------------------------------------------------ the tile gather --

def _gather_pair(kind, degree, ps, field, geom, order):
    ncomp = field.shape[-1]
    tiles = torch.empty((ncomp, ps.shape[1]), dtype=ps.dtype, device=DEV)
    plain = torch.empty_like(tiles)
    gather(KIND_NAMES[kind], degree, ps, field, tiles, geom, order=order)
    gather(KIND_NAMES[kind], degree, ps, field, plain, geom)
    return tiles, plain


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("kind,degree", KINDS, ids=[f"{k}{d}" for k, d in KINDS])
def test_tile_gather_equals_the_gather_bit_for_bit(ndim, kind, degree):
    rng = np.random.default_rng(100 + 10 * ndim + degree)
    shape = (40, 24, 18)[:ndim]
    tile = (8, 6, 5)[:ndim]
    geom, ps, _, order, ext = _store(rng, shape, (1,) * ndim, 20000, kind, degree, tile)
    field = torch.tensor(rng.normal(size=ext + (3,)), device=DEV)
    tiles, plain = _gather_pair(kind, degree, ps, field, geom, order)
    assert torch.equal(tiles, plain)
    oracle = O.gather(kind, degree, ps.cpu().numpy(), field.cpu().numpy(), geom)
    assert rel_err(tiles.cpu().numpy(), oracle) < RTOL_F64


@pytest.mark.parametrize("tile", [(1, 1, 1), (8, 8, 8), (8, 8, 16), (4, 4, 64), (16, 16, 8), (64, 64, 64)],
                         ids=lambda t: "x".join(map(str, t)))
@pytest.mark.parametrize("ncomp", [1, 2, 3, 5])
def test_tile_gather_shapes_and_components(tile, ncomp):
    # 64^3 tiles do not fit shared memory and 5 components take the L1 gather
    rng = np.random.default_rng(sum(tile) + ncomp)
    geom, ps, _, order, ext = _store(rng, (24, 20, 70), (1, 1, 1), 60000, "quadratic", 2, tile)
    field = torch.tensor(rng.normal(size=ext + (ncomp,)), device=DEV)
    tiles, plain = _gather_pair("quadratic", 2, ps, field, geom, order)
    assert torch.equal(tiles, plain)


def test_tile_gather_with_the_tile_starts_of_another_store():
    rng = np.random.default_rng(21)
    geom, ps, _, order, ext = _store(rng, (30, 26, 22), (1, 1, 1), 40000, "quadratic", 2, (8, 8, 8))
    perm = torch.randperm(ps.shape[1], generator=torch.Generator().manual_seed(1)).to(DEV)
    ps2 = ps[:, perm].contiguous()
    field = torch.tensor(rng.normal(size=ext + (3,)), device=DEV)
    tiles, plain = _gather_pair("quadratic", 2, ps2, field, geom, order)
    assert torch.equal(tiles, plain)


@pytest.mark.parametrize("codes", [(0, 0, 0), (2, 1, 1)], ids=["bounded", "clamped"])
def test_tile_gather_other_boundaries(codes):
    rng = np.random.default_rng(22)
    geom, ps, _, order, ext = _store(rng, (20, 18, 16), codes, 30000, "spline", 2, (8, 8, 8))
    field = torch.tensor(rng.normal(size=ext + (3,)), device=DEV)
    tiles, plain = _gather_pair("spline", 2, ps, field, geom, order)
    assert torch.equal(tiles, plain)


def test_tile_gather_float32_and_a_beam():
    rng = np.random.default_rng(23)
    shape = (48, 40, 64)
    beam = rng.normal(0.5, 0.02, (3, 80000)) * np.array(shape)[:, None]
    geom = (0.0, 0.0, 0.0, 1.0, 1.0, 1.0, *shape, 1, 1, 1)
    for dtype in (torch.float64, torch.float32):
        pos = torch.tensor(np.concatenate([beam, rng.uniform(0, 1, (3, 20000)) * np.array(shape)[:, None]], 1),
                           dtype=dtype, device=DEV)
        order = mf.sort_by_tile(pos, mf.QUADRATIC, geom, (4, 4, 64), within=True)
        ps = mf.permute(pos, order.order).contiguous()
        field = torch.tensor(rng.normal(size=shape + (3,)), dtype=dtype, device=DEV)
        tiles, plain = _gather_pair("quadratic", 2, ps, field, geom, order)
        assert torch.equal(tiles, plain)
    assert _lib.device_errors() == 0


def test_the_tile_gather_equals_the_gather_at_2_24_markers():
    n, grid = 1 << 24, 160
    g = torch.Generator(device=DEV).manual_seed(24)
    geom = (0.0, 0.0, 0.0, 1 / grid, 1 / grid, 1 / grid, grid, grid, grid, 1, 1, 1)
    pos = torch.rand((3, n), generator=g, dtype=torch.float64, device=DEV)
    order = mf.sort_by_tile(pos, mf.QUADRATIC, geom, (4, 4, 64), within=True)
    ps = mf.permute(pos, order.order).contiguous()
    del pos
    field = torch.randn((grid, grid, grid, 3), generator=g, dtype=torch.float64, device=DEV)
    tiles, plain = _gather_pair("quadratic", 2, ps, field, geom, order)
    assert torch.equal(tiles, plain)
