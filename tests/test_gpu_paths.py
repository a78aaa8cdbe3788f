"""GPU parity of the path deposits (WHITNEY, QUADRATIC_EDGES, CUBIC_EDGES) and edge gathers.

Against the reference's NumPy kernels (golden fixtures) and the oracle within 1e-12 of
max |oracle|, and discrete continuity G^T j = rho(end) - rho(start) with the node deposit
of the same degree, to roundoff (src/mpifield/tests/unit/test_edges.py:59-66,
test_spline_edges.py:67-87).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import mpifield_b200 as mf
from mpifield_b200 import _lib
from mpifield_b200.kernels import deposit_paths, gather_edges
from oracle import oracle as O
from tests.helpers import RTOL_F64, cases, geometry, load, rel_err

pytestmark = pytest.mark.gpu
PATHS = load("path_kernels.npz")
DEV = "cuda"


def cu(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


# one thread per path with global atomics (the default; variant 1 the launch of one CTA
# per SM), the tiled deposit (shared-memory edge boxes, path 2) and the same with boxes
# too small for most chunks
TUNINGS = {"direct": None, "tiled": _lib.tuning_struct(_lib.PATH_STAGED),
           "small_box": _lib.tuning_struct(_lib.PATH_STAGED, smem_bytes=2048, block=2),
           "direct_one_cta": _lib.tuning_struct(variant=1)}


def run_deposit(kind, degree, start, end, charges, shape, geom, dtype=torch.float64, tuning="direct"):
    edges = torch.zeros(shape, dtype=dtype, device=DEV)
    deposit_paths(kind, degree, cu(start, dtype), cu(end, dtype), cu(charges, dtype), edges, geom, TUNINGS[tuning])
    return edges.double().cpu().numpy()


@pytest.mark.parametrize("tag", cases(PATHS))
def test_golden_cases(tag):
    degree = int(tag[5])
    geom = geometry(PATHS[f"{tag}/geometry"])
    shape = PATHS[f"{tag}/spline"].shape
    args = (PATHS[f"{tag}/start"], PATHS[f"{tag}/end"], PATHS[f"{tag}/charges"])
    got = run_deposit(_lib.SPLINE, degree, *args, shape, geom)
    np.testing.assert_allclose(got, PATHS[f"{tag}/spline"], rtol=0, atol=1e-12 * max(1, np.abs(got).max()))
    field = torch.zeros(PATHS[f"{tag}/points"].shape, dtype=torch.float64, device=DEV)
    gather_edges(_lib.SPLINE, degree, cu(PATHS[f"{tag}/points"]), cu(PATHS[f"{tag}/edges"]), field, geom)
    assert rel_err(field.cpu().numpy(), PATHS[f"{tag}/edge_gather"]) < RTOL_F64
    if f"{tag}/whitney" in PATHS:
        got = run_deposit(_lib.LINEAR, 1, *args, shape, geom)
        np.testing.assert_allclose(got, PATHS[f"{tag}/whitney"], rtol=0, atol=1e-12 * max(1, np.abs(got).max()))
        gather_edges(_lib.LINEAR, 1, cu(PATHS[f"{tag}/points"]), cu(PATHS[f"{tag}/edges"]), field, geom)
        assert rel_err(field.cpu().numpy(), PATHS[f"{tag}/whitney_gather"]) < RTOL_F64


def _case(rng, ndim, codes, degree, n, reach):
    shape = (13, 11, 9)[:ndim]
    lower = rng.uniform(-1, 1, ndim)
    cell = rng.uniform(0.2, 0.6, ndim)
    upper = lower + cell * (np.array(shape) - 1)
    start = rng.uniform(lower - 2 * cell, upper + 2 * cell, (n, ndim)).T.copy()
    end = start + rng.normal(scale=reach * cell[:, None], size=start.shape)
    charges = rng.normal(size=n)
    ext = tuple(s + (degree - 1 if c == 2 else 0) for s, c in zip(shape, codes))
    return (*lower, *cell, *shape, *codes), start, end, charges, ext


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("degree", [1, 2, 3])
def test_random_paths_match_the_oracle_and_conserve_charge(ndim, degree):
    rng = np.random.default_rng(degree * 7 + ndim)
    for codes in ((0,) * ndim, (1,) * ndim, tuple(i % 2 for i in range(ndim)), (2,) + (1,) * (ndim - 1)):
        if 2 in codes and degree == 1:
            continue
        for reach in (0.5, 3.0, 9.0):
            geom, start, end, charges, ext = _case(rng, ndim, codes, degree, 4000, reach)
            charges[::17] = 0.0
            expected = O.deposit_spline(degree, start, end, charges, np.zeros((*ext, ndim)), geom)
            for tuning in TUNINGS:
                got = run_deposit(_lib.SPLINE, degree, start, end, charges, (*ext, ndim), geom, tuning=tuning)
                np.testing.assert_allclose(got, expected, rtol=0, atol=1e-12 * np.abs(expected).max())
            if degree == 1 and 2 not in codes:
                expected = O.deposit_whitney(start, end, charges, np.zeros((*ext, ndim)), geom)
                for tuning in TUNINGS:
                    got = run_deposit(_lib.LINEAR, 1, start, end, charges, (*ext, ndim), geom, tuning=tuning)
                    np.testing.assert_allclose(got, expected, rtol=0, atol=1e-12 * np.abs(expected).max())
            if 2 not in codes:
                kind = "linear" if degree == 1 else ("quadratic" if degree == 2 else "spline")
                before = O.scatter(kind, degree, start, charges[None], np.zeros((*ext, 1)), geom)
                after = O.scatter(kind, degree, end, charges[None], np.zeros((*ext, 1)), geom)
                div = O.divergence_block(got, tuple(c == 1 for c in codes))
                np.testing.assert_allclose(div, (after - before)[..., 0], rtol=0, atol=1e-11)


def test_the_edge_weightings_through_the_block_api():
    grid = mf.BlockGrid.from_geometry((0.0, 0.0), (1.0, 1.0), (4, 4), (False, False))
    current = torch.zeros((4, 4, 2), dtype=torch.float64, device=DEV)
    mf.WHITNEY.deposit_paths_block(torch.tensor([[0.5], [-1.0]]), torch.tensor([[2.5], [-1.0]]), [1.0], current, grid)
    np.testing.assert_allclose(current[:3, 0, 0].cpu().numpy(), [0.5, 1.0, 0.5])
    assert int(torch.count_nonzero(current)) == 3
    # degree 1 spline edges are WHITNEY (test_spline_edges.py:46-59)
    rng = np.random.default_rng(2)
    grid = mf.BlockGrid.from_geometry((0.0, -1.0, 2.0), (0.25, 0.5, 0.1), (9, 8, 7), (True, False, True))
    start = rng.uniform(-0.5, 2.5, (3, 2000))
    end = start + rng.normal(scale=0.4, size=start.shape)
    q = rng.normal(size=2000)
    a = torch.zeros((9, 8, 7, 3), dtype=torch.float64, device=DEV)
    b = torch.zeros_like(a)
    mf.WHITNEY.deposit_paths_block(start, end, q, a, grid)
    mf.splines(1, clamped=True).edges.deposit_paths_block(start, end, q, b, grid)
    np.testing.assert_allclose(a.cpu().numpy(), b.cpu().numpy(), rtol=0, atol=1e-12)
    with pytest.raises(ValueError, match="an edge field on this grid"):
        mf.WHITNEY.deposit_paths_block(start, end, q, torch.zeros((9, 8, 7, 2), dtype=torch.float64, device=DEV), grid)


def test_dead_and_non_finite_paths_deposit_nothing():
    start = np.array([[0.1, np.nan, 0.2], [0.3, 0.1, np.inf]])
    geom = (0.0, 0.0, 0.3, 0.3, 6, 5, 0, 1)
    for kind, degree in ((_lib.LINEAR, 1), (_lib.SPLINE, 1), (_lib.SPLINE, 2), (_lib.SPLINE, 3)):
        got = run_deposit(kind, degree, start, start + 0.4, np.array([0.0, 1.0, 2.0]), (6, 5, 2), geom)
        assert np.all(got == 0.0)


def test_very_long_and_huge_paths_end():
    """Bounded work per path: a path of 1e200 cells stops at the step limit, no hang."""
    geom = (0.0, 0.0, 0.0, 0.1, 0.1, 0.1, 8, 8, 8, 1, 1, 1)
    start = np.array([[0.1, 0.2], [0.1, 0.2], [0.1, 0.2]])
    end = np.array([[0.1 + 200.0, 1e200], [0.1, 0.3], [0.1, 0.2]])
    for kind, degree in ((_lib.LINEAR, 1), (_lib.SPLINE, 2)):
        got = run_deposit(kind, degree, start[:, :1], end[:, :1], np.ones(1), (8, 8, 8, 3), geom)
        expected = (O.deposit_whitney if degree == 1 else
                    (lambda *a: O.deposit_spline(2, *a)))(start[:, :1], end[:, :1], np.ones(1), np.zeros((8, 8, 8, 3)), geom)
        np.testing.assert_allclose(got, expected, rtol=0, atol=1e-10)
        run_deposit(kind, degree, start, end, np.ones(2), (8, 8, 8, 3), geom)
        torch.cuda.synchronize()


@pytest.mark.parametrize("degree", [1, 2, 3])
def test_full_size_continuity_128_cubed(degree):
    """The path-deposit configuration: 128^3 periodic, 2^22 paths (of 2^25), |displacement| < 0.9 cell."""
    n = 1 << 22
    g = torch.Generator(device=DEV).manual_seed(11)
    start = torch.rand((3, n), generator=g, device=DEV, dtype=torch.float64)
    end = start + (torch.rand((3, n), generator=g, device=DEV, dtype=torch.float64) * 1.8 - 0.9) / 128
    q = torch.rand(n, generator=g, device=DEV, dtype=torch.float64) + 0.5
    grid = mf.BlockGrid.from_geometry((0.0,) * 3, (1 / 128,) * 3, (128,) * 3, (True,) * 3)
    edges = torch.zeros((128, 128, 128, 3), dtype=torch.float64, device=DEV)
    ew = mf.splines(degree).edges
    nodes = mf.splines(degree).nodes
    # sorted by the start's cell tile: the tiled deposit keeps its chunks in shared memory
    order = mf.sort_by_tile(start, mf.LINEAR, grid.geometry, (8, 8, 8), within=True).order
    start, end, q = mf.permute(start, order), mf.permute(end, order), mf.permute(q, order)
    ew.deposit_paths_block(start, end, q, edges, grid)
    tiled = torch.zeros_like(edges)
    deposit_paths(_lib.LINEAR if degree == 1 else _lib.SPLINE, degree, start, end, q, tiled, grid.geometry,
                  TUNINGS["tiled"])
    assert float((edges - tiled).abs().max()) < 1e-12 * float(edges.abs().max())
    before = torch.zeros((128, 128, 128, 1), dtype=torch.float64, device=DEV)
    after = torch.zeros_like(before)
    nodes.scatter_block(start, q, before, grid)
    nodes.scatter_block(end, q, after, grid)
    div = ew.divergence_block(edges, grid)
    change = (after - before)[..., 0]
    assert float((div - change).abs().max()) < 1e-10 * max(1.0, float(change.abs().max()))


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("degree", [1, 2, 3])
def test_small_fields_through_private_copies_match_the_oracle(ndim, degree):
    """Edge fields of a few hundred entries with many paths: each CTA deposits into a
    private copy in shared memory (the default there) -- the same as the oracle and as the
    global-atomic kernel (variant 7), for every boundary code."""
    rng = np.random.default_rng(300 + 10 * ndim + degree)
    shape = {1: (24,), 2: (12, 10), 3: (7, 6, 5)}[ndim]
    for codes in ((1,) * ndim, (0,) * ndim, (2,) + (1,) * (ndim - 1)):
        if 2 in codes and degree == 1:
            continue
        lower = rng.uniform(-1, 1, ndim)
        cell = rng.uniform(0.2, 0.6, ndim)
        upper = lower + cell * (np.array(shape) - 1)
        n = 40_000
        start = rng.uniform(lower - cell, upper + cell, (n, ndim)).T.copy()
        end = start + rng.normal(scale=1.5 * cell[:, None], size=start.shape)
        charges = rng.normal(size=n)
        charges[::13] = 0.0
        geom = (*lower, *cell, *shape, *codes)
        ext = tuple(s + (degree - 1 if c == 2 else 0) for s, c in zip(shape, codes))
        expected = O.deposit_spline(degree, start, end, charges, np.zeros((*ext, ndim)), geom)
        got = run_deposit(_lib.SPLINE, degree, start, end, charges, (*ext, ndim), geom)
        np.testing.assert_allclose(got, expected, rtol=0, atol=1e-12 * np.abs(expected).max())
        edges = torch.zeros((*ext, ndim), dtype=torch.float64, device=DEV)
        deposit_paths(_lib.SPLINE, degree, cu(start), cu(end), cu(charges), edges, geom, _lib.tuning_struct(variant=7))
        np.testing.assert_allclose(edges.cpu().numpy(), expected, rtol=0, atol=1e-12 * np.abs(expected).max())
        if degree == 1 and 2 not in codes:
            exp_w = O.deposit_whitney(start, end, charges, np.zeros((*ext, ndim)), geom)
            got = run_deposit(_lib.LINEAR, 1, start, end, charges, (*ext, ndim), geom)
            np.testing.assert_allclose(got, exp_w, rtol=0, atol=1e-12 * np.abs(exp_w).max())


@pytest.mark.parametrize("degree", [1, 2, 3])
def test_float32_deposits_stay_within_their_bound(degree):
    """The float32 build of the deposit (the direct kernel on a large field, the private
    copies on a small one) against the float64 deposit of the float32-rounded paths."""
    rng = np.random.default_rng(500 + degree)
    for shape, n in (((40, 36, 32), 200_000), ((6, 5, 4), 60_000)):
        geom = (0.0, 0.0, 0.0, *(1.0 / s for s in shape), *shape, 1, 1, 1)
        start = rng.uniform(0, 1, (3, n)).astype(np.float32).astype(np.float64)
        step = rng.uniform(-0.9, 0.9, (3, n)) / np.array(shape)[:, None]
        end = (start + step).astype(np.float32).astype(np.float64)
        charges = rng.uniform(0.5, 1.5, n).astype(np.float32).astype(np.float64)
        ref = run_deposit(_lib.SPLINE, degree, start, end, charges, (*shape, 3), geom)
        got = run_deposit(_lib.SPLINE, degree, start, end, charges, (*shape, 3), geom, dtype=torch.float32)
        assert np.abs(got - ref).max() <= 2e-4 * np.abs(ref).max(), degree
