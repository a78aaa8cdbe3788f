"""GPU parity of the node gather and scatter with the oracle (and the reference's fixtures).

FP64 results agree with the oracle within RTOL_F64 = 1e-12 of max |oracle| (the
atomic and summation order only); every kernel variant and launch path (direct global
memory, staged shared-memory boxes, boxes too small) is checked, on sorted and unsorted
markers, periodic seams, bounded folds, clamped knots, dense cells, dead markers,
strided rows and the FP32 variant.
"""

from __future__ import annotations

import itertools

import numpy as np
import pytest
import torch

import mpifield_b200 as mf
from mpifield_b200 import _lib
from mpifield_b200.kernels import gather, scatter
from oracle import oracle as O
from tests.helpers import KIND_NAMES, RTOL_F32, RTOL_F64, cases, geometry, load, node_case, random_case, rel_err

pytestmark = pytest.mark.gpu

NODES = load("node_kernels.npz")
DEV = "cuda"
# Variant 0 is the default: the gather through L1, the segment scatter (one component,
# at most 27 stencil points; direct: global atomics; small_box: boxes too small for most
# chunks). Variant 1: the gather with staged boxes. Variant 2: the scatter's
# warp-transposed run reduction (the default for the other shapes).
PATHS = {"staged": _lib.tuning_struct(_lib.PATH_STAGED),
         "direct": _lib.tuning_struct(_lib.PATH_DIRECT),
         "small_box": _lib.tuning_struct(_lib.PATH_STAGED, smem_bytes=4096),
         "boxed": _lib.tuning_struct(_lib.PATH_STAGED, variant=1),
         "boxed_direct": _lib.tuning_struct(_lib.PATH_DIRECT, variant=1),
         "boxed_small": _lib.tuning_struct(_lib.PATH_STAGED, smem_bytes=4096, variant=1),
         "transposed": _lib.tuning_struct(_lib.PATH_STAGED, variant=2),
         "transposed_small": _lib.tuning_struct(_lib.PATH_STAGED, smem_bytes=4096, variant=2)}
GATHER_PATHS = ("staged", "boxed", "boxed_direct", "boxed_small")
SCATTER_PATHS = ("staged", "direct", "small_box", "transposed", "transposed_small")


def cu(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


def run_gather(kind, degree, pos, field, geom, path="staged", dtype=torch.float64):
    result = torch.empty((field.shape[-1], pos.shape[1]), dtype=dtype, device=DEV)
    gather(KIND_NAMES[kind], degree, cu(pos, dtype), cu(field, dtype), result, geom, PATHS[path])
    return result.double().cpu().numpy()


def run_scatter(kind, degree, pos, values, shape, geom, path="staged", dtype=torch.float64):
    field = torch.zeros(shape, dtype=dtype, device=DEV)
    scatter(KIND_NAMES[kind], degree, cu(pos, dtype), cu(values, dtype), field, geom, PATHS[path])
    return field.double().cpu().numpy()


@pytest.mark.parametrize("path", ["staged", "direct", "boxed", "transposed"])
@pytest.mark.parametrize("tag", cases(NODES))
def test_golden_cases(tag, path):
    kind, degree = node_case(tag)
    geom = geometry(NODES[f"{tag}/geometry"])
    field = NODES[f"{tag}/field"]
    got = run_gather(kind, degree, NODES[f"{tag}/positions"], field, geom, path)
    assert rel_err(got, NODES[f"{tag}/gather"]) < RTOL_F64
    dep = run_scatter(kind, degree, NODES[f"{tag}/dead_positions"], NODES[f"{tag}/values"], field.shape, geom, path)
    assert rel_err(dep, NODES[f"{tag}/scatter"]) < RTOL_F64


KINDS = [("linear", 1), ("quadratic", 2), ("spline", 0), ("spline", 1), ("spline", 2), ("spline", 3)]


def _code_sets(ndim, kind, degree):
    sets = [(0,) * ndim, (1,) * ndim, tuple(i % 2 for i in range(ndim))]
    if kind == "spline" and degree >= 1:
        sets.append((2,) + (1,) * (ndim - 1))
    return sets


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("kind,degree", KINDS)
def test_random_cases_sorted_and_unsorted(kind, degree, ndim):
    rng = np.random.default_rng(hash((kind, degree, ndim)) % 2**32)
    for codes in _code_sets(ndim, kind, degree):
        for ncomp in (1, 3, 5):
            geom, pos, field, values = random_case(rng, ndim, codes, degree, n=3000, ncomp=ncomp,
                                                   shape=(23, 17, 13)[:ndim])
            values[:, ::13] = 0.0
            expected_g = O.gather(kind, degree, pos, field, geom)
            expected_s = O.scatter(kind, degree, pos, values, np.zeros_like(field), geom)
            # sorted by a coarse cell order: chunks then fit the shared-memory boxes
            keys = np.floor((pos - np.array(geom[:ndim])[:, None]) / np.array(geom[ndim:2 * ndim])[:, None] / 4)
            order = np.lexsort(keys[::-1])
            for p, v, eg in ((pos, values, expected_g), (pos[:, order], values[:, order], expected_g[:, order])):
                for path in GATHER_PATHS:
                    assert rel_err(run_gather(kind, degree, p, field, geom, path), eg) < RTOL_F64
                for path in SCATTER_PATHS:
                    got = run_scatter(kind, degree, p, v, field.shape, geom, path)
                    assert rel_err(got, expected_s) < RTOL_F64


@pytest.mark.parametrize("kind,degree", [("quadratic", 2), ("spline", 3), ("linear", 1)])
def test_large_sorted_3d_uses_the_boxes_and_agrees(kind, degree):
    rng = np.random.default_rng(3)
    shape = (40, 36, 32)
    geom = (0.0, 0.0, 0.0, 1 / 40, 1 / 36, 1 / 32, *shape, 1, 1, 1)
    n = 400_000
    pos = rng.uniform(0, 1, (3, n))
    pos[:, : n // 5] = np.mod(rng.normal(0.5, 0.05, (3, n // 5)), 1.0)
    field = rng.normal(size=(*shape, 3))
    values = rng.uniform(0.5, 1.5, (1, n))
    t = mf.sort_by_tile(cu(pos), (KIND_NAMES[kind], degree), geom, (8, 8, 8))
    order = t.order.cpu().numpy()
    ps, vs = pos[:, order], values[:, order]
    eg = O.gather(kind, degree, ps, field, geom)
    es = O.scatter(kind, degree, ps, vs, np.zeros((*shape, 1)), geom)
    for path in ("staged", "boxed"):
        assert rel_err(run_gather(kind, degree, ps, field, geom, path), eg) < RTOL_F64
    for path in ("staged", "transposed"):
        assert rel_err(run_scatter(kind, degree, ps, vs, (*shape, 1), geom, path), es) < RTOL_F64


@pytest.mark.parametrize("kind,degree,ndim", [("quadratic", 2, 3), ("linear", 1, 2), ("spline", 0, 3)])
def test_dense_cells_sum_runs_across_the_warp(kind, degree, ndim):
    # thousands of markers in a few cells, sorted: whole warps close runs of one anchor
    rng = np.random.default_rng(6)
    shape = (12, 10, 9)[:ndim]
    geom = (*[0.0] * ndim, *[1.0] * ndim, *shape, *[1] * ndim)
    n = 60_000
    centres = np.array([[3.2, 4.7, 5.1], [3.6, 4.2, 5.9], [9.5, 0.1, 8.9]])[:, :ndim]
    pick = np.sort(rng.integers(0, 3, n))
    pos = (centres[pick] + rng.uniform(-0.05, 0.05, (n, ndim))).T.copy()
    values = rng.uniform(0.5, 1.5, (1, n))
    values[:, ::7] = 0.0
    es = O.scatter(kind, degree, pos, values, np.zeros((*shape, 1)), geom)
    for path in ("staged", "small_box", "transposed"):
        assert rel_err(run_scatter(kind, degree, pos, values, (*shape, 1), geom, path), es) < RTOL_F64


def test_strided_rows_and_noncontiguous_outputs():
    rng = np.random.default_rng(4)
    geom, pos, field, values = random_case(rng, 3, (1, 0, 1), 2, n=1000, ncomp=2)
    storage = torch.zeros((3, 1500), dtype=torch.float64, device=DEV)
    storage[:, :1000] = cu(pos)
    vstore = torch.zeros((2, 1200), dtype=torch.float64, device=DEV)
    vstore[:, :1000] = cu(values)
    out_store = torch.zeros((2, 1100), dtype=torch.float64, device=DEV)
    mf.KERNELS["gather_quadratic_3d"](storage[:, :1000], cu(field), out_store[:, :1000], *geom)
    assert rel_err(out_store[:, :1000].cpu().numpy(), O.gather("quadratic", 2, pos, field, geom)) < RTOL_F64
    # a transposed (column-major) output is written through a copy
    out_t = torch.zeros((1000, 2), dtype=torch.float64, device=DEV).t()
    mf.KERNELS["gather_quadratic_3d"](storage[:, :1000], cu(field), out_t, *geom)
    assert rel_err(out_t.cpu().numpy(), O.gather("quadratic", 2, pos, field, geom)) < RTOL_F64
    dep = torch.zeros(field.shape, dtype=torch.float64, device=DEV)
    mf.KERNELS["scatter_quadratic_3d"](storage[:, :1000], vstore[:, :1000], dep, *geom)
    assert rel_err(dep.cpu().numpy(), O.scatter("quadratic", 2, pos, values, np.zeros_like(field), geom)) < RTOL_F64


def test_dead_markers_with_non_finite_positions_deposit_nothing():
    rng = np.random.default_rng(5)
    geom, pos, field, values = random_case(rng, 2, (0, 1), 3, n=2000, ncomp=2)
    values[:, ::3] = 0.0
    pos[:, ::3] = np.nan
    pos[0, 3::9] = np.inf
    values[:, 3::9] = 0.0
    expected = O.scatter("spline", 3, pos, values, np.zeros_like(field), geom)
    for path in ("direct", "staged"):
        got = run_scatter("spline", 3, pos, values, field.shape, geom, path)
        assert np.isfinite(got).all()
        assert rel_err(got, expected) < RTOL_F64


def test_markers_far_outside_and_non_finite_stay_in_bounds():
    """Any position indexes inside the arrays; finite results where the oracle's are."""
    geom = (0.0, 0.0, 0.1, 0.1, 10, 10, 0, 1)
    pos = np.array([[1e12, -1e12, np.nan, np.inf, -np.inf, 0.35, 1e300, -1e300],
                    [0.2, 0.3, 0.4, 0.5, 0.6, np.nan, 1e300, 5.0]])
    field = np.arange(200.0).reshape(10, 10, 2)
    for kind, degree in KINDS:
        for path in ("direct", "staged"):
            got = run_gather(kind, degree, pos, field, geom, path)
            assert got.shape == (2, 8)
            np.testing.assert_allclose(got[:, :2], O.gather(kind, degree, pos[:, :2], field, geom), rtol=1e-12)


def test_the_reference_known_answers_on_the_gpu():
    # test_weighting.py:121-141 through the Field API
    f = mf.Field(1, (0.0,), (1.0,), 11)
    dx = float(f.grid_spacing[0])
    f.scatter(torch.tensor([[5 * dx]]), 1.0, mf.QUADRATIC)
    f.scatter(torch.tensor([[2.5 * dx]]), 8.0, mf.QUADRATIC)
    np.testing.assert_allclose(f.local[:, 0].cpu().numpy(), [0, 0, 4, 4, 0.125, 0.75, 0.125, 0, 0, 0, 0],
                               atol=1e-15)
    f = mf.Field(1, (0.0,), (1.0,), 11)
    f.scatter(torch.tensor([[0.0]]), 1.0, mf.QUADRATIC)
    np.testing.assert_allclose(f.local[:3, 0].cpu().numpy(), [0.875, 0.125, 0.0])
    f = mf.Field(1, (0.0,), (1.0,), 11, periodic=(True,))
    f.scatter(torch.tensor([[0.0]]), 1.0, mf.QUADRATIC)
    np.testing.assert_allclose(f.local[[-1, 0, 1], 0].cpu().numpy(), [0.125, 0.75, 0.125])
    f = mf.Field(1, (0.0,), (1.0,), 11)
    f.scatter(torch.tensor([[1.2, -0.3]]), torch.tensor([1.0, 2.0]))
    data = f.local[:, 0].cpu().numpy()
    assert data[-1] == 1.0 and data[0] == 2.0 and data.sum() == 3.0
    f = mf.Field(1, (0.0,), (1.0,), 4, periodic=True)
    f.set_field_data(np.array([0.0, 1.0, 2.0, 3.0]))
    np.testing.assert_allclose(f.gather(torch.tensor([[0.875, 1.125]])).cpu().numpy(), [[1.5, 0.5]])


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("weighting", [mf.LINEAR, mf.QUADRATIC, mf.CUBIC], ids=lambda w: w.name)
def test_linear_fields_are_gathered_exactly_inside(ndim, weighting):
    # test_weighting.py:92-103
    f = mf.Field(ndim, (0.0,) * ndim, (1.0,) * ndim, (11, 9, 7)[:ndim])
    nodes = np.meshgrid(*(np.linspace(0.0, 1.0, n) for n in f.num_gridpoints), indexing="ij")
    f.set_field_data(2.0 + sum((d + 1) * x for d, x in enumerate(nodes)))
    points = np.random.default_rng(3).uniform(0.2, 0.8, (ndim, 300))
    got = f.gather(points, weighting).cpu().numpy()[0]
    np.testing.assert_allclose(got, 2.0 + sum((d + 1) * points[d] for d in range(ndim)), rtol=1e-12)


@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("ndim", [1, 2, 3])
def test_deposits_keep_all_the_charge(ndim, periodic):
    # test_weighting.py:106-118
    f = mf.Field(ndim, (0.0,) * ndim, (1.0,) * ndim, (11, 9, 7)[:ndim], num_components=2, periodic=(periodic,) * ndim)
    rng = np.random.default_rng(4)
    points = rng.uniform(-0.1, 1.1, (ndim, 500))
    points[:, :50] = rng.choice([0.0, 1.0], (ndim, 50))
    values = rng.normal(size=(2, 500))
    for w in (mf.LINEAR, mf.QUADRATIC, mf.CUBIC):
        f.set_field_data(0.0)
        f.scatter(points, values, w)
        np.testing.assert_allclose(f.local_with_halos.reshape(-1, 2).sum(0).cpu().numpy(), values.sum(1), rtol=1e-12)


@pytest.mark.parametrize("kind,degree", [k for k in KINDS if k != ("spline", 0)])
def test_the_float32_variant_error_is_bounded(kind, degree):
    """Degree 0 is left out: its weights jump at half-integers, where float32 rounding
    of a position may pick the other node."""
    rng = np.random.default_rng(6)
    geom, pos, field, values = random_case(rng, 3, (1, 1, 1), degree, n=20000, ncomp=3, spread=0.0,
                                           shape=(32, 32, 32))
    eg = O.gather(kind, degree, pos, field, geom)
    es = O.scatter(kind, degree, pos, values, np.zeros_like(field), geom)
    for path in ("direct", "staged"):
        assert rel_err(run_gather(kind, degree, pos, field, geom, path, torch.float32), eg) < RTOL_F32
        assert rel_err(run_scatter(kind, degree, pos, values, field.shape, geom, path, torch.float32), es) < RTOL_F32


def test_adjoint_identity():
    # test_catalog_and_pyccel.py:163-182: sum_i g(x_i) q_i = sum_n G_n rho_n
    rng = np.random.default_rng(8)
    for kind, degree in KINDS:
        geom, pos, field, values = random_case(rng, 3, (1, 0, 2) if kind == "spline" and degree else (1, 0, 1),
                                               degree, n=5000, ncomp=2)
        g = run_gather(kind, degree, pos, field, geom)
        rho = run_scatter(kind, degree, pos, values, field.shape, geom)
        np.testing.assert_allclose((g * values).sum(1), (field * rho).reshape(-1, 2).sum(0), rtol=1e-12)
