"""The oracle, pinned before it is trusted (CPU only).

- against the reference's own NumPy kernels: the golden fixtures of tests/golden
  (generated by tests/golden/make_golden.py from src/mpifield/kernels/*/..._numpy.py);
- against the reference's own CUDA kernel bodies compiled as C++ (oracle/_ref), bit for
  bit where the arithmetic is the same;
- against the known answers and invariants of the reference's tests
  (src/mpifield/tests/unit/test_weighting.py, test_splines.py, test_edges.py,
  test_spline_edges.py, test_field.py).
"""

from __future__ import annotations

import itertools
import os
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import cases, geometry, load, node_case, rel_err

NODES = load("node_kernels.npz")
PATHS = load("path_kernels.npz")
FORMS = load("form_kernels.npz")


@pytest.mark.parametrize("tag", cases(NODES))
def test_node_oracle_matches_the_reference_numpy_kernels(tag):
    kind, degree = node_case(tag)
    geom = geometry(NODES[f"{tag}/geometry"])
    result = O.gather(kind, degree, NODES[f"{tag}/positions"], NODES[f"{tag}/field"], geom)
    assert rel_err(result, NODES[f"{tag}/gather"]) < 1e-14
    deposit = np.zeros_like(NODES[f"{tag}/field"])
    O.scatter(kind, degree, NODES[f"{tag}/dead_positions"], NODES[f"{tag}/values"], deposit, geom)
    assert rel_err(deposit, NODES[f"{tag}/scatter"]) < 1e-14


@pytest.mark.parametrize("tag", cases(PATHS))
def test_path_oracle_matches_the_reference_numpy_kernels(tag):
    degree = int(tag[5])
    geom = geometry(PATHS[f"{tag}/geometry"])
    current = np.zeros_like(PATHS[f"{tag}/spline"])
    O.deposit_spline(degree, PATHS[f"{tag}/start"], PATHS[f"{tag}/end"], PATHS[f"{tag}/charges"], current, geom)
    np.testing.assert_allclose(current, PATHS[f"{tag}/spline"], rtol=0, atol=1e-13)
    field = O.gather_edges(degree, PATHS[f"{tag}/points"], PATHS[f"{tag}/edges"], geom)
    np.testing.assert_allclose(field, PATHS[f"{tag}/edge_gather"], rtol=0, atol=1e-12)
    if f"{tag}/whitney" in PATHS:
        whitney = np.zeros_like(current)
        O.deposit_whitney(PATHS[f"{tag}/start"], PATHS[f"{tag}/end"], PATHS[f"{tag}/charges"], whitney, geom)
        np.testing.assert_allclose(whitney, PATHS[f"{tag}/whitney"], rtol=0, atol=1e-13)
        field = O.gather_edges(0, PATHS[f"{tag}/points"], PATHS[f"{tag}/edges"], geom)
        np.testing.assert_allclose(field, PATHS[f"{tag}/whitney_gather"], rtol=0, atol=1e-12)


def _form_case(tag):
    """(degree, form, ndim) of a k-form fixture tag such as ``forms2_1of3d_111``."""
    head = tag.split("_")
    return int(head[0][5:]), int(head[1][0]), int(head[1][3])


@pytest.mark.parametrize("tag", cases(FORMS))
def test_form_oracle_matches_the_reference_numpy_kernels(tag):
    degree, form, _ = _form_case(tag)
    geom = geometry(FORMS[f"{tag}/geometry"])
    result = O.gather_forms(degree, form, FORMS[f"{tag}/positions"], FORMS[f"{tag}/field"], geom)
    np.testing.assert_allclose(result, FORMS[f"{tag}/gather"], rtol=0, atol=1e-13)
    deposit = np.zeros_like(FORMS[f"{tag}/field"])
    O.scatter_forms(degree, form, FORMS[f"{tag}/dead_positions"], FORMS[f"{tag}/values"], deposit, geom)
    np.testing.assert_allclose(deposit, FORMS[f"{tag}/scatter"], rtol=0, atol=1e-13)


# ------------------------------------------------ the reference compiled as C++ --

REF_SRC = Path(os.environ.get("MPF_REFERENCE_SRC", Path(__file__).resolve().parents[2] / "reference" / "src")) / "mpifield" / "kernels"
needs_ref = pytest.mark.skipif(
    not REF_SRC.is_dir() or not (Path(O.HERE) / "_ref" / "libref_host.so").exists(),
    reason="the mpifield source tree (for oracle/_ref) is not here",
)


@needs_ref
@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("kind,degree", [("quadratic", 2), ("spline", 0), ("spline", 1), ("spline", 2), ("spline", 3)])
def test_node_oracle_is_the_reference_cuda_arithmetic_bit_for_bit(kind, degree, ndim):
    rng = np.random.default_rng(7 + degree + 10 * ndim)
    ref = O.RefHost()
    for codes in {(0,) * ndim, (1,) * ndim, ((2,) + (1,) * (ndim - 1)) if kind == "spline" and degree else (1,) * ndim}:
        shape = (9, 8, 7)[:ndim]
        ext = tuple(s + (degree - 1 if c == 2 else 0) for s, c in zip(shape, codes))
        geom = (*rng.uniform(-1, 1, ndim), *rng.uniform(0.2, 0.5, ndim), *shape, *codes)
        lower = np.array(geom[:ndim])
        cell = np.array(geom[ndim:2 * ndim])
        pos = (lower[:, None] + cell[:, None] * rng.uniform(-3, np.array(shape)[:, None] + 2, (ndim, 300)))
        field = rng.normal(size=(*ext, 2))
        expected = np.zeros((2, 300))
        name = f"gather_{kind}_{ndim}d"
        args = (pos, field, expected, *geom) + ((degree,) if kind == "spline" else ())
        ref.call(name, 300, *args)
        np.testing.assert_array_equal(O.gather(kind, degree, pos, field, geom), expected)
        values = rng.uniform(0.5, 1.5, (2, 300))
        values[:, ::11] = 0.0
        deposit = np.zeros_like(field)
        args = (pos, values, deposit, *geom) + ((degree,) if kind == "spline" else ())
        ref.call(f"scatter_{kind}_{ndim}d", 300, *args)
        mine = np.zeros_like(field)
        O.scatter(kind, degree, pos, values, mine, geom)
        np.testing.assert_array_equal(mine, deposit)


@needs_ref
@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("degree", [1, 2, 3])
def test_path_oracle_is_the_reference_cuda_arithmetic(ndim, degree):
    rng = np.random.default_rng(100 + degree + 10 * ndim)
    ref = O.RefHost()
    for codes in ((0,) * ndim, (1,) * ndim, (2,) + (1,) * (ndim - 1)):
        if 2 in codes and degree == 1:
            continue
        shape = (9, 8, 7)[:ndim]
        ext = tuple(s + (degree - 1 if c == 2 else 0) for s, c in zip(shape, codes))
        geom = (*rng.uniform(-1, 1, ndim), *rng.uniform(0.2, 0.5, ndim), *shape, *codes)
        lower = np.array(geom[:ndim])
        cell = np.array(geom[ndim:2 * ndim])
        start = lower[:, None] + cell[:, None] * rng.uniform(-2, np.array(shape)[:, None] + 1, (ndim, 200))
        end = start + cell[:, None] * rng.normal(0, 2.5, (ndim, 200))
        charges = rng.uniform(0.5, 1.5, 200)
        expected = np.zeros((*ext, ndim))
        ref.call(f"deposit_paths_spline_{ndim}d", 200, start, end, charges, expected, *geom, degree)
        mine = np.zeros_like(expected)
        O.deposit_spline(degree, start, end, charges, mine, geom)
        np.testing.assert_allclose(mine, expected, rtol=0, atol=1e-14)
        if degree == 1 and 2 not in codes:
            expected = np.zeros((*ext, ndim))
            ref.call(f"deposit_paths_{ndim}d", 200, start, end, charges, expected, *geom)
            mine = np.zeros_like(expected)
            O.deposit_whitney(start, end, charges, mine, geom)
            np.testing.assert_allclose(mine, expected, rtol=0, atol=1e-14)


@needs_ref
@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("degree", [1, 2, 3])
def test_form_oracle_is_the_reference_cuda_arithmetic(ndim, degree):
    rng = np.random.default_rng(200 + degree + 10 * ndim)
    ref = O.RefHost()
    for form in range(1, ndim + 1):
        ncomp = O.num_form_components(form, ndim)
        for codes in ((0,) * ndim, (1,) * ndim, (2,) + (1,) * (ndim - 1)):
            shape = (9, 8, 7)[:ndim]
            ext = tuple(s + (degree - 1 if c == 2 else 0) for s, c in zip(shape, codes))
            geom = (*rng.uniform(-1, 1, ndim), *rng.uniform(0.2, 0.5, ndim), *shape, *codes)
            lower = np.array(geom[:ndim])
            cell = np.array(geom[ndim:2 * ndim])
            pos = lower[:, None] + cell[:, None] * rng.uniform(-2, np.array(shape)[:, None] + 1, (ndim, 200))
            field = rng.normal(size=(*ext, ncomp))
            expected = np.zeros((ncomp, 200))
            ref.call(f"gather_forms_spline_{ndim}d", 200, pos, field, expected, *geom, degree, form)
            np.testing.assert_allclose(O.gather_forms(degree, form, pos, field, geom), expected, rtol=0, atol=1e-14)
            values = rng.uniform(0.5, 1.5, (ncomp, 200))
            deposit = np.zeros_like(field)
            ref.call(f"scatter_forms_spline_{ndim}d", 200, pos, values, deposit, *geom, degree, form)
            mine = np.zeros_like(field)
            O.scatter_forms(degree, form, pos, values, mine, geom)
            np.testing.assert_allclose(mine, deposit, rtol=0, atol=1e-14)


# --------------------------------------------------------------- known answers --


def test_quadratic_weights_on_a_node_and_between_two():
    # test_weighting.py:121-128: on node 5 -> 1/8, 3/4, 1/8; midway 2.5 with 8 -> 4, 4
    geom = (0.0, 0.1, 11, 0)
    field = np.zeros((11, 1))
    O.scatter("quadratic", 2, np.array([[0.5]]), np.array([[1.0]]), field, geom)
    O.scatter("quadratic", 2, np.array([[0.25]]), np.array([[8.0]]), field, geom)
    np.testing.assert_allclose(field[:, 0], [0, 0, 4, 4, 0.125, 0.75, 0.125, 0, 0, 0, 0], atol=1e-15)


def test_quadratic_folds_at_a_bounded_edge_and_wraps_at_a_periodic_one():
    # test_weighting.py:131-141
    field = np.zeros((11, 1))
    O.scatter("quadratic", 2, np.array([[0.0]]), np.array([[1.0]]), field, (0.0, 0.1, 11, 0))
    np.testing.assert_allclose(field[:3, 0], [0.875, 0.125, 0.0])
    field = np.zeros((11, 1))
    O.scatter("quadratic", 2, np.array([[0.0]]), np.array([[1.0]]), field, (0.0, 1.0 / 11, 11, 1))
    np.testing.assert_allclose(field[[-1, 0, 1], 0], [0.125, 0.75, 0.125])


def test_linear_deposit_past_a_bounded_end_stays_on_the_edge_node():
    # test_weighting.py:144-152
    field = np.zeros((11, 1))
    O.scatter("linear", 1, np.array([[1.2, -0.3]]), np.array([[1.0, 2.0]]), field, (0.0, 0.1, 11, 0))
    assert field[-1, 0] == 1.0 and field[0, 0] == 2.0 and field.sum() == 3.0


def test_linear_gather_wraps_on_a_periodic_axis():
    # test_weighting.py:155-165
    result = O.gather("linear", 1, np.array([[0.875, 1.125]]), np.array([[0.0], [1.0], [2.0], [3.0]]),
                      (0.0, 0.25, 4, 1))
    np.testing.assert_allclose(result, [[1.5, 0.5]])


def test_linear_gather_uses_the_edge_cell_outside_the_grid():
    # test_field.py:530-539
    result = O.gather("linear", 1, np.array([[-0.5, 0.5, 2.5, 3.0, 3.7]]),
                      np.array([[1.0], [2.0], [4.0], [8.0]]), (0.0, 1.0, 4, 0))
    np.testing.assert_allclose(result[0], [1.0, 1.5, 6.0, 8.0, 8.0])


def test_degree_zero_is_the_nearest_grid_point():
    # test_splines.py:108-113
    field = np.zeros((6, 1))
    O.scatter("spline", 0, np.array([[0.2, 1.49, 1.51, 4.7, 9.0, -3.0]]), np.ones((1, 6)), field, (0.0, 1.0, 6, 0))
    np.testing.assert_array_equal(field[:, 0], [2, 1, 1, 0, 0, 2])


def test_cubic_weights_and_folds():
    # test_splines.py:116-138 through a deposit of one marker
    d = 0.37
    field = np.zeros((10, 1))
    O.scatter("spline", 3, np.array([[3.0 + d]]), np.array([[1.0]]), field, (0.0, 1.0, 10, 1))
    expected = [(1 - d) ** 3 / 6, (3 * d**3 - 6 * d**2 + 4) / 6, (-3 * d**3 + 3 * d**2 + 3 * d + 1) / 6, d**3 / 6]
    np.testing.assert_allclose(field[2:6, 0], expected, rtol=1e-14)
    field = np.zeros((8, 1))
    O.scatter("spline", 3, np.array([[0.0]]), np.array([[1.0]]), field, (0.0, 1.0, 8, 0))
    np.testing.assert_allclose(field[:3, 0], [1 / 6 + 2 / 3, 1 / 6, 0.0], rtol=1e-14)


def test_a_path_outside_a_bounded_axis_moves_along_the_wall():
    # test_edges.py:175-182: from (0.5, -1) to (2.5, -1) -> [0.5, 1, 0.5] on the x edges of y = 0
    current = np.zeros((4, 4, 2))
    O.deposit_whitney(np.array([[0.5], [-1.0]]), np.array([[2.5], [-1.0]]), np.array([1.0]), current,
                      (0.0, 0.0, 1.0, 1.0, 4, 4, 0, 0))
    np.testing.assert_allclose(current[:3, 0, 0], [0.5, 1.0, 0.5])
    assert np.count_nonzero(current) == 3


def test_dead_and_non_finite_paths_deposit_nothing():
    # test_edges.py:102-107
    current = np.zeros((6, 5, 2))
    start = np.array([[0.1, np.nan, 0.2], [0.3, 0.1, np.inf]])
    O.deposit_whitney(start, start + 0.4, np.array([0.0, 1.0, 2.0]), current, (0.0, 0.0, 0.3, 0.3, 6, 5, 0, 1))
    assert np.all(current == 0.0)
    for degree in (1, 2, 3):
        O.deposit_spline(degree, start, start + 0.4, np.array([0.0, 1.0, 2.0]), current, (0.0, 0.0, 0.3, 0.3, 6, 5, 0, 1))
    assert np.all(current == 0.0)


def test_a_uniform_edge_field_is_gathered_exactly():
    # test_spline_edges.py:138-155
    geom = (0.0, 0.0, 0.5, 0.25, 8, 9, 0, 1)
    edges = np.zeros((8, 9, 2))
    edges[:-1, :, 0] = 0.5 * 3.0
    edges[:, :, 1] = 0.25 * -2.0
    points = np.random.default_rng(3).uniform([1.0, -1.0], [2.5, 3.0], (50, 2)).T
    for degree in (0, 1, 2, 3):
        field = O.gather_edges(degree, points, edges, geom)
        np.testing.assert_allclose(field[0], 3.0, atol=1e-12)
        np.testing.assert_allclose(field[1], -2.0, atol=1e-12)


# ---------------------------------------------------------------- invariants --


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("degree", [1, 2, 3])
def test_path_deposits_conserve_the_node_charge(ndim, periodic, degree):
    # test_edges.py:59-66 and test_spline_edges.py:67-87: G^T j = rho(end) - rho(start)
    rng = np.random.default_rng(degree * 10 + ndim)
    shape = (9, 8, 7)[:ndim]
    geom = (*[0.0, -1.0, 2.0][:ndim], *[0.25, 0.5, 0.1][:ndim], *shape, *(int(periodic),) * ndim)
    lower = np.array(geom[:ndim])
    cell = np.array(geom[ndim:2 * ndim])
    upper = lower + cell * (np.array(shape) - 1)
    start = rng.uniform(lower - 3 * cell, upper + 3 * cell, (200, ndim)).T.copy()
    end = start + rng.normal(scale=3.0 * cell[:, None], size=start.shape)
    charges = rng.normal(size=200)
    current = np.zeros((*shape, ndim))
    if degree == 1:
        O.deposit_whitney(start, end, charges, current, geom)
        kind = "linear"
    else:
        O.deposit_spline(degree, start, end, charges, current, geom)
        kind = "quadratic" if degree == 2 else "spline"
    before = np.zeros((*shape, 1))
    after = np.zeros((*shape, 1))
    O.scatter(kind, degree, start, charges[None], before, geom)
    O.scatter(kind, degree, end, charges[None], after, geom)
    np.testing.assert_allclose(O.divergence_block(current, (periodic,) * ndim), (after - before)[..., 0],
                               rtol=0, atol=1e-12)


@pytest.mark.parametrize("ndim", [2, 3])
def test_stored_block_with_halos_deposits_and_gathers_as_the_bare_grid(ndim):
    # test_field.py:542-581: a padded periodic first axis, folded, equals the bare periodic deposit;
    # after a fill, the gathers are equal
    rng = np.random.default_rng(5)
    shape = (7, 5, 4)[:ndim]
    h = 1
    spacing = np.array([1.0 / shape[0]] + [1.0 / (s - 1) for s in shape[1:]])
    bare_geom = (*([0.0] * ndim), *spacing, *shape, 1, *([0] * (ndim - 1)))
    padded_shape = (shape[0] + 2 * h,) + tuple(shape[1:])
    padded_geom = (-h * spacing[0], *([0.0] * (ndim - 1)), *spacing, *padded_shape, *([0] * ndim))
    positions = rng.uniform(0.0, 1.0, (ndim, 400))
    positions[1:] *= 0.999
    values = rng.uniform(0.5, 1.5, (1, 400))
    bare = np.zeros((*shape, 1))
    O.scatter("linear", 1, positions, values, bare, bare_geom)
    # the padded storage holds halos on every axis; the kernels see only the periodic axis padded
    stored = np.zeros(tuple(s + 2 * h for s in shape) + (1,))
    inner = (slice(None),) + tuple(slice(h, h + s) for s in shape[1:])
    view = stored[inner]
    block = np.zeros(padded_shape + (1,))
    O.scatter("linear", 1, positions, values, block, padded_geom)
    view[...] = block
    O.halo_fold(stored, h, (True,) + (False,) * (ndim - 1))
    owned = tuple(slice(h, h + s) for s in shape)
    np.testing.assert_allclose(stored[owned], bare, atol=1e-14)
    O.halo_fill(stored, h, (True,) + (False,) * (ndim - 1))
    gathered = O.gather("linear", 1, positions, np.ascontiguousarray(stored[inner]), padded_geom)
    np.testing.assert_allclose(gathered, O.gather("linear", 1, positions, bare, bare_geom), atol=1e-13)


def test_tile_keys_and_stable_order():
    rng = np.random.default_rng(0)
    geom = (0.0, 0.0, 0.0, 0.1, 0.1, 0.1, 10, 10, 10, 1, 1, 1)
    pos = rng.uniform(0, 1, (3, 1000))
    values = rng.uniform(0.5, 1.5, (1, 1000))
    values[0, ::7] = 0.0
    pos[:, ::7] = np.nan
    keys = O.tile_keys("quadratic", 2, pos, geom, (4, 4, 4), values)
    assert keys.max() == 27 and (keys[::7] == 27).all()
    live = keys[keys < 27]
    assert live.min() >= 0 and live.max() < 27
    order = O.sort_by_tile(keys)
    assert (np.diff(keys[order].astype(np.int64)) >= 0).all()
    for k in np.unique(keys):
        idx = order[keys[order] == k]
        assert (np.diff(idx) > 0).all()  # stable
    inner = O.tile_keys("quadratic", 2, pos, geom, (4, 4, 4), values, within=True)
    assert inner.max() == 27 * 64
    np.testing.assert_array_equal(inner[keys < 27] // 64, keys[keys < 27])


def test_adjoint_identity_of_the_oracle():
    # test_catalog_and_pyccel.py:163-182
    rng = np.random.default_rng(1)
    for kind, degree in (("linear", 1), ("quadratic", 2), ("spline", 3)):
        geom = (0.0, 0.0, 0.1, 0.2, 12, 7, 1, 0)
        pos = rng.uniform(-0.2, 1.4, (2, 300))
        q = rng.normal(size=(1, 300))
        f = rng.normal(size=(12, 7, 1))
        rho = np.zeros_like(f)
        O.scatter(kind, degree, pos, q, rho, geom)
        assert np.sum(O.gather(kind, degree, pos, f, geom) * q) == pytest.approx(np.sum(f * rho), rel=1e-12)
