"""GPU: halo fill and fold-back, deposit_density, sorting and the position gradient."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import mpifield_b200 as mf
from mpifield_b200 import _lib
from mpifield_b200.kernels import gather_grad
from oracle import oracle as O
from tests.helpers import KIND_NAMES, RTOL_F64, random_case, rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"


def cu(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("halo", [1, 2])
def test_halo_fill_and_fold_match_the_oracle(ndim, halo):
    rng = np.random.default_rng(ndim * 3 + halo)
    owned = (7, 5, 4)[:ndim]
    for periodic in [(True,) * ndim, tuple(d % 2 == 0 for d in range(ndim))]:
        stored = rng.normal(size=tuple(s + 2 * halo for s in owned) + (3,))
        f = mf.Field(ndim, (0.0,) * ndim, (1.0,) * ndim, owned, 3, periodic, halo)
        f.local_with_halos.copy_(cu(stored))
        f.fill_halos()
        np.testing.assert_array_equal(f.local_with_halos.cpu().numpy(), O.halo_fill(stored.copy(), halo, periodic))
        f.local_with_halos.copy_(cu(stored))
        f.exchange_halos()
        np.testing.assert_allclose(f.local_with_halos.cpu().numpy(), O.halo_fold(stored.copy(), halo, periodic),
                                   rtol=0, atol=1e-14)


@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("weighting", [mf.LINEAR, mf.QUADRATIC, mf.CUBIC], ids=lambda w: w.name)
def test_a_block_with_halos_deposits_and_gathers_as_the_bare_grid(ndim, weighting):
    # src/mpifield/tests/unit/test_field.py:542-581 (with the halo width of the weighting)
    shape = (9, 7, 6)[:ndim]
    periodic = (True,) + (False,) * (ndim - 1)
    kwargs = dict(ndim=ndim, lower_bound=(0.0,) * ndim, upper_bound=(1.0,) * ndim, num_gridpoints=shape,
                  periodic=periodic)
    bare = mf.Field(**kwargs)
    padded = mf.Field(**kwargs, num_ghost_points=weighting.halo)
    assert tuple(padded.block_grid().num_gridpoints) == tuple(n + 2 * weighting.halo for n in shape)
    assert padded.block_grid().periodic == (False,) * ndim
    rng = np.random.default_rng(5)
    positions = rng.uniform(0.0, 1.0, (ndim, 4000))
    positions[1:] *= 0.999
    values = rng.uniform(0.5, 1.5, 4000)
    bare.scatter(positions, values, weighting)
    padded.scatter(positions, values, weighting)
    padded.exchange_halos()
    np.testing.assert_allclose(padded.local.cpu().numpy(), bare.local.cpu().numpy(), rtol=0, atol=1e-12)
    padded.fill_halos()
    np.testing.assert_allclose(padded.gather(positions, weighting).cpu().numpy(),
                               bare.gather(positions, weighting).cpu().numpy(), rtol=0, atol=1e-12)


@pytest.mark.parametrize("periodic", [False, True])
def test_deposit_density(periodic):
    # field.py:1182-1218: local += deposit / node_volumes
    rng = np.random.default_rng(9)
    f = mf.Field(2, (0.0, 0.0), (1.0, 0.5), (11, 7), 2, (periodic, False))
    positions = rng.uniform(0, 1, (2, 3000)) * np.array([[1.0], [0.5]])
    values = rng.uniform(0.5, 1.5, (2, 3000))
    f.set_field_data(1.0)
    f.deposit_density(positions, values, mf.QUADRATIC)
    grid = f.block_grid(inside_domain=True)
    deposit = O.scatter("quadratic", 2, positions, values, np.zeros((11, 7, 2)), grid.geometry)
    vol = O.node_volumes((11, 7), f.grid_spacing, (periodic, False))
    np.testing.assert_allclose(f.local.cpu().numpy(), 1.0 + deposit / vol[..., None], rtol=1e-12)
    # the total charge is the sum of density times volume
    np.testing.assert_allclose(((f.local.cpu().numpy() - 1.0) * vol[..., None]).sum((0, 1)), values.sum(1), rtol=1e-12)
    np.testing.assert_allclose(f.node_volumes().local[..., 0].cpu().numpy(), vol, rtol=1e-15)


@pytest.mark.parametrize("kind,degree", [("linear", 1), ("quadratic", 2), ("spline", 0), ("spline", 3)])
@pytest.mark.parametrize("ndim", [1, 2, 3])
def test_tile_keys_and_order_are_bit_exact(kind, degree, ndim):
    rng = np.random.default_rng(ndim)
    for codes in ((1,) * ndim, (0,) * ndim) + ((((2,) + (0,) * (ndim - 1)),) if kind == "spline" and degree else ()):
        geom, pos, _, values = random_case(rng, ndim, codes, degree, n=300_003, ncomp=2, shape=(37, 29, 23)[:ndim])
        values[:, ::5] = 0.0
        pos[:, ::10] = np.nan  # dead markers: keys without reading the position
        # power-of-two extents (the key's quotient by a shift) and others (by a division)
        for tile, within in ((ext[:ndim], w) for ext in ((8, 4, 2), (5, 3, 7)) for w in (False, True)):
            t = mf.sort_by_tile(cu(pos), (KIND_NAMES[kind], degree), geom, tile, cu(values), within=within)
            keys = O.tile_keys(kind, degree, pos, geom, tile, values, within=within)
            np.testing.assert_array_equal(t.keys.cpu().numpy().view(np.uint32), keys)
            np.testing.assert_array_equal(t.order.cpu().numpy(), O.sort_by_tile(keys))
            cells = int(np.prod(tile)) if within else 1
            starts = np.searchsorted(np.sort(keys) // cells, np.arange(t.num_tiles + 1), side="left")
            np.testing.assert_array_equal(t.tile_start.cpu().numpy(), np.append(starts, keys.size))


def test_sort_edge_cases_and_permute():
    geom = (0.0, 0.1, 10, 1)
    for n in (0, 1, 2, 4095, 4096, 4097):
        pos = np.random.default_rng(n).uniform(0, 1, (1, n))
        t = mf.sort_by_tile(cu(pos), (1, 2), geom, (3,))
        keys = O.tile_keys("quadratic", 2, pos, geom, (3,))
        np.testing.assert_array_equal(t.order.cpu().numpy(), O.sort_by_tile(keys))
        assert int(t.tile_start[-1]) == n
    pos = np.random.default_rng(0).uniform(0, 1, (3, 1000))
    order = torch.randperm(1000, device=DEV).to(torch.int32)
    np.testing.assert_array_equal(mf.permute(cu(pos), order).cpu().numpy(), pos[:, order.cpu().numpy()])
    # a 25-bit key (256^3 cells within 8^3 tiles) takes three passes
    pos = np.random.default_rng(1).uniform(0, 1, (3, 200_000))
    geom3 = (0.0, 0.0, 0.0, 1 / 256, 1 / 256, 1 / 256, 256, 256, 256, 1, 1, 1)
    t = mf.sort_by_tile(cu(pos), (1, 2), geom3, (8, 8, 8), within=True)
    keys = O.tile_keys("quadratic", 2, pos, geom3, (8, 8, 8), within=True)
    np.testing.assert_array_equal(t.order.cpu().numpy(), O.sort_by_tile(keys))
    # equal keys keep the marker order (the sort is stable) for many equal keys
    same = np.full((1, 100_000), 0.55)
    t = mf.sort_by_tile(cu(same), (1, 2), geom, (3,))
    np.testing.assert_array_equal(t.order.cpu().numpy(), np.arange(100_000))


def test_correctly_rounded_division_matches_the_gpu_division():
    """The reciprocal-based quotient the kernels use for (x - lower) / h is bit-identical to
    the IEEE division: checked through the cell keys of markers near cell boundaries."""
    rng = np.random.default_rng(12)
    for h in (1 / 256, 0.1, 0.3, 1 / 3, 7.0, 1e-3, 2.0 ** -20 * 3):
        k = rng.integers(0, 200, 100_000)
        x = (k * h) * (1 + rng.integers(-4, 5, k.size) * 2.0 ** -52)
        geom = (0.0, h, 200, 1)
        t = mf.sort_by_tile(cu(x[None]), (0, 1), geom, (1,))
        np.testing.assert_array_equal(t.keys.cpu().numpy().view(np.uint32),
                                      O.tile_keys("linear", 1, x[None], geom, (1,)))


@pytest.mark.parametrize("kind,degree", [("linear", 1), ("quadratic", 2), ("spline", 1), ("spline", 2), ("spline", 3)])
@pytest.mark.parametrize("ndim", [1, 2, 3])
def test_position_gradient_matches_the_oracle_and_finite_differences(kind, degree, ndim):
    rng = np.random.default_rng(degree + 5 * ndim)
    for codes in ((1,) * ndim, (0,) * ndim) + ((((2,) + (1,) * (ndim - 1)),) if kind == "spline" else ()):
        geom, pos, field, values = random_case(rng, ndim, codes, degree, n=2000, ncomp=2, spread=0.5)
        grad = gather_grad(KIND_NAMES[kind], degree, cu(pos), cu(field), cu(values), geom).cpu().numpy()
        expected = O.gather_grad(kind, degree, pos, field, values, geom)
        assert rel_err(grad, expected) < RTOL_F64
        # central differences away from the knots and the bounded ends
        cell = np.array(geom[ndim:2 * ndim])
        lower = np.array(geom[:ndim])
        rel = (pos - lower[:, None]) / cell[:, None]
        num = np.array(geom[2 * ndim:3 * ndim])
        shift = 0.5 if degree % 2 == 0 else 0.0
        frac = np.mod(rel + shift, 1.0)
        inside = ((frac > 0.05) & (frac < 0.95)).all(0)
        inside &= ((rel > 0.1) & (rel < num[:, None] - 1.1)).all(0)
        eps = 1e-6
        for d in range(ndim):
            step = np.zeros((ndim, 1))
            step[d] = eps * cell[d]
            up = O.gather(kind, degree, pos + step, field, geom)
            dn = O.gather(kind, degree, pos - step, field, geom)
            fd = ((up - dn) * values).sum(0) / (2 * eps * cell[d])
            np.testing.assert_allclose(grad[d, inside], fd[inside], rtol=1e-5, atol=1e-5 * np.abs(fd).max())


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("halo", [1, 2])
def test_halo_slabs_and_the_one_rank_exchange(ndim, halo):
    """mpf_halo_pack / mpf_halo_unpack against tensor slicing, and the halo exchange of a
    field split over one rank against the one-process mpf_halo_fill / mpf_halo_fold."""
    from mpifield_b200.exchange import Decomposition, HaloExchange, kernel_pack, kernel_unpack

    rng = np.random.default_rng(ndim * 10 + halo)
    num = (9, 6, 5)[:ndim]
    stored = tuple(m + 2 * halo for m in num)
    for dtype in (torch.float64, torch.float32):
        t = torch.tensor(rng.normal(size=(*stored, 3)), dtype=dtype, device="cuda")
        for axis in range(ndim):
            for first in (0, halo, stored[axis] - halo):
                buf = torch.empty(t.numel() // stored[axis] * halo, dtype=dtype, device="cuda")
                kernel_pack(t, halo, axis, first, buf)
                assert torch.equal(buf, t.narrow(axis, first, halo).reshape(-1))
                before = t.clone()
                kernel_unpack(t, halo, axis, first, buf * 2, True)
                expected = before.clone()
                expected.narrow(axis, first, halo).mul_(3)
                torch.testing.assert_close(t, expected, rtol=1e-6, atol=1e-6)
                kernel_unpack(t, halo, axis, first, buf, False)
                assert torch.equal(t.narrow(axis, first, halo).reshape(-1), buf)
    for periodic in ((True,) * ndim, tuple(a % 2 == 0 for a in range(ndim))):
        ex = HaloExchange(Decomposition(num, periodic, (1,) * ndim, 0), halo)
        f = mf.Field(ndim, [0.0] * ndim, [1.0] * ndim, num, 3, periodic=periodic, num_ghost_points=halo,
                     device="cuda")
        data = torch.tensor(rng.normal(size=(*stored, 3)), device="cuda")
        f.local_with_halos.copy_(data)
        mine = data.clone()
        f.fill_halos()
        ex.fill(mine)
        assert torch.equal(mine, f.local_with_halos)
        f.local_with_halos.copy_(data)
        mine = data.clone()
        f.exchange_halos()
        ex.fold(mine)
        torch.testing.assert_close(mine, f.local_with_halos, rtol=0, atol=1e-13)
