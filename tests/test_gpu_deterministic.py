"""GPU: the bit-reproducible scatter (mpf_scatter_deterministic and its tile form).

The same bits for repeated runs and for the markers in another order; within RTOL_F64 of
the oracle (the fixed-point quantum is far below FP64 rounding), dead markers skipped. The
tile form (mpf_scatter_deterministic_tiles: markers sorted by cell tile, sums gathered in
shared memory per tile) gives the same bits as the plain form on every store, tile shape,
boundary and component count it is given, including tile starts of another store.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import mpifield_b200 as mf
from mpifield_b200.kernels import scatter_deterministic
from oracle import oracle as O
from tests.helpers import KIND_NAMES, RTOL_F64, random_case, rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _det(kind, degree, pos, values, shape, geom):
    field = torch.zeros(shape, dtype=torch.float64, device=DEV)
    scatter_deterministic(KIND_NAMES[kind], degree, pos, values, field, geom)
    return field


def test_the_same_bits_every_run_and_every_marker_order():
    g = torch.Generator(device=DEV).manual_seed(3)
    n = 1 << 20
    pos = torch.rand((3, n), generator=g, device=DEV, dtype=torch.float64)
    pos[:, : n // 4] = torch.remainder(0.5 + 0.03 * torch.randn((3, n // 4), generator=g, device=DEV,
                                                                 dtype=torch.float64), 1.0)
    w = torch.rand((1, n), generator=g, device=DEV, dtype=torch.float64) + 0.5
    geom = (0.0, 0.0, 0.0, 1 / 48, 1 / 48, 1 / 48, 48, 48, 48, 1, 1, 1)
    first = _det("quadratic", 2, pos, w, (48, 48, 48, 1), geom)
    for _ in range(2):
        again = _det("quadratic", 2, pos, w, (48, 48, 48, 1), geom)
        assert torch.equal(first.view(torch.int64), again.view(torch.int64))
    perm = torch.randperm(n, generator=torch.Generator().manual_seed(1)).to(DEV)
    shuffled = _det("quadratic", 2, pos[:, perm], w[:, perm], (48, 48, 48, 1), geom)
    assert torch.equal(first.view(torch.int64), shuffled.view(torch.int64))
    expected = O.scatter("quadratic", 2, pos[:, :200000].cpu().numpy(), w[:, :200000].cpu().numpy(),
                         np.zeros((48, 48, 48, 1)), geom)
    part = _det("quadratic", 2, pos[:, :200000], w[:, :200000], (48, 48, 48, 1), geom)
    assert rel_err(part.cpu().numpy(), expected) < RTOL_F64


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("kind,degree", [("linear", 1), ("quadratic", 2), ("spline", 0), ("spline", 3)])
def test_random_cases_match_the_oracle(kind, degree, ndim):
    rng = np.random.default_rng(hash((kind, degree, ndim, "det")) % 2**32)
    codes_list = [(1,) * ndim, (0,) * ndim]
    if kind == "spline" and degree >= 1:
        codes_list.append((2,) + (1,) * (ndim - 1))
    for codes in codes_list:
        geom, pos, field, values = random_case(rng, ndim, codes, degree, n=5000, ncomp=2, shape=(17, 13, 11)[:ndim])
        values[:, ::9] = 0.0
        pos[:, ::27] = np.nan  # dead markers: never read
        values[:, ::27] = 0.0
        expected = O.scatter(kind, degree, pos, values, np.zeros_like(field), geom)
        got = _det(kind, degree, torch.tensor(pos, device=DEV), torch.tensor(values, device=DEV), field.shape, geom)
        assert rel_err(got.cpu().numpy(), expected) < RTOL_F64


def test_it_adds_into_the_field():
    geom = (0.0, 0.5, 8, 1)
    base = torch.arange(8, dtype=torch.float64, device=DEV).view(8, 1)
    field = base.clone()
    scatter_deterministic(KIND_NAMES["linear"], 1, torch.tensor([[1.25]], device=DEV, dtype=torch.float64),
                          torch.tensor([[2.0]], device=DEV, dtype=torch.float64), field, geom)
    delta = (field - base).cpu().numpy()[:, 0]
    np.testing.assert_allclose(delta[2:4], [1.0, 1.0], rtol=0, atol=1e-15)
    assert delta.sum() == pytest.approx(2.0, abs=1e-14)


def _sorted_store(n, shape, codes, kind, degree, tile, seed, ncomp=1, dead=0.0):
    g = torch.Generator(device=DEV).manual_seed(seed)
    ndim = len(shape)
    pos = torch.rand((ndim, n), generator=g, device=DEV, dtype=torch.float64) * 1.2 - 0.1
    w = torch.rand((ncomp, n), generator=g, device=DEV, dtype=torch.float64) + 0.5
    if dead:
        w[:, torch.rand(n, generator=g, device=DEV) < dead] = 0.0
    geom = (*[0.0] * ndim, *[1.0 / s for s in shape], *shape, *codes)
    order = mf.sort_by_tile(pos, (KIND_NAMES[kind], degree), geom, tile, values=w, within=True)
    return geom, mf.permute(pos, order.order).contiguous(), mf.permute(w, order.order).contiguous(), order


CASES = [((64, 48, 128), (1, 1, 1), "quadratic", 2, (4, 4, 64), 1),
         ((40, 40, 40), (1, 1, 1), "quadratic", 2, (8, 8, 8), 1),
         ((40, 36, 30), (1, 1, 1), "spline", 3, (6, 5, 8), 1),
         ((90, 70), (1, 1), "linear", 1, (16, 16), 1),
         ((300,), (1,), "spline", 0, (32,), 1),
         ((40, 40, 40), (1, 1, 1), "quadratic", 2, (8, 8, 8), 2),
         ((30, 30, 30), (0, 1, 2), "spline", 2, (8, 8, 8), 1)]


@pytest.mark.parametrize("shape,codes,kind,degree,tile,ncomp", CASES,
                         ids=["q3d_4x4x64", "q3d_8cubed", "cubic3d_runtime", "linear2d", "ngp1d", "two_comp",
                              "mixed_codes"])
def test_the_tile_form_has_the_same_bits(shape, codes, kind, degree, tile, ncomp):
    ext = tuple(s + (degree - 1 if c == 2 else 0) for s, c in zip(shape, codes))
    geom, ps, ws, order = _sorted_store(200000, shape, codes, kind, degree, tile, 7, ncomp, dead=0.05)
    plain = torch.zeros(ext + (ncomp,), dtype=torch.float64, device=DEV)
    scatter_deterministic(KIND_NAMES[kind], degree, ps, ws, plain, geom)
    tiles = torch.zeros_like(plain)
    scatter_deterministic(KIND_NAMES[kind], degree, ps, ws, tiles, geom, order=order)
    assert torch.equal(plain.view(torch.int64), tiles.view(torch.int64))
    oracle = O.scatter(kind, degree, ps.cpu().numpy(), ws.cpu().numpy(), np.zeros(ext + (ncomp,)), geom)
    assert rel_err(tiles.cpu().numpy(), oracle) < RTOL_F64


def test_the_tile_form_with_the_tile_starts_of_another_store():
    geom, ps, ws, order = _sorted_store(100000, (40, 40, 40), (1, 1, 1), "quadratic", 2, (8, 8, 8), 8)
    perm = torch.randperm(ps.shape[1], generator=torch.Generator().manual_seed(2)).to(DEV)
    ps, ws = ps[:, perm].contiguous(), ws[:, perm].contiguous()
    plain = torch.zeros((40, 40, 40, 1), dtype=torch.float64, device=DEV)
    scatter_deterministic(KIND_NAMES["quadratic"], 2, ps, ws, plain, geom)
    tiles = torch.zeros_like(plain)
    scatter_deterministic(KIND_NAMES["quadratic"], 2, ps, ws, tiles, geom, order=order)
    assert torch.equal(plain.view(torch.int64), tiles.view(torch.int64))
