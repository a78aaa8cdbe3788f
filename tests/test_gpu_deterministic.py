"""GPU: the bit-reproducible scatter (mpf_scatter_deterministic).

The same bits for repeated runs and for the markers in another order; within RTOL_F64 of
the oracle (the fixed-point quantum is far below FP64 rounding), dead markers skipped.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

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
