"""GPU: the differentiable gather and scatter (mpifield_b200.autograd).

Checked three ways, as the method's identities give them: finite differences
(torch.autograd.gradcheck in float64 at 16 x 16, N = 256, cubic, periodic), the FP64
oracle's own gradient (the oracle's scatter, gather and position gradient composed by
hand, within RTOL_F64), and the adjoint identity <scatter(x, w), f> = <w, gather(f, x)>.
The float32 variant is held to RTOL_F32 of the float64 gradients.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import mpifield_b200 as mf
from mpifield_b200 import autograd as AG
from oracle import oracle as O
from tests.helpers import RTOL_F32, RTOL_F64, rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _loss(f, w, x, weighting, geom):
    """The differentiation workload: sum(w * gather(f, x)) + 0.5 * ||scatter(x, w)||^2."""
    rho = AG.scatter(x, w, weighting, geom)
    return (w * AG.gather(f, x, weighting, geom)).sum() + 0.5 * (rho * rho).sum()


def _case(n_side, n, seed, dtype=torch.float64):
    rng = np.random.default_rng(seed)
    geom = (0.0, 0.0, 1.0 / n_side, 1.0 / n_side, n_side, n_side, 1, 1)
    f = torch.tensor(rng.normal(size=(n_side, n_side, 1)), dtype=dtype, device=DEV)
    w = torch.tensor(rng.uniform(0, 1, (1, n)), dtype=dtype, device=DEV)
    x = torch.tensor(rng.uniform(0, 1, (2, n)), dtype=dtype, device=DEV)
    return geom, f, w, x


def test_gradcheck_cubic_16x16():
    geom, f, w, x = _case(16, 256, 0)
    f.requires_grad_(True)
    w.requires_grad_(True)
    x.requires_grad_(True)
    # scatter adds with atomics: the order of the adds moves results by a few ulp
    assert torch.autograd.gradcheck(lambda f, w, x: _loss(f, w, x, mf.CUBIC, geom), (f, w, x),
                                    eps=1e-6, atol=1e-6, rtol=1e-4, nondet_tol=1e-10)


@pytest.mark.parametrize("weighting", [mf.LINEAR, mf.QUADRATIC, mf.CUBIC], ids=["linear", "quadratic", "cubic"])
def test_gathers_and_scatters_pass_gradcheck(weighting):
    geom, _, _, x = _case(12, 64, 1)
    f = torch.rand((12, 12, 2), dtype=torch.float64, device=DEV, requires_grad=True)
    v = torch.rand((2, 64), dtype=torch.float64, device=DEV, requires_grad=True)
    x.requires_grad_(True)
    assert torch.autograd.gradcheck(lambda f, x: AG.gather(f, x, weighting, geom), (f, x), eps=1e-6, atol=1e-6,
                                    rtol=1e-4, nondet_tol=1e-10)
    assert torch.autograd.gradcheck(lambda x, v: AG.scatter(x, v, weighting, geom), (x, v), eps=1e-6, atol=1e-6,
                                    rtol=1e-4, nondet_tol=1e-10)


def test_gradients_equal_the_fp64_oracle():
    # d/df = scatter(x, w); d/dw = gather(f + rho, x); d/dx = w * grad gather(f + rho, x)
    geom, f, w, x = _case(64, 4096, 2)
    f.requires_grad_(True)
    w.requires_grad_(True)
    x.requires_grad_(True)
    _loss(f, w, x, mf.CUBIC, geom).backward()
    pos, wn, fn = x.detach().cpu().numpy(), w.detach().cpu().numpy(), f.detach().cpu().numpy()
    rho = O.scatter("spline", 3, pos, wn, np.zeros_like(fn), geom)
    assert rel_err(f.grad.cpu().numpy(), rho) < RTOL_F64
    assert rel_err(w.grad.cpu().numpy(), O.gather("spline", 3, pos, fn + rho, geom)) < RTOL_F64
    assert rel_err(x.grad.cpu().numpy(), O.gather_grad("spline", 3, pos, fn + rho, wn, geom)) < RTOL_F64


@pytest.mark.parametrize("ndim,weighting,codes", [(1, mf.LINEAR, (0,)), (2, mf.CUBIC, (1, 0)),
                                                  (3, mf.QUADRATIC, (1, 1, 1)),
                                                  (2, mf.splines(2, clamped=True).nodes, (2, 1))])
def test_adjoint_identity(ndim, weighting, codes):
    rng = np.random.default_rng(3)
    shape = (9, 7, 6)[:ndim]
    geom = (*[0.0] * ndim, *[1.0] * ndim, *shape, *codes)
    extent = tuple(n + (weighting.degree - 1 if c == 2 else 0) for n, c in zip(shape, codes))
    f = torch.tensor(rng.normal(size=extent + (2,)), device=DEV)
    x = torch.tensor(rng.uniform(-0.5, np.array(shape)[:, None] - 0.5, (ndim, 3000)), device=DEV)
    w = torch.tensor(rng.normal(size=(2, 3000)), device=DEV)
    left = (AG.scatter(x, w, weighting, geom) * f).sum()
    right = (w * AG.gather(f, x, weighting, geom)).sum()
    assert abs(left - right).item() <= 1e-12 * max(abs(left).item(), 1.0)


def test_position_gradient_vanishes_where_a_bounded_axis_clamps():
    geom = (0.0, 1.0, 8, 0)
    f = torch.linspace(0, 1, 8, dtype=torch.float64, device=DEV).view(8, 1)
    x = torch.tensor([[-2.0, 3.3, 9.5]], dtype=torch.float64, device=DEV, requires_grad=True)
    AG.gather(f, x, mf.QUADRATIC, geom).sum().backward()
    g = x.grad.cpu().numpy()[0]
    assert g[0] == 0.0 and g[2] == 0.0 and g[1] != 0.0


def test_float32_gradients_are_within_the_stated_bound():
    geom, f, w, x = _case(64, 4096, 4)
    grads = {}
    for dtype in (torch.float64, torch.float32):
        ff, ww, xx = (t.to(dtype).clone().requires_grad_(True) for t in (f, w, x))
        _loss(ff, ww, xx, mf.CUBIC, geom).backward()
        grads[dtype] = [t.grad.double().cpu().numpy() for t in (ff, ww, xx)]
    for g32, g64 in zip(grads[torch.float32], grads[torch.float64]):
        assert rel_err(g32, g64) < RTOL_F32 * 10
