"""The give-up path of the gathers' bounded waits, made to run out on purpose.

The gathers prefetch positions with bulk copies that complete on an mbarrier; every wait
on one is bounded, and a CTA that gives up waits for its copies still in flight, raises
MPF_DEVICE_ERROR_WAIT and leaves. A launch with ``wait_limit < 0`` gives up at the first
wait (no fault, no hang: the copies themselves complete normally). The call must return,
the error bit must be reported and cleared, and the next call with the default limit
must be exact again.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from mpifield_b200 import _lib
from mpifield_b200.kernels import gather
from oracle import oracle as O
from tests.helpers import RTOL_F64, rel_err

pytestmark = pytest.mark.gpu


def _case(n=200_000, grid=24):
    rng = np.random.default_rng(11)
    geom = (0.0, 0.0, 0.0, 1 / grid, 1 / grid, 1 / grid, grid, grid, grid, 1, 1, 1)
    pos = rng.uniform(0.0, 1.0, (3, n))
    field = rng.normal(size=(grid, grid, grid, 3))
    return geom, pos, field


@pytest.mark.parametrize("variant", [0, 1])
def test_a_wait_that_runs_out_is_reported_and_the_next_call_is_exact(variant):
    geom, pos, field = _case()
    expected = O.gather("quadratic", 2, pos, field, geom)
    p = torch.tensor(pos, device="cuda")
    f = torch.tensor(field, device="cuda")
    out = torch.zeros((3, pos.shape[1]), dtype=torch.float64, device="cuda")
    assert _lib.device_errors(clear=True) == 0
    # variant 0: the gather through L1; 1: the staged-box gather (both prefetch by bulk copy)
    gather(_lib.QUADRATIC, 2, p, f, out, geom, _lib.tuning_struct(variant=variant, wait_limit=-1))
    torch.cuda.synchronize()
    assert _lib.device_errors(clear=True) & 1  # MPF_DEVICE_ERROR_WAIT
    assert _lib.device_errors(clear=True) == 0  # cleared
    gather(_lib.QUADRATIC, 2, p, f, out, geom, _lib.tuning_struct(variant=variant))
    torch.cuda.synchronize()
    assert _lib.device_errors(clear=False) == 0
    assert rel_err(out.cpu().numpy(), expected) <= RTOL_F64
