"""GPU: the host-resident gather/scatter pipeline (mpifield_b200.streaming) equals one call
over all markers: the gathered result bit for bit, the deposit within RTOL_F64."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from mpifield_b200 import _lib
from mpifield_b200 import kernels as K
from mpifield_b200.streaming import HostPipeline
from tests.helpers import RTOL_F64, rel_err

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


@pytest.mark.parametrize("n,chunk,slots", [(100_000, 8192, 2), (70_001, 65536, 3), (1000, 4096, 2)])
def test_the_pipeline_equals_one_call(n, chunk, slots):
    rng = np.random.default_rng(n)
    geom = (0.0, 0.0, 0.0, 1 / 24, 1 / 20, 1 / 16, 24, 20, 16, 1, 0, 1)
    field = torch.tensor(rng.normal(size=(24, 20, 16, 3)), device=DEV)
    pos = torch.tensor(rng.uniform(0, 1, (3, n)), device=DEV)
    w = torch.tensor(rng.uniform(0.5, 1.5, (1, n)), device=DEV)
    E = torch.empty((3, n), dtype=torch.float64, device=DEV)
    rho = torch.zeros((24, 20, 16, 1), dtype=torch.float64, device=DEV)
    K.gather(_lib.QUADRATIC, 2, pos, field, E, geom)
    K.scatter(_lib.QUADRATIC, 2, pos, w, rho, geom)
    hp, hw = pos.cpu().pin_memory(), w.cpu().pin_memory()
    hE = torch.empty((3, n), dtype=torch.float64).pin_memory()
    hD = torch.empty((24, 20, 16, 1), dtype=torch.float64).pin_memory()
    pipe = HostPipeline(DEV, 3, 3, 1, chunk=chunk, slots=slots)
    for _ in range(2):  # the slots are reused across steps
        density = torch.zeros_like(rho)
        pipe.step(_lib.QUADRATIC, 2, hp, hw, field, density, hE, geom, hD)
        torch.cuda.synchronize()
        assert torch.equal(hE, E.cpu())
        assert rel_err(hD.numpy(), rho.cpu().numpy()) < RTOL_F64
