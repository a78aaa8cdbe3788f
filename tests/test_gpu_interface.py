"""The kernels on arrays of other producers, on the caller's stream, and the reference's
special LINEAR signatures, on the GPU.

- A CuPy-like array (``__cuda_array_interface__`` version 3 naming its producer's
  stream) is used in place, with no copy, and the call runs on the stream it names.
- ``__dlpack__`` producers are taken as well.
- The signatures mpifield's LINEAR weighting gives its kernels (src/mpifield/
  weighting.py:259-330): the 1D deposit one component at a time, ``(N,)`` markers into an
  ``(nx,)`` column of the field with the launch keywords ``shared_mem`` and ``n_threads``,
  and the 3D kernels with the grid as rows ``(nx * ny * nz, ncomp)``; all against the
  oracle within 1e-12.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import mpifield_b200 as mf
from mpifield_b200 import _lib
from oracle import oracle as O
from tests.helpers import RTOL_F64, rel_err

pytestmark = pytest.mark.gpu


class InterfaceArray:
    """A device array known only through ``__cuda_array_interface__`` (as CuPy's)."""

    def __init__(self, tensor: torch.Tensor, stream: int | None):
        self.t, self.stream = tensor, stream

    @property
    def __cuda_array_interface__(self):
        t = self.t
        return {"shape": tuple(t.shape), "typestr": "<f8", "data": (t.data_ptr(), False),
                "strides": tuple(s * t.element_size() for s in t.stride()), "version": 3, "stream": self.stream}


class _Streams:
    """Forwards to the real library and records the stream of every gather/scatter."""

    def __init__(self, real):
        self.real, self.seen = real, []

    def __getattr__(self, name):
        fn = getattr(self.real, name)
        if name not in ("mpf_gather", "mpf_scatter"):
            return fn

        def call(*args):
            self.seen.append(args[-1])
            return fn(*args)

        return call


def test_interface_arrays_are_used_in_place_on_their_stream(monkeypatch):
    rng = np.random.default_rng(1)
    geom = (0.0, 0.0, 0.0, 0.1, 0.1, 0.1, 12, 10, 8, 1, 0, 1)
    pos = rng.uniform(-0.2, 1.3, (3, 5000))
    field = rng.normal(size=(12, 10, 8, 3))
    side = torch.cuda.Stream()
    spy = _Streams(_lib.library())
    monkeypatch.setattr(_lib, "library", lambda: spy)
    p = torch.tensor(pos, device="cuda")
    f = torch.tensor(field, device="cuda")
    out = torch.zeros((3, 5000), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    mf.KERNELS["gather_quadratic_3d"](InterfaceArray(p, side.cuda_stream), InterfaceArray(f, side.cuda_stream),
                                      InterfaceArray(out, side.cuda_stream), *geom)
    side.synchronize()
    assert spy.seen == [side.cuda_stream]
    assert rel_err(out.cpu().numpy(), O.gather("quadratic", 2, pos, field, geom)) <= RTOL_F64
    # an interface without a stream runs on the legacy default stream; use_stream overrides both
    dens = torch.zeros((12, 10, 8, 1), dtype=torch.float64, device="cuda")
    w = torch.ones((1, 5000), dtype=torch.float64, device="cuda")
    mf.KERNELS["scatter_quadratic_3d"](InterfaceArray(p, None), InterfaceArray(w, None), InterfaceArray(dens, None),
                                       *geom)
    with mf.use_stream(side):
        mf.KERNELS["scatter_quadratic_3d"](InterfaceArray(p, None), InterfaceArray(w, None),
                                           InterfaceArray(dens, None), *geom)
    torch.cuda.synchronize()
    assert spy.seen[1:] == [0, side.cuda_stream]
    expected = O.scatter("quadratic", 2, pos, np.ones((1, 5000)), np.zeros((12, 10, 8, 1)), geom)
    assert rel_err(dens.cpu().numpy(), 2 * expected) <= RTOL_F64


def test_dlpack_producers_are_taken():
    rng = np.random.default_rng(2)
    geom = (0.0, 0.0, 0.2, 0.2, 9, 7, 1, 1)
    pos = rng.uniform(0.0, 1.8, (2, 3000))
    field = rng.normal(size=(9, 7, 2))

    class Capsule:  # only __dlpack__ / __dlpack_device__
        def __init__(self, t):
            self.t = t

        def __dlpack__(self, stream=None):
            return self.t.__dlpack__(stream=stream)

        def __dlpack_device__(self):
            return self.t.__dlpack_device__()

    out = torch.zeros((2, 3000), dtype=torch.float64, device="cuda")
    mf.KERNELS["gather_spline_2d"](Capsule(torch.tensor(pos, device="cuda")), Capsule(torch.tensor(field, device="cuda")),
                                   Capsule(out), *geom, 3)
    assert rel_err(out.cpu().numpy(), O.gather("spline", 3, pos, field, geom)) <= RTOL_F64


@pytest.mark.parametrize("periodic", [0, 1])
def test_linear_1d_one_component_at_a_time(periodic):
    # src/mpifield/weighting.py:259-295: scatter_linear_1d(positions[0], values[c], field[:, c], ...)
    rng = np.random.default_rng(3 + periodic)
    nx, n, ncomp = 40, 20000, 3
    geom = (0.5, 0.05, nx, periodic)
    pos = rng.uniform(0.4, 0.5 + 0.05 * nx, (1, n))
    values = rng.uniform(0.5, 1.5, (ncomp, n))
    field = torch.zeros((nx, ncomp), dtype=torch.float64, device="cuda")
    p = torch.tensor(pos, device="cuda")
    v = torch.tensor(values, device="cuda")
    for c in range(ncomp):
        mf.KERNELS["scatter_linear_1d"](p[0], v[c], field[:, c], *geom, shared_mem=8 * nx, n_threads=(n + 3) // 4)
    expected = O.scatter("linear", 1, pos, values, np.zeros((nx, ncomp)), geom)
    assert rel_err(field.cpu().numpy(), expected) <= RTOL_F64
    out = torch.zeros((ncomp, n), dtype=torch.float64, device="cuda")
    mf.KERNELS["gather_linear_1d"](p, field, out, *geom)
    assert rel_err(out.cpu().numpy(), O.gather("linear", 1, pos, expected, geom)) <= RTOL_F64
    with pytest.raises(TypeError, match="unexpected keyword"):
        mf.KERNELS["scatter_linear_1d"](p[0], v[0], field[:, 0], *geom, blocks=3)


def test_linear_3d_grid_as_rows():
    # src/mpifield/weighting.py:298-330: the 3D kernels take the grid as (nx * ny * nz, ncomp)
    rng = np.random.default_rng(5)
    shape, ncomp, n = (10, 9, 8), 2, 30000
    geom = (0.0, 0.0, 0.0, 0.1, 0.1, 0.1, *shape, 1, 0, 1)
    pos = rng.uniform(-0.1, 1.0, (3, n))
    values = rng.uniform(0.5, 1.5, (ncomp, n))
    rows = torch.zeros((int(np.prod(shape)), ncomp), dtype=torch.float64, device="cuda")
    p = torch.tensor(pos, device="cuda")
    mf.KERNELS["scatter_linear_3d"](p, torch.tensor(values, device="cuda"), rows, *geom)
    expected = O.scatter("linear", 1, pos, values, np.zeros(shape + (ncomp,)), geom)
    assert rel_err(rows.cpu().numpy().reshape(shape + (ncomp,)), expected) <= RTOL_F64
    out = torch.zeros((ncomp, n), dtype=torch.float64, device="cuda")
    mf.KERNELS["gather_linear_3d"](p, rows, out, *geom)
    assert rel_err(out.cpu().numpy(), O.gather("linear", 1, pos, expected, geom)) <= RTOL_F64
