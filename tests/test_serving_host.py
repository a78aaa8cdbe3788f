"""The serving layer's host logic (CPU only): the request stream, memory accounting and
the batch table entries filled by mpf_batch_request_init (no kernel runs here)."""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from mpifield_b200 import _lib
from mpifield_b200 import serving as S


def test_the_stream_draws_the_configured_mix():
    reqs = S.make_stream(4000, 500.0, 7)
    assert [r.rid for r in reqs] == list(range(4000))
    arrivals = np.array([r.arrival for r in reqs])
    assert (np.diff(arrivals) > 0).all()
    # Poisson arrivals: mean gap 1 / rate
    assert abs(np.diff(arrivals).mean() - 1 / 500.0) < 0.1 / 500.0
    assert {r.ndim for r in reqs} == {1, 2, 3}
    assert {r.degree for r in reqs} == {1, 2, 3}
    assert {r.op for r in reqs} == {"gather", "scatter", "paths"}
    assert all(32 <= s <= 256 for r in reqs for s in r.shape)
    assert all(1000 <= r.n <= 10**7 for r in reqs)
    # log-uniform markers: the median is near sqrt(1e3 * 1e7)
    assert 0.5e5 < np.median([r.n for r in reqs]) < 2e5
    assert S.make_stream(50, 500.0, 7) == reqs[:50]


def test_requests_know_their_geometry_and_memory():
    r = S.Request(0, "gather", 2, (64, 32), 2, 1000, 0.0, 1)
    assert r.geometry == (0.0, 0.0, 1 / 64, 1 / 32, 64, 32, 1, 1)
    assert r.nbytes() >= 8 * (64 * 32 * 3 + 1000 * (2 + 3))
    p = S.Request(1, "paths", 3, (40, 40, 40), 3, 5000, 0.0, 1)
    assert p.nbytes() >= 8 * (40**3 * 3 + 5000 * 7)


def test_batch_entries_are_filled_and_checked_on_the_host():
    lib = _lib.library()
    assert lib.mpf_batch_request_size() == C.sizeof(_lib.BatchRequest)
    r = _lib.BatchRequest()
    lower, cell, num, code, ndim = _lib.geometry_arrays((0.0, -1.0, 0.25, 0.5, 4, 5, 1, 0))
    fake = 1 << 20  # never dereferenced on the host
    assert lib.mpf_batch_request_init(C.byref(r), _lib.OP_GATHER, _lib.QUADRATIC, 2, ndim, fake, 0, None, 0, 100,
                                      fake, fake, 0, 3, lower, cell, num, code) == _lib.OK
    assert (r.op, r.kind, r.degree, r.ndim, r.ncomp, r.n) == (0, 1, 2, 2, 3, 100)
    assert (r.pos_stride, r.out_stride) == (100, 100)
    assert list(r.inv)[:2] == [4.0, 2.0] and list(r.ext) == [4, 5, 1] and list(r.code) == [1, 0, 1]
    # the checks of mpf_gather / mpf_scatter
    assert lib.mpf_batch_request_init(C.byref(r), 2, 1, 2, ndim, fake, 0, None, 0, 100, fake, fake, 0, 3,
                                      lower, cell, num, code) == _lib.ERR_ARGUMENT
    assert lib.mpf_batch_request_init(C.byref(r), _lib.OP_GATHER, 1, 3, ndim, fake, 0, None, 0, 100, fake, fake, 0,
                                      3, lower, cell, num, code) == _lib.ERR_ARGUMENT
    assert lib.mpf_batch_request_init(C.byref(r), _lib.OP_SCATTER, 1, 2, ndim, fake + 3, 0, fake, 0, 100, None,
                                      fake, 0, 1, lower, cell, num, code) == _lib.ERR_ALIGNMENT
    assert lib.mpf_batch_request_init(C.byref(r), _lib.OP_GATHER, 1, 2, ndim, fake, 0, None, 0, 100, None, fake, 0,
                                      3, lower, cell, num, code) == _lib.ERR_ARGUMENT
    assert lib.mpf_batch_launch(None, None, 0, 0, None) == _lib.ERR_ARGUMENT


def test_tiles_of_a_batch_are_prefix_sums():
    # the host side of BatchRunner.fill: tile counts per request
    sizes = [1, 256, 257, 1000, 0, 70000]
    tm = 256
    firsts = np.concatenate([[0], np.cumsum([-(-n // tm) for n in sizes])])
    assert firsts.tolist() == [0, 1, 2, 4, 8, 8, 8 + math.ceil(70000 / 256)]
