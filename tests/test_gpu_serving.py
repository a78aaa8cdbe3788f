"""GPU: the serving layer (mpifield_b200.serving).

The batch launch against the single-request kernels, request by request; a graph replay
with a new table; the server's results against each request run alone (the same inputs,
one plain launch), within RTOL_F64 of max |alone| (FP64 atomic order only); and admission
under a budget far below the stream's total memory.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from mpifield_b200 import _lib
from mpifield_b200 import serving as S
from tests.helpers import RTOL_F64, rel_err

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


def _small_work(seed, count=40, markers=(1e3, 3e4)):
    reqs = S.make_stream(count, 1e6, seed, markers=markers)
    assert {r.op for r in reqs} == {"gather", "scatter", "paths"}
    return [(r, S.inputs_of(r, DEV)) for r in reqs]


def _check_against_alone(work):
    for req, b in work:
        alone = S.run_alone(req, S.inputs_of(req, DEV)).cpu().numpy()
        assert rel_err(b["out"].cpu().numpy(), alone) < RTOL_F64, req


def test_the_batch_launch_equals_single_launches():
    work = _small_work(1)
    runner = S.BatchRunner(DEV, capacity=64, tile_markers=256)
    runner.run(work).synchronize()
    _check_against_alone(work)
    assert _lib.device_errors() == 0


def test_a_graph_replays_new_tables_and_resets_its_counter():
    runner = S.BatchRunner(DEV, capacity=64, tile_markers=512, grid=7)
    for seed in (2, 3, 4):
        work = _small_work(seed, count=25)
        runner.run(work).synchronize()
        _check_against_alone(work)
    head = _lib.BatchHeader.from_buffer_copy(runner.header.cpu().numpy().tobytes())
    assert head.next_tile == 0 and head.finished == 0


def test_bounded_and_clamped_grids_in_a_batch():
    # table entries beyond the periodic stream: bounded and clamped axes, dead markers
    rng = np.random.default_rng(5)
    work = []
    for op, kind, degree, geom in [("gather", _lib.SPLINE, 2, (0.0, -1.0, 0.1, 0.2, 20, 11, 2, 0)),
                                   ("scatter", _lib.SPLINE, 3, (0.0, 0.1, 30, 2)),
                                   ("scatter", _lib.LINEAR, 1, (0.0, 0.0, 0.0, 0.5, 0.5, 0.5, 9, 8, 7, 0, 1, 0))]:
        ndim = len(geom) // 4
        ext = tuple(int(n) + (degree - 1 if c == 2 else 0) for n, c in zip(geom[2 * ndim:3 * ndim], geom[3 * ndim:]))
        lo = np.array(geom[:ndim]) - 0.5
        hi = np.array(geom[:ndim]) + np.array(geom[ndim:2 * ndim]) * np.array(geom[2 * ndim:3 * ndim]) + 0.5
        n = 5000
        pos = torch.tensor(rng.uniform(lo[:, None], hi[:, None], (ndim, n)), device=DEV)
        if op == "gather":
            b = {"positions": pos, "field": torch.tensor(rng.normal(size=ext + (3,)), device=DEV),
                 "out": torch.empty((3, n), dtype=torch.float64, device=DEV)}
        else:
            v = rng.uniform(0.5, 1.5, (1, n))
            v[:, ::7] = 0.0
            b = {"positions": pos, "values": torch.tensor(v, device=DEV),
                 "out": torch.zeros(ext + (1,), dtype=torch.float64, device=DEV)}
        work.append((op, kind, degree, geom, b))
    runner = S.BatchRunner(DEV, capacity=8, tile_markers=256)
    lib = _lib.library()
    import ctypes as C
    tiles = 0
    for i, (op, kind, degree, geom, b) in enumerate(work):
        lower, cell, num, code, ndim = _lib.geometry_arrays(geom)
        g = op == "gather"
        n = b["positions"].shape[1]
        st = lib.mpf_batch_request_init(C.byref(runner.entries[i]), 0 if g else 1, kind, degree, ndim,
                                        b["positions"].data_ptr(), n, None if g else b["values"].data_ptr(), n,
                                        n, b["field"].data_ptr() if g else None, b["out"].data_ptr(), n if g else 0,
                                        3 if g else 1, lower, cell, num, code)
        assert st == 0
        runner.entries[i].first_tile = tiles
        tiles += -(-n // 256)
    runner.head.requests, runner.head.tiles, runner.head.tile_markers = len(work), tiles, 256
    runner._launch()
    torch.cuda.synchronize()
    from mpifield_b200 import kernels as K
    for op, kind, degree, geom, b in work:
        if op == "gather":
            ref = torch.empty_like(b["out"])
            K.gather(kind, degree, b["positions"], b["field"], ref, geom)
        else:
            ref = torch.zeros_like(b["out"])
            K.scatter(kind, degree, b["positions"], b["values"], ref, geom)
        assert rel_err(b["out"].cpu().numpy(), ref.cpu().numpy()) < RTOL_F64


def test_served_results_equal_each_request_alone():
    requests = S.make_stream(90, 3000.0, 11, markers=(1e3, 4e5), nodes=(16, 96))
    # the sorted path too: large requests on large 3D fields
    requests += [S.Request(90, "gather", 3, (160, 150, 140), 2, 1_500_000, 0.01, 5),
                 S.Request(91, "scatter", 3, (260, 260, 260), 3, 1_200_000, 0.02, 6)]
    assert requests[-1].sorts and requests[-2].sorts
    server = S.Server(DEV, budget_bytes=3 * 10**9, small_markers=20000, keep_results=True,
                      tile_markers=256, batch_grid=296)
    done = server.run(requests)
    assert sorted(d.req.rid for d in done) == list(range(92))
    assert any(server._small(r) for r in requests) and any(not server._small(r) for r in requests)
    for d in done:
        alone = S.run_alone(d.req, S.inputs_of(d.req, DEV)).cpu().numpy()
        assert rel_err(d.result.cpu().numpy(), alone) < RTOL_F64, d.req
        assert d.latency >= 0.0
    assert server.used_bytes == 0
    assert _lib.device_errors() == 0


def test_admission_holds_to_the_budget():
    requests = S.make_stream(40, 1e5, 12, markers=(1e4, 2e5), nodes=(16, 64))
    budget = int(max(r.nbytes() for r in requests) * 1.5)
    assert sum(r.nbytes() for r in requests) > 4 * budget
    server = S.Server(DEV, budget_bytes=budget, small_markers=30000, tile_markers=256, batch_grid=148)
    done = server.run(requests)
    assert len(done) == 40
    assert server.peak_bytes <= budget
    with pytest.raises(ValueError, match="above the budget"):
        S.Server(DEV, budget_bytes=1000, tile_markers=256, batch_grid=148).run(requests[:1])


def test_the_autotuner_picks_a_measured_candidate():
    best = S.autotune_batch(DEV)
    assert best["tile_markers"] in (128, 256, 512, 1024, 2048)
    assert best["grid"] % torch.cuda.get_device_properties(DEV).multi_processor_count == 0
    assert best["ms"] > 0
