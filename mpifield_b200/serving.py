"""Serving many gather / scatter / path-deposit requests on one GPU with continuous batching.

The reference has no serving layer; this is the added form of the method's use. A
`Server` takes a stream of requests of uneven sizes (dimension, nodes per axis, marker
count, degree, operation), and:

- admits a request when its device memory fits under the HBM budget (its markers, its
  field and its outputs stay resident until it completes), in arrival order;
- runs a large gather or scatter on its markers sorted by cell tile (the sort once at
  admission, the kernels on the sorted copy, a gather's result returned to the request's
  marker order), and a large path deposit as one launch, each on one stream of a pool, so
  that the work of several requests overlaps on the device;
- packs the small gathers, scatters and path deposits that arrived since the last batch into one
  persistent launch (``mpf_batch_launch``) from a per-request tile table, captured once
  in a CUDA graph and replayed with each new table; the tile size and the CTA count come
  from `autotune_batch`;
- polls completions, releases the memory of finished requests and admits waiting ones,
  while the other requests are still on the device.

Every result equals the request's stand-alone result (`run_alone`: one plain launch of
the public kernels) within the kernels' FP64 tolerance (atomic order only). Latency is
completion minus arrival on the host clock; `serve_benchmark` reports requests/s and the
p50/p99 latencies beside the same stream run one plain launch per request.
"""

from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass, field as dc_field

import numpy as np
import torch

from mpifield_b200 import _lib
from mpifield_b200 import kernels as K
from mpifield_b200.sorting import num_tiles, permute, sort_by_tile, sort_workspace_bytes, unpermute

#: gather / scatter weighting of each degree, and the path deposit's edge kind
NODE_KIND = {1: (_lib.LINEAR, 1), 2: (_lib.QUADRATIC, 2), 3: (_lib.SPLINE, 3)}
PATH_KIND = {1: (_lib.LINEAR, 1), 2: (_lib.SPLINE, 2), 3: (_lib.SPLINE, 3)}
OPS = ("gather", "scatter", "paths")
GATHER_COMPONENTS = 3


ALIGN = 256
#: gathers and scatters sort their markers by cell tile when the request has at least
#: this many markers and a field of at least this many bytes (smaller fields stay in L2)
SORT_MARKERS = 1 << 20
SORT_FIELD_BYTES = 64 << 20


@dataclass(frozen=True)
class Request:
    """One request: ``op`` on an ``ndim`` grid of ``shape`` nodes (periodic, on the unit
    cube) with ``n`` markers uniform in the box, B-spline ``degree`` 1-3; its inputs are
    generated from ``seed``; ``arrival`` in seconds from the start of the stream."""

    rid: int
    op: str
    ndim: int
    shape: tuple
    degree: int
    n: int
    arrival: float
    seed: int

    @property
    def geometry(self) -> tuple:
        return ((0.0,) * self.ndim + tuple(1.0 / s for s in self.shape) + tuple(self.shape)
                + (1,) * self.ndim)

    @property
    def sorts(self) -> bool:
        """Whether the request runs on its markers sorted by cell tile."""
        comps = GATHER_COMPONENTS if self.op == "gather" else 1
        return (self.op != "paths" and self.n >= SORT_MARKERS
                and math.prod(self.shape) * comps * 8 >= SORT_FIELD_BYTES)

    def layout(self) -> list[tuple[str, tuple, torch.dtype]]:
        """The request's device buffers, in the order they are carved."""
        f64, nd, n = torch.float64, self.ndim, self.n
        out = [("positions", (nd, n), f64)]
        if self.op == "gather":
            out += [("field", self.shape + (GATHER_COMPONENTS,), f64), ("out", (GATHER_COMPONENTS, n), f64)]
        elif self.op == "scatter":
            out += [("values", (1, n), f64), ("out", self.shape + (1,), f64)]
        else:
            out += [("end", (nd, n), f64), ("values", (n,), f64), ("out", self.shape + (nd,), f64)]
        if self.sorts:
            ntiles = num_tiles(NODE_KIND[self.degree], self.geometry, (8,) * nd)
            out += [("workspace", (sort_workspace_bytes(n, ntiles),), torch.uint8), ("keys", (n,), torch.int32),
                    ("order", (n,), torch.int32), ("tile_start", (ntiles + 2,), torch.int64),
                    ("sorted_positions", (nd, n), f64)]
            out += [("sorted_out", (GATHER_COMPONENTS, n), f64)] if self.op == "gather" else [
                ("sorted_values", (1, n), f64)]
        return out

    def nbytes(self) -> int:
        """Device bytes the request holds while admitted: every buffer of its layout."""
        return sum(_aligned(_size(shape, dt)) for _, shape, dt in self.layout())


_ITEMSIZE = {torch.float64: 8, torch.float32: 4, torch.int64: 8, torch.int32: 4, torch.uint8: 1}


def _size(shape, dtype) -> int:
    return math.prod(shape) * _ITEMSIZE[dtype]


def _aligned(nbytes: int) -> int:
    return max(ALIGN, -(-nbytes // ALIGN) * ALIGN)


def make_stream(count: int, rate: float, seed: int, markers=(1e3, 1e7), nodes=(32, 256)) -> list[Request]:
    """The mixed stream: Poisson arrivals of ``rate`` per second; ndim from {1, 2, 3}; nodes
    per axis log-uniform in ``nodes``; markers log-uniform in ``markers``; degree 1-3;
    operation gather (3 components) / scatter / path deposit, uniformly."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for rid in range(count):
        t += rng.exponential(1.0 / rate)
        ndim = int(rng.integers(1, 4))
        shape = tuple(int(round(math.exp(rng.uniform(math.log(nodes[0]), math.log(nodes[1]))))) for _ in range(ndim))
        n = int(round(math.exp(rng.uniform(math.log(markers[0]), math.log(markers[1])))))
        out.append(Request(rid, OPS[int(rng.integers(0, 3))], ndim, shape, int(rng.integers(1, 4)), n, t,
                           int(rng.integers(0, 2**31))))
    return out


# ------------------------------------------------------------------ request data --

class Arena:
    """One device allocation carved into request buffers: first fit, 256-byte aligned.
    Serving allocates nothing else while it runs (no allocator call that could stall)."""

    def __init__(self, nbytes: int, device):
        self.buffer = torch.empty(int(nbytes), dtype=torch.uint8, device=device)
        self.free = [(0, int(nbytes))]
        self.used = 0
        self.peak = 0

    def alloc(self, nbytes: int) -> tuple[int, int] | None:
        need = _aligned(nbytes)
        for k, (off, size) in enumerate(self.free):
            if size >= need:
                if size == need:
                    del self.free[k]
                else:
                    self.free[k] = (off + need, size - need)
                self.used += need
                self.peak = max(self.peak, self.used)
                return off, need
        return None

    def release(self, block: tuple[int, int]) -> None:
        off, size = block
        self.used -= size
        k = 0
        while k < len(self.free) and self.free[k][0] < off:
            k += 1
        self.free.insert(k, (off, size))
        # coalesce with the neighbours
        if k + 1 < len(self.free) and off + size == self.free[k + 1][0]:
            self.free[k] = (off, size + self.free[k + 1][1])
            del self.free[k + 1]
        if k > 0 and self.free[k - 1][0] + self.free[k - 1][1] == off:
            self.free[k - 1] = (self.free[k - 1][0], self.free[k - 1][1] + self.free[k][1])
            del self.free[k]


class Buffers(dict):
    """A request's buffers by name (views of an arena block, or new tensors)."""


def carve(req: Request, device, arena: Arena | None = None, block=None) -> Buffers:
    """The buffers of ``req``'s layout: views of ``arena`` from ``block``'s offset, or new
    tensors when no arena is given."""
    out = Buffers()
    cursor = block[0] if block is not None else 0
    for name, shape, dtype in req.layout():
        if arena is None:
            out[name] = torch.empty(shape, dtype=dtype, device=device)
            continue
        size = _size(shape, dtype)
        out[name] = arena.buffer[cursor: cursor + size].view(dtype).view(shape)
        cursor += _aligned(size)
    return out


def materialize(req: Request, buffers: Buffers, generator: torch.Generator | None = None) -> Buffers:
    """Fills the request's inputs from its seed (the same every time) and zeroes its
    accumulated output; returns ``buffers``."""
    device = buffers["positions"].device
    g = generator or torch.Generator(device=device)
    g.manual_seed(req.seed)
    buffers["positions"].uniform_(0.0, 1.0, generator=g)
    if req.op == "gather":
        buffers["field"].normal_(0.0, 1.0, generator=g)
    elif req.op == "scatter":
        buffers["values"].uniform_(0.5, 1.5, generator=g)
        buffers["out"].zero_()
    else:
        end = buffers["end"]
        end.uniform_(-0.9, 0.9, generator=g)
        for d, s in enumerate(req.shape):
            end[d].mul_(1.0 / s)
        end.add_(buffers["positions"])
        buffers["values"].uniform_(0.5, 1.5, generator=g)
        buffers["out"].zero_()
    return buffers


def inputs_of(req: Request, device) -> Buffers:
    """A request's inputs in new tensors (for running it alone)."""
    return materialize(req, carve(req, device))


def run_alone(req: Request, b: Buffers) -> torch.Tensor:
    """The request as one plain launch of the public kernel on the current stream, on its
    markers in their own order; returns its output buffer."""
    geom = req.geometry
    if req.op == "gather":
        kind, degree = NODE_KIND[req.degree]
        K.gather(kind, degree, b["positions"], b["field"], b["out"], geom)
    elif req.op == "scatter":
        kind, degree = NODE_KIND[req.degree]
        K.scatter(kind, degree, b["positions"], b["values"], b["out"], geom)
    else:
        kind, degree = PATH_KIND[req.degree]
        K.deposit_paths(kind, degree, b["positions"], b["end"], b["values"], b["out"], geom)
    return b["out"]


def run_sorted(req: Request, b: Buffers) -> torch.Tensor:
    """A gather or scatter on its markers sorted by cell tile (8 cells a side), the sort's
    buffers from the request's own, the kernels given the sort's tile starts (the tile
    gather and scatter); a gather's result goes back to the marker order."""
    kind, degree = NODE_KIND[req.degree]
    geom = req.geometry
    scratch = iter([b["workspace"], b["keys"], b["order"], b["tile_start"]])
    tiles = sort_by_tile(b["positions"], (kind, degree), geom, (8,) * req.ndim, within=True,
                         alloc=lambda shape, dt: next(scratch))
    pos = permute(b["positions"], tiles.order, out=b["sorted_positions"])
    if req.op == "gather":
        K.gather(kind, degree, pos, b["field"], b["sorted_out"], geom, order=tiles)
        unpermute(b["sorted_out"], tiles.order, out=b["out"])
    else:
        K.scatter(kind, degree, pos, permute(b["values"], tiles.order, out=b["sorted_values"]), b["out"], geom,
                  order=tiles)
    return b["out"]


def run(req: Request, b: Buffers) -> torch.Tensor:
    return run_sorted(req, b) if req.sorts else run_alone(req, b)


# ------------------------------------------------------------------------ batches --

class BatchRunner:
    """Small gathers, scatters and path deposits in one launch from a device table, replayed from a CUDA
    graph: the pinned host table and header are rewritten, then the graph copies them to
    the device and launches ``mpf_batch_launch``."""

    def __init__(self, device, capacity: int = 1024, tile_markers: int = 256, grid: int = 0):
        self.device = torch.device(device)
        self.capacity = capacity
        self.tile_markers = tile_markers
        self.grid = grid
        size = C.sizeof(_lib.BatchRequest)
        if size != _lib.library().mpf_batch_request_size():
            raise RuntimeError("mpf_batch_request layout differs between the library and the binding")
        self.host_table = torch.empty(capacity * size, dtype=torch.uint8, pin_memory=True)
        self.host_header = torch.zeros(C.sizeof(_lib.BatchHeader), dtype=torch.uint8, pin_memory=True)
        self.table = torch.empty(capacity * size, dtype=torch.uint8, device=self.device)
        self.header = torch.zeros(C.sizeof(_lib.BatchHeader), dtype=torch.uint8, device=self.device)
        self.entries = (_lib.BatchRequest * capacity).from_address(self.host_table.data_ptr())
        self.head = _lib.BatchHeader.from_address(self.host_header.data_ptr())
        self.stream = torch.cuda.Stream(self.device)
        self.graph = None
        self.done = None  # event of the launch in flight

    def _launch(self) -> None:
        self.table.copy_(self.host_table, non_blocking=True)
        self.header.copy_(self.host_header, non_blocking=True)
        status = _lib.library().mpf_batch_launch(self.table.data_ptr(), self.header.data_ptr(), self.grid,
                                                 256, torch.cuda.current_stream(self.device).cuda_stream)
        _lib.check(status, "batch_launch")

    def _capture(self) -> None:
        self.head.requests = 0
        self.head.tiles = 0
        self.head.tile_markers = self.tile_markers
        with torch.cuda.stream(self.stream):
            self._launch()  # warm up outside the capture
        self.stream.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=self.stream):
            self._launch()
        self.stream.synchronize()

    def busy(self) -> bool:
        return self.done is not None and not self.done.query()

    def fill(self, work: list) -> None:
        """Writes the table for ``work``: (request, buffers) pairs of small requests."""
        tiles = 0
        lib = _lib.library()
        for i, (req, b) in enumerate(work):
            lower, cell, num, code, ndim = _lib.geometry_arrays(req.geometry)
            if req.op == "paths":  # starts, ends (rows n apart), charges, the edge field
                kind, degree = PATH_KIND[req.degree]
                status = lib.mpf_batch_request_init(
                    C.byref(self.entries[i]), _lib.OP_PATHS, kind, degree, ndim, b["positions"].data_ptr(), req.n,
                    b["values"].data_ptr(), req.n, req.n, b["end"].data_ptr(), b["out"].data_ptr(), req.n, ndim,
                    lower, cell, num, code)
                _lib.check(status, "batch_request_init")
                self.entries[i].first_tile = tiles
                tiles += -(-req.n // self.tile_markers)
                continue
            kind, degree = NODE_KIND[req.degree]
            gather = req.op == "gather"
            status = lib.mpf_batch_request_init(
                C.byref(self.entries[i]), _lib.OP_GATHER if gather else _lib.OP_SCATTER, kind, degree, ndim,
                b["positions"].data_ptr(), req.n, None if gather else b["values"].data_ptr(), req.n, req.n,
                b["field"].data_ptr() if gather else None, b["out"].data_ptr(), req.n if gather else 0,
                GATHER_COMPONENTS if gather else 1, lower, cell, num, code)
            _lib.check(status, "batch_request_init")
            self.entries[i].first_tile = tiles
            tiles += -(-req.n // self.tile_markers)
        self.head.requests = len(work)
        self.head.tiles = tiles
        self.head.tile_markers = self.tile_markers
        self.head.next_tile = 0
        self.head.finished = 0

    def run(self, work: list, wait_for: torch.cuda.Event | None = None) -> torch.cuda.Event:
        """Launches the batch of ``work`` (at most ``capacity`` requests) on the batch stream."""
        if len(work) > self.capacity:
            raise ValueError(f"a batch holds at most {self.capacity} requests, got {len(work)}")
        if self.graph is None:
            self._capture()
        if self.done is not None:
            self.done.synchronize()  # the previous replay has read the host table
        self.fill(work)
        if wait_for is not None:
            self.stream.wait_event(wait_for)
        with torch.cuda.stream(self.stream):
            self.graph.replay()
            self.done = torch.cuda.Event()
            self.done.record(self.stream)
        return self.done


_TUNED: dict = {}


def autotune_batch(device, reps: int = 3, seed: int = 3) -> dict:
    """The batch launch's tile size (markers per tile) and CTA count, measured on a
    synthetic mix of small requests (gathers, scatters and path deposits of 1-3 dimensions,
    degrees 1-3, 1e3-1e5 markers); the fastest pair is kept for the process."""
    key = str(torch.device(device))
    if key in _TUNED:
        return _TUNED[key]
    dev = torch.device(device)
    reqs = make_stream(48, 1e6, seed, markers=(1e3, 1e5))
    work = [(r, inputs_of(r, dev)) for r in reqs]
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    best = None
    for tile in (128, 256, 512, 1024, 2048):
        for per_sm in (1, 2):
            runner = BatchRunner(dev, capacity=64, tile_markers=tile, grid=sms * per_sm)
            runner.run(work).synchronize()
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(runner.stream)
            for _ in range(reps):
                runner.run(work)
            stop.record(runner.stream)
            stop.synchronize()
            ms = start.elapsed_time(stop) / reps
            if best is None or ms < best["ms"]:
                best = {"tile_markers": tile, "grid": sms * per_sm, "ms": ms}
    _TUNED[key] = best
    return best


# ------------------------------------------------------------------------- server --

@dataclass
class Done:
    req: Request
    latency: float
    result: torch.Tensor | None


@dataclass
class _Job:
    req: Request
    block: tuple
    buffers: Buffers
    event: torch.cuda.Event | None = None


@dataclass
class Server:
    """Continuous batching under an HBM budget (see the module docstring). The budget is
    taken as one arena when the server starts."""

    device: object = "cuda"
    budget_bytes: int = 120 * 10**9
    small_markers: int = 65536
    streams: int = 4
    batch_capacity: int = 512
    tile_markers: int | None = None
    batch_grid: int | None = None
    keep_results: bool = False
    _stats: dict = dc_field(default_factory=dict)

    def __post_init__(self):
        self.device = torch.device(self.device)
        if self.tile_markers is None or self.batch_grid is None:
            tuned = autotune_batch(self.device)
            self.tile_markers = self.tile_markers or tuned["tile_markers"]
            self.batch_grid = self.batch_grid or tuned["grid"]
        self.pool = [torch.cuda.Stream(self.device) for _ in range(self.streams)]
        self.generators = {id(s): torch.Generator(device=self.device) for s in self.pool}
        self.batch = BatchRunner(self.device, self.batch_capacity, self.tile_markers, self.batch_grid)
        self.batch_generator = torch.Generator(device=self.device)
        self.batch._capture()
        self.arena = Arena(self.budget_bytes, self.device)
        self._next = 0

    @property
    def used_bytes(self) -> int:
        return self.arena.used

    @property
    def peak_bytes(self) -> int:
        return self.arena.peak

    def _small(self, req: Request) -> bool:
        return req.n <= self.small_markers

    def _admit(self, req: Request) -> _Job | None:
        block = self.arena.alloc(req.nbytes())
        if block is None:
            return None
        b = carve(req, self.device, self.arena, block)
        if self._small(req):
            with torch.cuda.stream(self.batch.stream):
                materialize(req, b, self.batch_generator)
            return _Job(req, block, b)
        stream = self.pool[self._next % len(self.pool)]
        self._next += 1
        with torch.cuda.stream(stream):
            materialize(req, b, self.generators[id(stream)])
            run(req, b)
            event = torch.cuda.Event()
            event.record(stream)
        return _Job(req, block, b, event)

    def run(self, requests: list[Request], clock=time.perf_counter) -> list[Done]:
        """Serves ``requests`` in real time (by arrival); returns them as they complete."""
        pending = sorted(requests, key=lambda r: r.arrival)
        for r in pending:
            if r.nbytes() > self.budget_bytes:
                raise ValueError(f"request {r.rid} needs {r.nbytes()} bytes, above the budget {self.budget_bytes}")
        waiting: list[Request] = []
        flying: list[_Job] = []
        batch_jobs: list[_Job] = []   # admitted small requests not yet launched
        in_batch: list[_Job] = []     # the batch on the device
        done: list[Done] = []
        t0 = clock()
        i = 0
        while len(done) < len(requests):
            now = clock() - t0
            while i < len(pending) and pending[i].arrival <= now:
                waiting.append(pending[i])
                i += 1
            # admission in arrival order, while the arena has room
            while waiting:
                job = self._admit(waiting[0])
                if job is None:
                    break
                waiting.pop(0)
                (batch_jobs if job.event is None else flying).append(job)
            # the next batch, once the previous one is off the device
            if batch_jobs and not in_batch:
                take, batch_jobs = batch_jobs[: self.batch_capacity], batch_jobs[self.batch_capacity:]
                event = self.batch.run([(j.req, j.buffers) for j in take])
                for j in take:
                    j.event = event
                in_batch = take
            # completions
            finished = [j for j in flying if j.event.query()]
            if in_batch and in_batch[0].event.query():
                finished += in_batch
                in_batch = []
            if finished:
                stamp = clock() - t0
                for j in finished:
                    if j in flying:
                        flying.remove(j)
                    result = j.buffers["out"].clone() if self.keep_results else None
                    done.append(Done(j.req, stamp - j.req.arrival, result))
                if self.keep_results:
                    # the copies run on this thread's stream: they are done before the memory
                    # returns to the arena (a request admitted next writes it from another stream)
                    torch.cuda.current_stream(self.device).synchronize()
                for j in finished:
                    self.arena.release(j.block)
            elif not waiting and i < len(pending) and not flying and not in_batch and not batch_jobs:
                # idle until the next arrival
                time.sleep(max(0.0, min(pending[i].arrival - (clock() - t0), 0.001)))
        self._stats = {"makespan": clock() - t0}
        return done


def run_one_by_one(requests: list[Request], device, clock=time.perf_counter, keep_results=False) -> list[Done]:
    """The baseline: each request in arrival order as one plain launch on its markers in
    their own order, waited for, its buffers new tensors."""
    device = torch.device(device)
    done = []
    g = torch.Generator(device=device)
    t0 = clock()
    for req in sorted(requests, key=lambda r: r.arrival):
        while clock() - t0 < req.arrival:
            time.sleep(max(0.0, min(req.arrival - (clock() - t0), 0.001)))
        b = materialize(req, carve(req, device), g)
        out = run_alone(req, b)
        torch.cuda.synchronize(device)
        done.append(Done(req, clock() - t0 - req.arrival, out if keep_results else None))
        del b, out
    return done


def summarize(done: list[Done], makespan: float) -> dict:
    lat = np.array([d.latency for d in done])
    return {"requests": len(done), "requests_per_s": len(done) / makespan, "makespan_s": makespan,
            "p50_ms": float(np.percentile(lat, 50) * 1000.0), "p99_ms": float(np.percentile(lat, 99) * 1000.0)}


def serve_benchmark(count: int, rate: float, seed: int, device="cuda", budget_bytes: int = 120 * 10**9,
                    markers=(1e3, 1e7)) -> dict:
    """The mixed stream served with continuous batching, and one plain launch per request;
    both warmed up on a short stream of the same mix first."""
    requests = make_stream(count, rate, seed, markers=markers)
    warm = make_stream(30, rate, seed + 1, markers=markers)
    server = Server(device, budget_bytes=budget_bytes)
    server.run(warm)
    run_one_by_one(warm, device)
    torch.cuda.synchronize()
    served = server.run(requests)
    ours = summarize(served, server._stats["makespan"])
    peak = server.peak_bytes
    del server
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain = run_one_by_one(requests, device)
    base = summarize(plain, time.perf_counter() - t0)
    return {"served": ours, "one_launch_per_request": base, "rate_per_s": rate, "seed": seed,
            "budget_bytes": budget_bytes, "peak_admitted_bytes": peak,
            "batch": {"tile_markers": _TUNED.get(str(torch.device(device)), {}).get("tile_markers"),
                      "grid": _TUNED.get(str(torch.device(device)), {}).get("grid"),
                      "small_markers": 65536, "streams": 4}}
