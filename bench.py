#!/usr/bin/env python
"""The particle-grid hot path on B200: markers/s of the 3D quadratic gather + scatter.

Workload (the configuration the metric is quoted on): a 256^3 periodic grid on the unit
cube, QUADRATIC weights, float64; a 3-component field, each component a sum of 8
Fourier modes cos(2 pi k.x + phi) with integer wave-vector components k_d in 1..8 and
unit amplitude (seeded); N = 2^26 markers, 80% uniform in the cube and 20% in a
Gaussian beam (sigma 0.05, centre 0.5, wrapped into the cube), in random order; marker
weights uniform in [0.5, 1.5]. All inputs are synthetic (there is no dataset).

The marker store is kept in cell-tile order, as particle-in-cell codes keep their
markers (picnic's sort_by_cell): the markers are sorted once before timing (tiles of
4 x 4 x 64 cells, cells in a tile in row-major order: mpifield_b200.sort_by_tile(within=True)).
One step = gather E (3, N) from the field at the markers + scatter the weights into a
zeroed 1-component density. `value` is N / step time with every input resident in HBM.
`full_step` times the whole path from markers in random order instead: tile sort,
permute positions and weights, gather, scatter, and E returned to the markers' own
order. `e2e` is the step through the public API with host buffers: every step the
pinned-host-to-device copy of positions and weights and the device-to-host copy of E
and the density. The positions alone (1.6 GB) exceed the 126 MB L2, so no flush is
needed between steps.

With --impl reference the same metric is measured on the reference's CPU
implementation (the OpenMP restatement of its Pyccel kernels, oracle/cpu_baseline.c,
with all host threads) on a bounded sample of the workload per step.

Under torchrun (N GPUs) every rank runs the same workload on its own GPU (replicas: the
hot path has no cross-GPU step on one grid); the time is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "markers/s: 3D quadratic gather/scatter"
GRID = 256
TILE = (4, 4, 64)
PEAK_FALLBACK_GBS = 6650.0


def parse() -> argparse.Namespace:
    p = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=40)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("ours", "reference"), default="ours")
    p.add_argument("--markers", type=int, default=1 << 26)
    p.add_argument("--grid", type=int, default=256, help="nodes per axis (smaller grids for profiling)")
    p.add_argument("--dtype", choices=("f64", "f32"), default="f64")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-ref-cuda", action="store_true")
    p.add_argument("--no-extras", action="store_true", help="skip the other configurations' measurements")
    p.add_argument("--serve-requests", type=int, default=10000, help="requests of the serving stream (0: skip)")
    p.add_argument("--paths-only", type=int, default=0, metavar="N",
                   help="measure only the path deposits, at N paths on 128^3 (a profiling case)")
    p.add_argument("--steady-only", action="store_true",
                   help="measure only the steady step (push, re-sort, permute, gather, scatter; a profiling case)")
    p.add_argument("--autograd-only", action="store_true",
                   help="measure only the differentiation step (512^2 cubic, 2^22 markers; a profiling case)")
    p.add_argument("--serve-rate", type=float, default=20000.0,
                   help="Poisson arrival rate of the stream, per s (the default outruns both arms: capacity)")
    p.add_argument("--serve-latency-rate", type=float, default=1500.0,
                   help="a second, sustainable arrival rate at which latencies are reported (0: skip)")
    return p.parse_args()


# ------------------------------------------------------------------ workload --


def geometry() -> tuple:
    h = 1.0 / GRID
    return (0.0, 0.0, 0.0, h, h, h, GRID, GRID, GRID, 1, 1, 1)


def make_field(device, dtype, seed: int = 0) -> torch.Tensor:
    """(256, 256, 256, 3): per component a sum of 8 unit Fourier modes, k_d in 1..8."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    x = torch.arange(GRID, dtype=torch.float64, device=device) / GRID
    field = torch.zeros((GRID, GRID, GRID, 3), dtype=torch.float64, device=device)
    for c in range(3):
        for _ in range(8):
            k = torch.randint(1, 9, (3,), generator=g).tolist()
            phi = float(torch.rand((), generator=g, dtype=torch.float64)) * 2 * np.pi
            phase = 2 * np.pi * (k[0] * x[:, None, None] + k[1] * x[None, :, None] + k[2] * x[None, None, :])
            field[..., c] += torch.cos(phase + phi)
    return field.to(dtype)


def make_markers(n: int, device, dtype, seed: int = 1) -> tuple[torch.Tensor, torch.Tensor]:
    """Positions (3, n) -- 80% uniform, 20% beam N(0.5, 0.05) wrapped -- and weights (1, n)."""
    g = torch.Generator(device=device).manual_seed(seed)
    pos = torch.rand((3, n), generator=g, dtype=torch.float64, device=device)
    beam = torch.rand(n, generator=g, dtype=torch.float64, device=device) < 0.2
    gauss = 0.5 + 0.05 * torch.randn((3, n), generator=g, dtype=torch.float64, device=device)
    pos = torch.where(beam[None, :], torch.remainder(gauss, 1.0), pos)
    weights = 0.5 + torch.rand((1, n), generator=g, dtype=torch.float64, device=device)
    return pos.to(dtype).contiguous(), weights.to(dtype).contiguous()


def algorithmic_bytes(n: int, itemsize: int) -> dict[str, int]:
    """Compulsory traffic: gather N (3 pos + 3 out) + field; scatter N (3 pos + 1 w) + 2 x density."""
    nodes = GRID ** 3
    return {
        "gather": n * 6 * itemsize + nodes * 3 * itemsize,
        "scatter": n * 4 * itemsize + nodes * 2 * itemsize,
    }


# -------------------------------------------------------------- clock samples --


class ClockSampler:
    """nvidia-smi clock and throttle samples of one GPU during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int) -> None:
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "20",
                 "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the timed region starts once the sampler is live (its first line is out)
            deadline = time.perf_counter() + 3.0
            while not self.lines and self.proc.poll() is None and time.perf_counter() < deadline:
                time.sleep(0.005)
            self.skip = len(self.lines)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self) -> None:
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc) -> None:
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict | None:
        rows = [line.split(", ") for line in self.lines[getattr(self, "skip", 0):] if line.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        maxsm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(maxsm) if maxsm else None,
                "reasons": reasons, "samples": len(rows)}


# -------------------------------------------------------------------- helpers --


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() and args.impl == "ours" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return world, rank, local


def max_over_ranks(value: float, world: int, device) -> float:
    if world == 1:
        return value
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def read_peak() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        peaks = json.loads(path.read_text())
        return float(peaks["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return PEAK_FALLBACK_GBS, "fallback"


def read_traffic(key: str) -> int | None:
    """DRAM bytes per launch of a kernel from the committed ncu summary, if present."""
    path = ROOT / "profiles" / "traffic.txt"
    try:
        for line in path.read_text().splitlines():
            parts = line.split()
            if len(parts) >= 2 and parts[0] == key:
                return int(float(parts[1]))
    except OSError:
        pass
    return None


# ----------------------------------------------------------------- our step --


class Step:
    """The hot path on one GPU: sort, permute, gather, scatter, unpermute."""

    def __init__(self, n: int, device, dtype) -> None:
        import mpifield_b200 as mf
        from mpifield_b200 import _lib

        self.mf, self.lib = mf, _lib
        self.n, self.device, self.dtype = n, device, dtype
        self.geom = geometry()
        self.field = make_field(device, dtype)
        self.density = torch.zeros((GRID, GRID, GRID, 1), dtype=dtype, device=device)
        self.E = torch.empty((3, n), dtype=dtype, device=device)
        self.E_out = torch.empty((3, n), dtype=dtype, device=device)
        self.kernels = (mf.KERNELS["gather_quadratic_3d"], mf.KERNELS["scatter_quadratic_3d"])
        self.order = None

    def sort(self, pos, w):
        """Sorts the markers by cell tile; the store keeps the order (its tile starts)."""
        t = self.mf.sort_by_tile(pos, self.mf.QUADRATIC, self.geom, TILE, within=True)
        self.order = t
        return t, self.mf.permute(pos, t.order), self.mf.permute(w, t.order)

    def gather_scatter(self, pos, w, events=None):
        """Gather E and scatter the weights on the sorted store; both take the store's tile
        starts (mpf_gather_tiles, mpf_scatter_tiles)."""
        if events is not None:
            events[0].record()
        self.mf.kernels.gather(self.lib.QUADRATIC, 2, pos, self.field, self.E, self.geom, order=self.order)
        if events is not None:
            events[1].record()
        self.density.zero_()
        self.mf.kernels.scatter(self.lib.QUADRATIC, 2, pos, w, self.density, self.geom, order=self.order)
        if events is not None:
            events[2].record()

    def full(self, pos, w, events=None):
        t, ps, ws = self.sort(pos, w)
        self.gather_scatter(ps, ws, events)
        self.mf.unpermute(self.E, t.order, out=self.E_out)


def time_loop(fn, steps: int, warmup: int, world: int, device) -> float:
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(steps):
        fn()
    stop.record()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    return max_over_ranks(start.elapsed_time(stop) / 1000.0, world, device)


def ref_cuda_time(pos, w, field, density, E, steps: int) -> dict | None:
    """The reference's CUDA gather_quadratic_3d + scatter_quadratic_3d (one thread per
    marker, block 256), compiled for sm_100a from the reference sources (oracle/_ref)."""
    import ctypes as C

    path = ROOT / "oracle" / "_ref" / "libref_cuda.so"
    if not path.exists():
        return None
    lib = C.CDLL(str(path))
    n = pos.shape[1]
    stream = torch.cuda.current_stream().cuda_stream

    def view(t):
        shape = (C.c_longlong * t.dim())(*t.shape)
        strides = (C.c_longlong * t.dim())(*t.stride())
        return [C.c_void_p(t.data_ptr()), shape, strides]

    h = 1.0 / GRID
    scal = [C.c_double(0.0)] * 3 + [C.c_double(h)] * 3 + [C.c_int(GRID)] * 3 + [C.c_int(1)] * 3
    head = [C.c_longlong(n), C.c_int(256), C.c_int(0), C.c_void_p(stream)]
    g_args = head + view(pos) + view(field) + view(E) + scal
    s_args = head + view(pos) + view(w) + view(density) + scal

    def step():
        lib.refcuda_gather_quadratic_3d(*g_args)
        density.zero_()
        lib.refcuda_scatter_quadratic_3d(*s_args)

    step()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    g_ms, s_ms = 0.0, 0.0
    for _ in range(steps):
        ev[0].record()
        lib.refcuda_gather_quadratic_3d(*g_args)
        ev[1].record()
        density.zero_()
        lib.refcuda_scatter_quadratic_3d(*s_args)
        ev[2].record()
        torch.cuda.synchronize()
        g_ms += ev[0].elapsed_time(ev[1])
        s_ms += ev[1].elapsed_time(ev[2])
    t = (g_ms + s_ms) / steps / 1000.0
    return {"value": n / t, "unit": "markers/s", "gather_ms": g_ms / steps, "scatter_ms": s_ms / steps,
            "marker_order": "random", "kernels": "reference gather_quadratic_3d + scatter_quadratic_3d, sm_100a"}


def _ref_cuda_lib():
    """The reference's CUDA kernels compiled for sm_100a from its sources (oracle/_ref), or None."""
    import ctypes as C

    path = ROOT / "oracle" / "_ref" / "libref_cuda.so"
    return C.CDLL(str(path)) if path.exists() else None


def _ref_call(lib, name: str, n_threads: int, arrays, doubles, ints) -> None:
    """Launch reference kernel ``name`` (one thread per marker or path, block 256) on torch's
    current stream: its array views (data, shape, strides in elements), then its double and
    int arguments, in the order of its signature."""
    import ctypes as C

    args = [C.c_longlong(n_threads), C.c_int(256), C.c_int(0), C.c_void_p(torch.cuda.current_stream().cuda_stream)]
    keep = []
    for t in arrays:
        shape = (C.c_longlong * t.dim())(*t.shape)
        strides = (C.c_longlong * t.dim())(*t.stride())
        keep += [shape, strides]
        args += [C.c_void_p(t.data_ptr()), shape, strides]
    args += [C.c_double(float(v)) for v in doubles] + [C.c_int(int(v)) for v in ints]
    status = getattr(lib, f"refcuda_{name}")(*args)
    if status != 0:
        raise RuntimeError(f"reference kernel {name} failed with CUDA error {status}")


def _event_stats(fn, reps: int) -> tuple[float, float]:
    """Mean and best (minimum) milliseconds of ``fn`` over ``reps`` timed calls after one
    warm-up call, each timed with CUDA events on the current stream (best of N as the
    reference's examples/12_kernel_backends.py:27-34 reports)."""
    fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    return sum(times) / len(times), min(times)


def measure_steady(step, ps, ws, reps: int) -> dict:
    """The steady state of a particle-in-cell store kept sorted across steps: every step
    pushes the markers (a fixed displacement of up to 0.3 cell per axis, per rank), re-sorts
    the store against its previous sorted keys (mpf_resort_by_tile: only the markers whose
    cell changed are sorted), permutes positions and weights, and gathers and scatters on
    the new order. The last step's order is checked against a full sort of the store."""
    mf = step.mf
    saved = step.order
    g = torch.Generator(device=ps.device).manual_seed(9)
    disp = (torch.rand(ps.shape, generator=g, device=ps.device, dtype=ps.dtype) * 0.6 - 0.3) / GRID
    pos, w = ps.clone(), ws.clone()
    t = mf.resort_by_tile(pos, mf.QUADRATIC, step.geom, TILE, within=True)
    pos, w = mf.permute(pos, t.order), mf.permute(w, t.order)
    spare = [torch.empty_like(pos), torch.empty_like(w)]
    state = {"pos": pos, "w": w, "t": t}
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]

    def one(events=None):
        pos, w = state["pos"], state["w"]
        pos.add_(disp).remainder_(1.0)
        if events:
            events[0].record()
        t = mf.resort_by_tile(pos, mf.QUADRATIC, step.geom, TILE, within=True, previous=state["t"])
        mf.permute(pos, t.order, out=spare[0])
        mf.permute(w, t.order, out=spare[1])
        if events:
            events[1].record()
        state["pos"], spare[0] = spare[0], pos
        state["w"], spare[1] = spare[1], w
        state["t"] = t
        step.order = t
        step.gather_scatter(state["pos"], state["w"])
        if events:
            events[2].record()

    ms = _event_ms(one, reps)
    resort = []
    torch.cuda.nvtx.range_push("steady")
    for _ in range(max(2, reps // 4)):
        one(ev)
        torch.cuda.synchronize()
        resort.append(ev[0].elapsed_time(ev[1]))
    torch.cuda.nvtx.range_pop()
    # the last re-sort against a full sort of the same pushed store (spare[0]: the store
    # before the last permute)
    full = mf.sort_by_tile(spare[0], mf.QUADRATIC, step.geom, TILE, within=True)
    same = bool(torch.equal(full.order, state["t"].order)) and bool(torch.equal(full.tile_start, state["t"].tile_start))
    step.order = saved
    n = ps.shape[1]
    del disp, spare, state
    torch.cuda.empty_cache()
    return {"value": n / (ms / 1000.0), "unit": "markers/s", "ms_per_step": ms,
            "resort_and_permute_ms": sum(resort) / len(resort), "order_equals_full_sort": same,
            "what": "push (up to 0.3 cell per axis) + incremental re-sort against the previous sorted keys + "
                    "permute positions and weights + gather + scatter, the store kept in cell-tile order"}


def sorted_sample(sample: int) -> tuple[np.ndarray, np.ndarray]:
    """A sample of the workload's markers in the store's cell-tile order."""
    from oracle import oracle as O

    pos, w = make_markers(sample, "cpu", torch.float64, seed=7)
    pos, w = pos.numpy(), w.numpy()
    order = O.sort_by_tile(O.tile_keys("quadratic", 2, pos, geometry(), TILE, within=True))
    return np.ascontiguousarray(pos[:, order]), np.ascontiguousarray(w[:, order])


def cpu_baseline(sample: int, threads: int = 0) -> dict:
    """The reference's CPU kernels (OpenMP restatement of the Pyccel versions) on a sample."""
    from oracle import oracle as O

    pos, w = sorted_sample(sample)
    field = make_field("cpu", torch.float64).numpy()
    density = np.zeros((GRID, GRID, GRID, 1))
    nthreads = threads or os.cpu_count() or 1
    O.cpu_gather("quadratic", 2, pos[:, :1000], field, geometry(), nthreads)  # warm
    t0 = time.perf_counter()
    O.cpu_gather("quadratic", 2, pos, field, geometry(), nthreads)
    t1 = time.perf_counter()
    used = O.cpu_scatter("quadratic", 2, pos, w, density, geometry(), nthreads)
    t2 = time.perf_counter()
    seconds = t2 - t0
    return {"value": sample / seconds, "unit": "markers/s", "cores": nthreads, "kind": "port",
            "sample": f"{sample} markers of the workload in the store's cell-tile order (gather {t1 - t0:.3f} s on {nthreads} threads, "
                      f"scatter {t2 - t1:.3f} s on {used} thread(s): the reference's 256^3 deposit "
                      "runs serially, its per-thread grids exceed 16,777,216 values)"}


def run_ours(args, world, rank, local) -> None:
    device = torch.device("cuda", local)
    dtype = torch.float64 if args.dtype == "f64" else torch.float32
    itemsize = 8 if dtype == torch.float64 else 4
    n = args.markers
    step = Step(n, device, dtype)
    pos, w = make_markers(n, device, dtype, seed=1 + rank)
    from mpifield_b200 import _lib

    # the marker store, sorted once by cell tile (untimed set-up)
    _, ps, ws = step.sort(pos, w)
    torch.cuda.synchronize()

    # the headline: gather + scatter on the sorted store
    launches0 = _lib.library().mpf_launch_count()
    torch.cuda.nvtx.range_push("timed")
    with ClockSampler(local) as clocks:
        seconds = time_loop(lambda: step.gather_scatter(ps, ws), args.steps, args.warmup, world, device)
    torch.cuda.nvtx.range_pop()
    launches = (_lib.library().mpf_launch_count() - launches0) // (args.steps + args.warmup) * args.steps
    per_step = seconds / args.steps

    # per-kernel times inside the step (events on the launching stream)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    g_ms = s_ms = 0.0
    for _ in range(args.steps):
        step.gather_scatter(ps, ws, ev)
        torch.cuda.synchronize()
        g_ms += ev[0].elapsed_time(ev[1])
        s_ms += ev[1].elapsed_time(ev[2])
    g_ms, s_ms = g_ms / args.steps, s_ms / args.steps

    # the full step from markers in random order, and its sort alone
    full = time_loop(lambda: step.full(pos, w), args.steps, 1, world, device)
    sort_ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    sort_ms = 0.0
    for _ in range(args.steps):
        sort_ev[0].record()
        step.sort(pos, w)
        sort_ev[1].record()
        torch.cuda.synchronize()
        sort_ms += sort_ev[0].elapsed_time(sort_ev[1])
    sort_ms /= args.steps

    alg = algorithmic_bytes(n, itemsize)
    peak, peak_kind = read_peak()
    dominant = "gather" if g_ms >= s_ms else "scatter"
    dom_ms = g_ms if dominant == "gather" else s_ms
    achieved = alg[dominant] / (dom_ms / 1000.0) / 1e9
    traffic = read_traffic(f"{dominant}_quadratic_3d_{args.dtype}")

    e2e = None
    if not args.no_e2e:
        # through the public API with host buffers: every step copies the positions and
        # weights in from pinned host memory and E and the density out, chunk by chunk,
        # the two copy directions and the kernels overlapped (mpifield_b200.streaming)
        from mpifield_b200 import _lib as L
        from mpifield_b200.streaming import HostPipeline

        hp = torch.empty((3, n), dtype=dtype, pin_memory=True)
        hw = torch.empty((1, n), dtype=dtype, pin_memory=True)
        hp.copy_(ps)
        hw.copy_(ws)
        hE = torch.empty((3, n), dtype=dtype, pin_memory=True)
        hD = torch.empty(step.density.shape, dtype=dtype, pin_memory=True)
        pipe = HostPipeline(device, 3, 3, 1, dtype)

        def e2e_step():
            step.density.zero_()
            pipe.step(L.QUADRATIC, 2, hp, hw, step.field, step.density, hE, step.geom, hD)

        e2e_steps = max(2, args.steps // 2)
        e2e_s = time_loop(e2e_step, e2e_steps, 1, world, device)
        e2e = {"value": n * world / (e2e_s / e2e_steps), "unit": "markers/s",
               "h2d_bytes_per_step": (hp.numel() + hw.numel()) * itemsize,
               "d2h_bytes_per_step": (hE.numel() + hD.numel()) * itemsize,
               "what": "positions + weights in, E + density out, per step, chunks of 2^22 markers with "
                       "host-to-device, kernels and device-to-host on three streams"}
        del pipe

    ref_cuda = None
    if not args.no_ref_cuda and rank == 0 and dtype == torch.float64:
        ref_cuda = ref_cuda_time(ps, ws, step.field, step.density, step.E, max(2, args.steps // 2))
        if ref_cuda is not None:
            ref_cuda["marker_order"] = "the same sorted store"
            random_order = ref_cuda_time(pos, w, step.field, step.density, step.E, max(2, args.steps // 2))
            ref_cuda["random_order"] = {k: random_order[k] for k in ("value", "gather_ms", "scatter_ms")}

    cpu = None
    if not args.no_cpu and rank == 0 and world == 1:
        cpu = cpu_baseline(1 << 21)

    extras = {}
    if not args.no_extras and rank == 0 and world == 1 and dtype == torch.float64:
        reps = max(2, args.steps // 2)
        extras["steady_step"] = measure_steady(step, ps, ws, reps)
        extras["fp32_variant"] = measure_fp32(step, ps, ws, reps)
        extras["deterministic_scatter"] = measure_deterministic(step, ps, ws, reps)
        extras["plain_2d"] = measure_plain_2d(device, max(10, args.steps))
        del pos, w
        torch.cuda.empty_cache()
        extras["autograd"] = measure_autograd(device, reps, peak)
        extras["path_deposit"] = measure_paths(device, reps, peak)
        extras["forms_and_clamped"] = measure_forms_and_clamped(device, reps)
        if args.serve_requests > 0:
            from mpifield_b200 import serving

            torch.cuda.empty_cache()
            extras["serving"] = serving.serve_benchmark(args.serve_requests, args.serve_rate, seed=0, device=device)
            extras["serving"]["what"] = (
                "mixed stream (Poisson arrivals, ndim 1-3, nodes per axis log-U[32,256], markers log-U[1e3,1e7], "
                "degree 1-3, gather 3-comp / scatter / path deposit, FP64, 120 GB budget) served with continuous "
                "batching vs one plain launch per request; latency = completion - arrival; at this rate both arms "
                "are saturated (requests/s = capacity, latency mostly queueing)")
            if args.serve_latency_rate > 0:
                torch.cuda.empty_cache()
                at_rate = serving.serve_benchmark(args.serve_requests, args.serve_latency_rate, seed=0, device=device)
                extras["serving"]["at_sustainable_rate"] = {
                    "rate_per_s": args.serve_latency_rate, "served": at_rate["served"],
                    "one_launch_per_request": at_rate["one_launch_per_request"],
                    "what": "the same stream arriving at a rate below both arms' capacity: latencies"}

    clock = clocks.summary()
    if rank == 0:
        line = {
            "metric": METRIC, "value": n * world / per_step, "unit": "markers/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1000.0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": args.dtype, "data": "synthetic",
            "config": {"workload": f"3D QUADRATIC gather E (3 comp) + scatter weights (1 comp), "
                                   f"{GRID}^3 periodic, N={n} markers (80% uniform, 20% beam sigma 0.05); "
                                   "marker store kept in cell-tile order (sorted once before timing)",
                       "markers": n, "grid": [GRID] * 3, "tile": list(TILE),
                       "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (positions 1.6 GB)"},
            "full_step": {"value": n * world / (full / args.steps), "unit": "markers/s",
                          "ms_per_step": full / args.steps * 1000.0,
                          "what": "from random marker order: tile sort + permute + gather + scatter + "
                                  "E back to marker order", "sort_and_permute_ms": sort_ms},
            "kernel_ms": {"gather": g_ms, "scatter": s_ms},
            "roofline": {"bound": "hbm", "kernel": f"{dominant}_quadratic_3d", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                         "algorithmic_bytes": alg[dominant], "traffic": traffic},
            "cpu_baseline": cpu, "ref_cuda": ref_cuda, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clock,
        }
        line.update(extras)
        print(json.dumps(line), flush=True)


# ------------------------------------------------------ the other configurations --
#
# Reported beside the headline in the same JSON line (keys "fp32_variant", "path_deposit",
# "autograd", "plain_2d"); each is a short measurement of its own configuration with
# CUDA events on the current stream.

def _event_ms(fn, reps: int) -> float:
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def measure_fp32(step, ps, ws, reps: int) -> dict:
    """The float32 variant of the headline step on the same sorted store, and its error
    against the float64 results (max |f32 - f64| / max |f64|, per output)."""
    import mpifield_b200 as mf

    n = ps.shape[1]
    step.gather_scatter(ps, ws)
    E64, D64 = step.E.clone(), step.density.clone()
    p32, w32, f32 = ps.float(), ws.float(), step.field.float()
    E32 = torch.empty((3, n), dtype=torch.float32, device=ps.device)
    D32 = torch.zeros(step.density.shape, dtype=torch.float32, device=ps.device)
    def go():
        mf.kernels.gather(step.lib.QUADRATIC, 2, p32, f32, E32, step.geom, order=step.order)
        D32.zero_()
        mf.kernels.scatter(step.lib.QUADRATIC, 2, p32, w32, D32, step.geom, order=step.order)

    ms = _event_ms(go, reps)
    err_e = float((E32.double() - E64).abs().max() / E64.abs().max())
    err_d = float((D32.double() - D64).abs().max() / D64.abs().max())
    del p32, w32, f32, E32, D32, E64, D64
    return {"value": n / (ms / 1000.0), "unit": "markers/s", "ms_per_step": ms,
            "max_rel_err_vs_f64": {"gather": err_e, "scatter": err_d},
            "what": "gather + scatter in float32 on the same store (positions, weights and field rounded "
                    "to float32); error relative to max |float64 result|"}


PATH_GRID = 128


def path_case(device, n: int = 1 << 25, seed: int = 7):
    """The path-deposit workload: 128^3 periodic on the unit cube, start uniform, end =
    start + U[-0.9, 0.9] cells per axis, charges U[0.5, 1.5] (dt = 1). Returns start,
    end (3, n), charges (1, n) and the `BlockGrid`."""
    import mpifield_b200 as mf

    g_n = PATH_GRID
    g = torch.Generator(device=device).manual_seed(seed)
    start = torch.rand((3, n), generator=g, device=device, dtype=torch.float64)
    end = start + (torch.rand((3, n), generator=g, device=device, dtype=torch.float64) * 1.8 - 0.9) / g_n
    q = torch.rand((1, n), generator=g, device=device, dtype=torch.float64) + 0.5
    grid = mf.BlockGrid.from_geometry((0.0,) * 3, (1.0 / g_n,) * 3, (g_n,) * 3, (True,) * 3)
    return start, end, q, grid


def measure_paths(device, reps: int, peak: float, n: int = 1 << 25, cpu_sample: int | None = 1 << 21) -> dict:
    """The path deposit on `path_case`: WHITNEY, QUADRATIC_EDGES and CUBIC_EDGES, paths in
    random order and sorted by the start's cell tile; continuity residual max |rho(end) -
    rho(start) - G^T J| with the node deposit of the same degree; beside them the
    reference's CUDA kernels on the same GPU and its CPU kernels on a sample of the paths
    (``cpu_sample`` None: neither)."""
    import mpifield_b200 as mf

    g_n = PATH_GRID
    start, end, q, grid = path_case(device, n)
    geom = grid.geometry
    t = mf.sort_by_tile(start, mf.LINEAR, geom, TILE, within=True)
    s_start, s_end, s_q = mf.permute(start, t.order), mf.permute(end, t.order), mf.permute(q, t.order)
    edges = torch.zeros((g_n, g_n, g_n, 3), dtype=torch.float64, device=device)
    nbytes = n * 56 + g_n ** 3 * 24 * 2
    out = {"config": f"{g_n}^3 periodic, N={n} paths, |displacement| <= 0.9 cell per axis", "unit": "paths/s",
           "algorithmic_bytes": nbytes, "timing": "CUDA events, mean and best of the timed repetitions"}
    ref = _ref_cuda_lib() if cpu_sample is not None else None
    for degree, name in ((1, "whitney"), (2, "quadratic_edges"), (3, "cubic_edges")):
        ew, nodes = mf.splines(degree).edges, mf.splines(degree).nodes
        res = {}
        for order, (a, b, c) in (("random", (start, end, q)), ("sorted", (s_start, s_end, s_q))):
            def go():
                edges.zero_()
                ew.deposit_paths_block(a, b, c[0], edges, grid)
            ms, best = _event_stats(go, reps)
            res[order] = {"value": n / (ms / 1000.0), "ms": ms, "best_ms": best,
                          "hbm_frac": nbytes / (ms / 1000.0) / 1e9 / peak}
        if ref is not None:
            # the reference's own CUDA deposit (deposit_paths_3d / deposit_paths_spline_3d,
            # one thread per path) on the same paths and GPU
            kernel = "deposit_paths_3d" if degree == 1 else "deposit_paths_spline_3d"
            ints = [g_n] * 3 + [1] * 3 + ([] if degree == 1 else [degree])
            refs = {}
            for order, (a, b, c) in (("random", (start, end, q)), ("sorted", (s_start, s_end, s_q))):
                def go_ref():
                    edges.zero_()
                    _ref_call(ref, kernel, n, [a, b, c[0], edges], [0.0] * 3 + [1.0 / g_n] * 3, ints)
                ms, best = _event_stats(go_ref, max(2, reps // 2))
                refs[order] = {"value": n / (ms / 1000.0), "ms": ms, "best_ms": best}
            res["ref_cuda"] = refs
        if cpu_sample:
            # the reference's CPU path (its Pyccel kernels restated with OpenMP: WHITNEY on
            # every host thread, the spline edges serial as the reference runs them)
            from oracle import oracle as O

            m = cpu_sample if degree == 1 else cpu_sample // 8
            hs, he, hq = (t[:, :m].cpu().numpy() for t in (start, end, q))
            host = np.zeros((g_n, g_n, g_n, 3))
            threads = os.cpu_count() or 1
            t0 = time.perf_counter()
            used = O.cpu_deposit(degree, hs, he, hq[0], host, grid.geometry, threads)
            sec = time.perf_counter() - t0
            res["cpu"] = {"value": m / sec, "unit": "paths/s", "cores": used or 1, "kind": "port",
                          "sample": f"{m} paths of the workload"}
            del host
        before = torch.zeros((g_n, g_n, g_n, 1), dtype=torch.float64, device=device)
        after = torch.zeros_like(before)
        nodes.scatter_block(start, q[0], before, grid)
        nodes.scatter_block(end, q[0], after, grid)
        edges.zero_()
        ew.deposit_paths_block(start, end, q[0], edges, grid)
        change = (after - before)[..., 0]
        resid = float((ew.divergence_block(edges, grid) - change).abs().max())
        res["continuity_residual"] = resid
        res["continuity_scale"] = float(change.abs().max())
        out[name] = res
        del before, after, change
    return out


def measure_autograd(device, reps: int, peak: float) -> dict:
    """Differentiation: 512^2 periodic, CUBIC, 1-component field of seeded Fourier modes,
    N = 2^22 uniform markers, weights U[0, 1]; forward + backward of
    sum(w gather(f, x)) + 0.5 ||scatter(x, w)||^2 with respect to f, w and x."""
    import mpifield_b200 as mf
    from mpifield_b200 import autograd as AG

    n, g_n = 1 << 22, 512
    geom = (0.0, 0.0, 1.0 / g_n, 1.0 / g_n, g_n, g_n, 1, 1)
    gen = torch.Generator(device="cpu").manual_seed(5)
    xs = torch.arange(g_n, dtype=torch.float64) / g_n
    f0 = torch.zeros((g_n, g_n), dtype=torch.float64)
    for _ in range(8):
        k = torch.randint(1, 9, (2,), generator=gen)
        phase = float(torch.rand(1, generator=gen)) * 2 * np.pi
        f0 += torch.cos(2 * np.pi * (k[0] * xs[:, None] + k[1] * xs[None, :]) + phase)
    g = torch.Generator(device=device).manual_seed(6)
    x0 = torch.rand((2, n), generator=g, device=device, dtype=torch.float64)
    w0 = torch.rand((1, n), generator=g, device=device, dtype=torch.float64)
    out = {"config": f"{g_n}^2 periodic, CUBIC, N={n}", "unit": "markers/s"}
    for dtype, name in ((torch.float64, "f64"), (torch.float32, "f32")):
        f = f0.to(device=device, dtype=dtype).view(g_n, g_n, 1).clone().requires_grad_(True)
        w = w0.to(dtype).clone().requires_grad_(True)
        x = x0.to(dtype).clone().requires_grad_(True)

        def go():
            f.grad = w.grad = x.grad = None
            rho = AG.scatter(x, w, mf.CUBIC, geom)
            loss = (w * AG.gather(f, x, mf.CUBIC, geom)).sum() + 0.5 * (rho * rho).sum()
            loss.backward()

        ms, best = _event_stats(go, reps)
        # compulsory bytes of the step: every pass over the markers (forward gather and
        # scatter, backward gather, scatter and position gradient) reads positions and one
        # marker row and writes one; plus a few passes over the 512^2 grid
        item = 8 if dtype == torch.float64 else 4
        nbytes = n * 9 * item + 8 * g_n * g_n * item
        out[name] = {"value": n / (ms / 1000.0), "ms_per_step": ms, "best_ms": best,
                     "algorithmic_bytes": nbytes, "hbm_frac": nbytes / (ms / 1000.0) / 1e9 / peak}
    out["reference"] = "none: the reference has no differentiation"
    return out


def measure_forms_and_clamped(device, reps: int) -> dict:
    """The k-form kernels and clamped axes: 3D, 128^3 nodes on the unit cube, N = 2^24
    uniform markers (random order). Faces (2-forms, 3 components) and cells (top form)
    of degree 2, gather + scatter, periodic; then CUBIC node gather (3 components) +
    scatter with every axis clamped (Cox-de Boor knots) beside the same on periodic
    axes."""
    import mpifield_b200 as mf
    from mpifield_b200.kernels import gather, gather_forms, scatter, scatter_forms

    n, g_n = 1 << 24, 128
    g = torch.Generator(device=device).manual_seed(12)
    pos = torch.rand((3, n), generator=g, device=device, dtype=torch.float64)
    vals3 = torch.rand((3, n), generator=g, device=device, dtype=torch.float64) + 0.5
    out = {"config": f"{g_n}^3 on the unit cube, N={n} uniform markers in random order", "unit": "markers/s"}
    h = 1.0 / g_n
    periodic = (0.0, 0.0, 0.0, h, h, h, g_n, g_n, g_n, 1, 1, 1)
    res3 = torch.empty((3, n), dtype=torch.float64, device=device)
    for form, name, nc in ((2, "faces_quadratic", 3), (3, "cells_quadratic", 1)):
        field = torch.rand((g_n, g_n, g_n, nc), generator=g, device=device, dtype=torch.float64)
        dep = torch.zeros_like(field)

        def go():
            gather_forms(2, form, pos, field, res3[:nc], periodic)
            dep.zero_()
            scatter_forms(2, form, pos, vals3[:nc], dep, periodic)

        ms, best = _event_stats(go, reps)
        out[name] = {"value": n / (ms / 1000.0), "ms": ms, "best_ms": best}
        del field, dep
    hc = 1.0 / (g_n - 1)
    clamped = (0.0, 0.0, 0.0, hc, hc, hc, g_n, g_n, g_n, 2, 2, 2)
    for codes, geom, name in (("clamped", clamped, "cubic_clamped"), ("periodic", periodic, "cubic_periodic")):
        ext = g_n + 2 if codes == "clamped" else g_n
        field = torch.rand((ext, ext, ext, 3), generator=g, device=device, dtype=torch.float64)
        dens = torch.zeros((ext, ext, ext, 1), dtype=torch.float64, device=device)

        def go():
            gather(mf.kernels._lib.SPLINE, 3, pos, field, res3, geom)
            dens.zero_()
            scatter(mf.kernels._lib.SPLINE, 3, pos, vals3[:1], dens, geom)

        ms, best = _event_stats(go, reps)
        out[name] = {"value": n / (ms / 1000.0), "ms": ms, "best_ms": best}
        del field, dens
    del pos, vals3, res3
    torch.cuda.empty_cache()
    return out


def measure_deterministic(step, ps, ws, reps: int) -> dict:
    """The bit-reproducible scatter on the headline store (its tile form, with the store's
    tile starts; the plain form beside it): time, identical bits on a repeat and between
    the two forms, and the largest difference from the FP64 atomic scatter (relative to
    max |density|)."""
    from mpifield_b200 import _lib
    from mpifield_b200.kernels import scatter_deterministic

    density = torch.zeros_like(step.density)
    workspace = torch.empty(16 * density.numel() + 4096, dtype=torch.uint8, device=ps.device)

    def go(order):
        density.zero_()
        scatter_deterministic(_lib.QUADRATIC, 2, ps, ws, density, step.geom, workspace, order=order)

    plain_ms = _event_ms(lambda: go(None), reps)
    plain = density.clone()
    ms = _event_ms(lambda: go(step.order), reps)
    first = density.clone()
    go(step.order)
    same = bool(torch.equal(first.view(torch.int64), density.view(torch.int64)))
    same_forms = bool(torch.equal(first.view(torch.int64), plain.view(torch.int64)))
    step.gather_scatter(ps, ws)
    diff = float((density - step.density).abs().max() / step.density.abs().max())
    return {"value": ps.shape[1] / (ms / 1000.0), "unit": "markers/s", "ms": ms, "bitwise_repeatable": same,
            "plain_form_ms": plain_ms, "same_bits_as_plain_form": same_forms,
            "max_rel_diff_vs_atomic_scatter": diff}


def plain_2d_case():
    """The plain 2D workload: 101 x 51 nodes on [0, 0.1] x [0, 0.05], bounded (geometry);
    N = 100,000 uniform markers from numpy default_rng(0) (2, N); E = -gradient(phi),
    phi = 1000 exp(-((x - 0.05)^2 + (y - 0.025)^2) / 1e-4), by numpy.gradient (101, 51, 2)."""
    nx, ny, n = 101, 51, 100_000
    hx, hy = 0.1 / (nx - 1), 0.05 / (ny - 1)
    geom = (0.0, 0.0, hx, hy, nx, ny, 0, 0)
    X, Y = np.meshgrid(np.linspace(0, 0.1, nx), np.linspace(0, 0.05, ny), indexing="ij")
    phi = 1000.0 * np.exp(-((X - 0.05) ** 2 + (Y - 0.025) ** 2) / 1e-4)
    ex, ey = np.gradient(phi, hx, hy)
    rng = np.random.default_rng(0)
    pos = np.stack([rng.uniform(0, 0.1, n), rng.uniform(0, 0.05, n)])
    return geom, pos, np.stack([-ex, -ey], axis=-1)


def measure_plain_2d(device, reps: int) -> dict:
    """The plain 2D configuration: 101 x 51 nodes on [0, 0.1] x [0, 0.05], bounded; LINEAR;
    E = -gradient(phi), phi = 1000 exp(-((x - 0.05)^2 + (y - 0.025)^2) / 1e-4); N = 100,000
    uniform markers (numpy default_rng(0)); scatter unit weights + gather E (2, N). The
    kernels on the block itself (its halo nodes trimmed at the bounded walls)."""
    import mpifield_b200 as mf

    geom, pos_np, E_np = plain_2d_case()
    nx, ny, n = geom[4], geom[5], pos_np.shape[1]
    E = torch.tensor(E_np, device=device)
    pos = torch.tensor(pos_np, device=device)
    ones = torch.ones((1, n), dtype=torch.float64, device=device)
    rho = torch.zeros((nx, ny, 1), dtype=torch.float64, device=device)
    out_e = torch.empty((2, n), dtype=torch.float64, device=device)
    gather, scatter = mf.KERNELS["gather_linear_2d"], mf.KERNELS["scatter_linear_2d"]

    def go():
        rho.zero_()
        scatter(pos, ones, rho, *geom)
        gather(pos, E, out_e, *geom)

    ms = _event_ms(go, reps)
    # the same step captured once in a CUDA graph and replayed: the kernels neither allocate
    # nor synchronise, so their launches replay without the host's per-call work
    expected = (rho.clone(), out_e.clone())
    stream = torch.cuda.Stream(device)
    with torch.cuda.stream(stream):
        go()  # warm-up outside the capture (kernel attributes are set once)
    stream.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        go()
    graph_ms = _event_ms(graph.replay, reps)
    torch.cuda.synchronize()
    same = bool(torch.equal(out_e, expected[1])) and float((rho - expected[0]).abs().max()) <= 1e-12 * float(
        expected[0].abs().max())
    _, best_ms = _event_stats(go, reps)
    result = {"value": n / (ms / 1000.0), "unit": "markers/s", "us_per_step": ms * 1000.0,
              "best_us_per_step": best_ms * 1000.0, "graph_us_per_step": graph_ms * 1000.0, "graph_matches": same,
              "config": "101x51 bounded, LINEAR, N=100000: scatter + gather (launch-bound); graph_us_per_step: "
                        "the step replayed from a CUDA graph"}
    ref = _ref_cuda_lib()
    if ref is not None:
        # the reference's CUDA scatter_linear_2d + gather_linear_2d on the same arrays and GPU
        doubles, ints = [0.0, 0.0, geom[2], geom[3]], [nx, ny, 0, 0]

        def go_ref():
            rho.zero_()
            _ref_call(ref, "scatter_linear_2d", n, [pos, ones, rho], doubles, ints)
            _ref_call(ref, "gather_linear_2d", n, [pos, E, out_e], doubles, ints)

        ref_ms, ref_best = _event_stats(go_ref, reps)
        result["ref_cuda"] = {"value": n / (ref_ms / 1000.0), "us_per_step": ref_ms * 1000.0,
                              "best_us_per_step": ref_best * 1000.0}
    # the reference's CPU kernels (OpenMP restatement of its Pyccel versions), all host threads
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    hp, hE = pos.cpu().numpy(), E.cpu().numpy()
    hrho = np.zeros((nx, ny, 1))
    O.cpu_gather("linear", 1, hp, hE, geom, threads)
    cpu = []
    for _ in range(5):
        t0 = time.perf_counter()
        hrho[...] = 0.0
        O.cpu_scatter("linear", 1, hp, np.ones((1, n)), hrho, geom, threads)
        O.cpu_gather("linear", 1, hp, hE, geom, threads)
        cpu.append(time.perf_counter() - t0)
    result["cpu"] = {"value": n / min(cpu), "us_per_step": min(cpu) * 1e6, "cores": threads, "kind": "port",
                     "sample": "the whole workload, best of 5"}
    return result


def run_reference(args, world, rank) -> None:
    if rank != 0:
        return
    sample = 1 << 21
    from oracle import oracle as O

    pos, w = sorted_sample(sample)
    field = make_field("cpu", torch.float64).numpy()
    density = np.zeros((GRID, GRID, GRID, 1))
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        O.cpu_gather("quadratic", 2, pos[:, :65536], field, geometry(), threads)
        O.cpu_scatter("quadratic", 2, pos[:, :65536], w[:, :65536], density, geometry(), threads)
    t0 = time.perf_counter()
    used = 1
    for _ in range(args.steps):
        O.cpu_gather("quadratic", 2, pos, field, geometry(), threads)
        density[...] = 0.0
        used = O.cpu_scatter("quadratic", 2, pos, w, density, geometry(), threads)
    seconds = (time.perf_counter() - t0) / args.steps
    value = sample / seconds
    sample_text = (f"{sample} markers of the workload per step; gather on {threads} threads, scatter on "
                   f"{used} thread(s) (the reference's rule for a 256^3 deposit)")
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": "markers/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": seconds * 1000.0, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": f"3D QUADRATIC gather E (3 comp) + scatter weights (1 comp), {GRID}^3 periodic, "
                               "markers 80% uniform 20% beam; the reference's CPU kernels (OpenMP restatement "
                               "of its Pyccel versions)", "markers": sample, "grid": [GRID] * 3},
        "cpu_baseline": {"value": value, "unit": "markers/s", "cores": threads, "kind": "port",
                         "sample": sample_text},
        "e2e": {"value": value, "unit": "markers/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main() -> None:
    global GRID
    args = parse()
    GRID = args.grid
    world, rank, local = dist_setup(args)
    try:
        if args.paths_only > 0:
            device = torch.device("cuda", local)
            torch.cuda.set_device(device)
            if rank == 0:
                peak, _ = read_peak()
                print(json.dumps({"path_deposit": measure_paths(device, max(1, args.steps), peak, args.paths_only,
                                                                cpu_sample=None)}))
            return
        if args.steady_only:
            device = torch.device("cuda", local)
            torch.cuda.set_device(device)
            if rank == 0:
                step = Step(args.markers, device, torch.float64)
                pos, w = make_markers(args.markers, device, torch.float64, seed=1)
                _, ps, ws = step.sort(pos, w)
                del pos, w
                print(json.dumps({"steady_step": measure_steady(step, ps, ws, max(2, args.steps))}))
            return
        if args.autograd_only:
            device = torch.device("cuda", local)
            torch.cuda.set_device(device)
            if rank == 0:
                peak, _ = read_peak()
                print(json.dumps({"autograd": measure_autograd(device, max(1, args.steps), peak)}))
            return
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
