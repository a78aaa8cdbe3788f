"""The bench's multi-process plumbing on CPU (gloo, world size 2): ranks agree on the max
time over ranks, and under torchrun only rank 0 prints the one JSON line."""

from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import torch
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import argparse

    import bench
    import torch.distributed as dist

    w, r, _ = bench.dist_setup(argparse.Namespace(impl="reference"))
    try:
        bench.barrier(w)
        out[r] = bench.max_over_ranks(1.5 + r, w, torch.device("cpu"))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_gloo():
    port = _free_port()
    with mp.Manager() as manager:
        out = manager.dict()
        mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        assert dict(out) == {0: 2.5, 1: 2.5}


def test_the_reference_arm_under_torchrun_prints_one_line():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0"]
    res = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [l for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
