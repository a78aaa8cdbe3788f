"""The halo exchange of a field split over ranks (mpifield_b200.exchange) on CPU ranks.

gloo, world sizes 2 and 4, 1D-3D Cartesian splits, periodic and bounded axes, halos of 1
and 2 layers. Each rank holds its block of one global field; the slab copies are plain
tensor slicing here (the library's kernels need a GPU; they are checked against the same
slicing in tests/test_gpu_field.py). Expected results are computed from the whole field
in NumPy, as one process would see them:

- fill: every halo node holds the global node it overlaps (wrapped on a periodic axis);
  beyond the wall of a bounded axis it keeps what it held;
- fold: the owned nodes receive every rank's storage entry that overlaps them (wrapped
  on a periodic axis; beyond a wall dropped), and every halo is zero.
"""

from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from mpifield_b200.exchange import Decomposition

ROOT = Path(__file__).resolve().parents[1]

CASES = [
    # (num_gridpoints, periodic, dims, halo)
    ((12,), (True,), (2,), 2),
    ((9,), (False,), (2,), 1),
    ((10, 7), (True, False), (2, 1), 2),
    ((10, 7), (False, True), (1, 2), 1),
    ((8, 9), (True, True), (2, 2), 2),
    ((6, 5, 7), (True, False, True), (2, 1, 2), 1),
    ((8, 6, 6), (True, True, True), (4, 1, 1), 2),
]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def slice_pack(storage, halo, axis, first, buffer):
    buffer.copy_(storage.narrow(axis, first, halo).reshape(-1))


def slice_unpack(storage, halo, axis, first, buffer, accumulate):
    view = storage.narrow(axis, first, halo)
    part = buffer.reshape(view.shape)
    if accumulate:
        view += part
    else:
        view.copy_(part)


def _window(dec: Decomposition, h: int):
    """Per axis the global indices of the rank's stored nodes (wrapped on a periodic axis,
    -1 beyond a wall)."""
    out = []
    for a in range(dec.ndim):
        idx = np.arange(dec.offset[a] - h, dec.offset[a] + dec.owned[a] + h)
        num = dec.num_gridpoints[a]
        if dec.periodic[a]:
            idx = idx % num
        else:
            idx = np.where((idx >= 0) & (idx < num), idx, -1)
        out.append(idx)
    return out


def _rank(rank, world, port, case, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    from mpifield_b200.exchange import HaloExchange

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        num, periodic, dims, h = CASES[case]
        dec = Decomposition(num, periodic, dims, rank)
        ex = HaloExchange(dec, h, pack=slice_pack, unpack=slice_unpack)
        rng = np.random.default_rng(case)
        glob = rng.normal(size=(*num, 2))
        win = _window(dec, h)
        stored = tuple(m + 2 * h for m in dec.owned)
        # fill: owned nodes from the global field, halos a marker value
        block = np.full((*stored, 2), -7.0)
        own = tuple(slice(h, h + m) for m in dec.owned)
        block[own] = glob[tuple(np.ix_(*[w[h:-h] for w in win]))]
        t = torch.tensor(block)
        ex.fill(t)
        expected = np.full_like(block, -7.0)
        mesh = np.ix_(*win)
        inside = np.ones(stored, dtype=bool)
        for a, w in enumerate(win):
            shape = [1] * dec.ndim
            shape[a] = -1
            inside = inside & (w >= 0).reshape(shape)
        safe = tuple(np.where(m >= 0, m, 0) for m in mesh)
        expected[inside] = glob[safe][inside]
        fill_ok = bool(np.array_equal(t.numpy(), expected))
        # fold: every rank's storage random; the owned nodes collect what overlaps them
        deposit = np.random.default_rng(1000 + rank).normal(size=(*stored, 2))
        t = torch.tensor(deposit)
        ex.fold(t)
        out[rank] = (fill_ok, t.numpy().copy(), deposit, [w.copy() for w in win], dec.offset, dec.owned)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", range(len(CASES)))
def test_split_field_fill_and_fold(case):
    num, periodic, dims, h = CASES[case]
    world = int(np.prod(dims))
    port = _free_port()
    with mp.Manager() as manager:
        out = manager.dict()
        mp.start_processes(_rank, args=(world, port, case, out), nprocs=world, join=True, start_method="spawn")
        results = dict(out)
    assert all(results[r][0] for r in range(world)), "fill"
    total = np.zeros((*num, 2))
    for r in range(world):
        _, _, deposit, win, _, _ = results[r]
        mesh = np.ix_(*win)
        keep = np.ones(deposit.shape[:-1], dtype=bool)
        for a, w in enumerate(win):
            shape = [1] * len(num)
            shape[a] = -1
            keep = keep & (w >= 0).reshape(shape)
        idx = tuple(np.where(m >= 0, m, 0) for m in mesh)
        full = tuple(np.broadcast_to(i, deposit.shape[:-1])[keep] for i in idx)
        np.add.at(total, full, deposit[keep])
    for r in range(world):
        _, folded, _, _, offset, owned = results[r]
        own = tuple(slice(h, h + m) for m in owned)
        glob = tuple(slice(o, o + m) for o, m in zip(offset, owned))
        np.testing.assert_allclose(folded[own], total[glob], rtol=0, atol=1e-12)
        halo = np.ones(folded.shape[:-1], dtype=bool)
        halo[own] = False
        assert not folded[halo].any()


def test_decomposition_blocks_and_neighbours():
    d = Decomposition((10, 7), (True, False), (2, 3), 4)
    assert d.coords == (1, 1) and d.offset == (5, 3) and d.owned == (5, 2)
    assert d.neighbours(0) == (1, 1) and d.neighbours(1) == (3, 5)
    edge = Decomposition((10, 7), (True, False), (2, 3), 0)
    assert edge.neighbours(1) == (None, 1) and edge.owned == (5, 3)
    with pytest.raises(ValueError):
        Decomposition((3,), (True,), (4,), 0)
    with pytest.raises(ValueError):
        Decomposition((8,), (True,), (2,), 2)
