"""Edge fields on the B200 kernels: `EdgeWeighting`, `WHITNEY`, `QUADRATIC_EDGES`, `CUBIC_EDGES`.

An edge field holds, for every node and axis, the line integral along the edge from the
node to its neighbour along that axis: an array ``num_nodes + (ndim,)`` (``num_nodes +
p - 1`` entries along a clamped axis of degree p). `EdgeWeighting` is mpifield's plug-in
type for the two operations on it (src/mpifield/edges.py:98-265): ``EdgeWeighting(name,
gather={ndim: kernel}, deposit_paths={ndim: kernel}, halo, degree, clamps)`` with
`gather_block` (the field at markers) and `deposit_paths_block` (the current of charges
moving along straight paths), and the discrete gradient `gradient_block` and its
transpose `divergence_block`, with which the deposit conserves charge:
``divergence_block(J)`` equals the node deposit at the paths' ends minus at their starts.
"""

from __future__ import annotations

from collections.abc import Callable, Mapping
from dataclasses import dataclass
from typing import Any

from mpifield_b200 import _lib
from mpifield_b200._arrays import as_device_array
from mpifield_b200._plugins import KernelTable, on_device_of
from mpifield_b200._types import BlockGrid
from mpifield_b200.kernels import EdgeGatherKernel, PathKernel

__all__ = ["CUBIC_EDGES", "QUADRATIC_EDGES", "WHITNEY", "EdgeWeighting"]

KernelFunction = Callable[..., Any]


def _shift(t, axis: int, periodic: bool, toward_end: bool):
    """``t`` moved one node along ``axis`` (toward the end or the start); on a bounded
    axis the vacated entry is zero, on a periodic one it wraps."""
    import torch

    if periodic:
        return torch.roll(t, 1 if toward_end else -1, dims=axis)
    n = t.shape[axis]
    zero = torch.zeros_like(t.narrow(axis, 0, 1))
    if toward_end:
        return torch.cat((zero, t.narrow(axis, 0, n - 1)), dim=axis)
    return torch.cat((t.narrow(axis, 1, n - 1), zero), dim=axis)


def _last_node_cleared(t, axis: int):
    """``t`` with its last node along ``axis`` zero (no edge leaves it on a bounded axis)."""
    out = t.clone()
    out.narrow(axis, t.shape[axis] - 1, 1).zero_()
    return out


@dataclass(frozen=True, eq=False, repr=False)
class EdgeWeighting(KernelTable):
    """Edge gather and path-deposit kernels by number of dimensions, with the halo a split
    field needs, the B-spline degree (1 for Whitney) and whether they take clamped axes."""

    ROLES = ("gather", "deposit_paths")
    NOUN = "edge weighting"
    LOWEST_DEGREE = 1

    name: str
    gather: Mapping[int, KernelFunction]
    deposit_paths: Mapping[int, KernelFunction]
    halo: int = 1
    degree: int | None = None
    clamps: bool = False

    def gather_kernel(self, ndim: int) -> KernelFunction:
        return self.kernel("gather", ndim)

    def deposit_paths_kernel(self, ndim: int) -> KernelFunction:
        return self.kernel("deposit_paths", ndim)

    def _edge_field_ndim(self, edges, grid: BlockGrid) -> int:
        """The dimensions of ``grid``, after checking the shape of the edge field on it."""
        ndim = self.accept_grid(grid)
        extra = (self.degree or 1) - 1
        clamped = grid.clamped or (False,) * ndim
        want = tuple(int(n) + (extra if c else 0) for n, c in zip(grid.num_gridpoints, clamped)) + (ndim,)
        have = as_device_array(edges, "edges").shape
        if have != want:
            raise ValueError(f"an edge field on this grid is {want}, got {have}")
        return ndim

    def gather_block(self, positions, edges, result, grid: BlockGrid) -> None:
        """Write the field of ``edges`` at ``positions`` (ndim, N) into ``result`` (ndim, N)."""
        run = self.gather_kernel(self._edge_field_ndim(edges, grid))
        run(on_device_of(positions, edges), edges, result, *grid.geometry)

    def deposit_paths_block(self, start, end, charges, edges, grid: BlockGrid) -> None:
        """Add to ``edges`` the current of ``charges`` (N,) moving in straight lines from
        ``start`` to ``end`` (ndim, N)."""
        run = self.deposit_paths_kernel(self._edge_field_ndim(edges, grid))
        start, end, charges = (on_device_of(a, edges) for a in (start, end, charges))
        s, e, q = (as_device_array(a) for a in (start, end, charges))
        if s.shape != e.shape or s.shape[-1] != q.size:
            raise ValueError(f"paths from {s.shape} to {e.shape} for {q.size} charges")
        run(start, end, charges, edges, *grid.geometry)

    @staticmethod
    def gradient_block(nodes, grid: BlockGrid):
        """``G phi`` (torch): every edge gets the difference of ``nodes`` between its end
        and its start node; edges that leave a bounded axis at its last node get zero."""
        import torch

        nodes = as_device_array(nodes, "nodes").torch()
        parts = []
        for axis, periodic in enumerate(grid.periodic):
            step = _shift(nodes, axis, periodic, toward_end=False) - nodes
            parts.append(step if periodic else _last_node_cleared(step, axis))
        return torch.stack(parts, dim=-1)

    @staticmethod
    def divergence_block(edges, grid: BlockGrid):
        """``G^T j`` (torch), the transpose of `gradient_block`: every node gets what its
        incoming edges carry minus what its outgoing edges carry -- the change of the
        node charge the current brings."""
        edges = as_device_array(edges, "edges").torch()
        total = None
        for axis, periodic in enumerate(grid.periodic):
            flow = edges[..., axis]
            if not periodic:
                flow = _last_node_cleared(flow, axis)
            term = _shift(flow, axis, periodic, toward_end=True) - flow
            total = term if total is None else total + term
        return total


def _edge_tables(kind: int, degree: int) -> tuple[dict, dict]:
    return ({n: EdgeGatherKernel(kind, n, False, degree) for n in (1, 2, 3)},
            {n: PathKernel(kind, n, False, degree) for n in (1, 2, 3)})


def spline_edges(name: str, degree: int) -> EdgeWeighting:
    """The spline edge weighting of degree 1-3 (along an edge degree - 1, across it
    degree), on the spline-edge kernels; takes clamped axes."""
    gather, deposit = _edge_tables(_lib.SPLINE, degree)
    return EdgeWeighting(name, gather=gather, deposit_paths=deposit, halo=2, degree=degree, clamps=True)


#: The lowest-order (Whitney) edges, whose node space is LINEAR's.
WHITNEY = EdgeWeighting("whitney", *_edge_tables(_lib.LINEAR, 1), halo=1, degree=1)
#: The edges that go with QUADRATIC (linear along an edge, quadratic across).
QUADRATIC_EDGES = spline_edges("quadratic", 2)
#: The edges that go with CUBIC (quadratic along an edge, cubic across).
CUBIC_EDGES = spline_edges("cubic", 3)
