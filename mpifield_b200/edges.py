"""Edge fields: the edge gather and the charge-conserving path deposit.

The same plug-in type as mpifield's ``EdgeWeighting`` (src/mpifield/edges.py:98-265):
``EdgeWeighting(name, gather={ndim: kernel}, deposit_paths={ndim: kernel}, halo, degree,
clamps)`` with ``gather_block``, ``deposit_paths_block``, ``gradient_block`` and
``divergence_block``, and the built-ins `WHITNEY` (degree 1), `QUADRATIC_EDGES` and
`CUBIC_EDGES` on the sm_100a kernels. An edge field is ``num_nodes + (ndim,)``: entry
``(k, a)`` the line integral along the edge from node k to its neighbour along axis a
(``num_nodes + p - 1`` entries along a clamped axis).
"""

from __future__ import annotations

from collections.abc import Callable, Mapping
from dataclasses import dataclass
from types import MappingProxyType
from typing import Any

import torch

from mpifield_b200 import _lib
from mpifield_b200._types import BlockGrid
from mpifield_b200.kernels import EdgeGatherKernel, PathKernel
from mpifield_b200.weighting import _as_marker_tensor, _check_clamps

__all__ = ["CUBIC_EDGES", "QUADRATIC_EDGES", "WHITNEY", "EdgeWeighting"]

KernelFunction = Callable[..., Any]


def _checked(kernels: Mapping[int, KernelFunction], role: str) -> Mapping[int, Any]:
    for ndim in kernels:
        if ndim not in (1, 2, 3):
            raise ValueError(f"{role} kernels are for 1, 2 or 3 dimensions, got {ndim}")
    return MappingProxyType(dict(kernels))


@dataclass(frozen=True)
class _WithDegree:
    """A spline edge kernel with its degree appended."""

    kernel: KernelFunction
    degree: int

    def __call__(self, *arguments: Any) -> None:
        self.kernel(*arguments, self.degree)


@dataclass(frozen=True, eq=False, repr=False)
class EdgeWeighting:
    """The edge gather and its path deposit, for each number of dimensions they cover."""

    name: str
    gather: Mapping[int, KernelFunction]
    deposit_paths: Mapping[int, KernelFunction]
    halo: int = 1
    degree: int | None = None
    clamps: bool = False

    def __post_init__(self) -> None:
        if self.halo < 0:
            raise ValueError(f"halo must be >= 0, got {self.halo}")
        if self.degree is not None and self.degree < 1:
            raise ValueError(f"degree must be >= 1, got {self.degree}")
        object.__setattr__(self, "gather", _checked(self.gather, "gather"))
        object.__setattr__(self, "deposit_paths", _checked(self.deposit_paths, "deposit_paths"))

    def _kernel(self, kernels, ndim: int, role: str):
        try:
            return kernels[ndim]
        except KeyError:
            have = ", ".join(f"{n}D" for n in sorted(kernels)) or "none"
            raise ValueError(f"the {self.name} edge weighting has no {ndim}D {role} kernel (has {have})") from None

    def gather_kernel(self, ndim: int) -> KernelFunction:
        return self._kernel(self.gather, ndim, "gather")

    def deposit_paths_kernel(self, ndim: int) -> KernelFunction:
        return self._kernel(self.deposit_paths, ndim, "deposit_paths")

    def _check(self, edges: torch.Tensor, grid: BlockGrid) -> int:
        """The number of dimensions of ``grid``, checking the shape of ``edges``."""
        _check_clamps(self, grid)
        ndim = len(grid.periodic)
        ends = grid.clamped or (False,) * ndim
        extra = 0 if self.degree is None else self.degree - 1
        expected = (*(int(n) + (extra if end else 0) for n, end in zip(grid.num_gridpoints, ends)), ndim)
        if tuple(edges.shape) != expected:
            raise ValueError(f"an edge field on this grid is {expected}, got {tuple(edges.shape)}")
        return ndim

    def gather_block(self, positions, edges: torch.Tensor, result: torch.Tensor, grid: BlockGrid) -> None:
        """Write the field of ``edges`` at ``positions`` (ndim, N) into ``result`` (ndim, N)."""
        kernel = self.gather_kernel(self._check(edges, grid))
        positions = _as_marker_tensor(positions, edges)
        kernel(positions, edges, result, *grid.geometry)

    def deposit_paths_block(self, start, end, charges, edges: torch.Tensor, grid: BlockGrid) -> None:
        """Add the current of ``charges`` (N,) moving from ``start`` to ``end`` (ndim, N) to ``edges``."""
        kernel = self.deposit_paths_kernel(self._check(edges, grid))
        start = _as_marker_tensor(start, edges)
        end = _as_marker_tensor(end, edges)
        charges = _as_marker_tensor(charges, edges).reshape(-1)
        if start.shape != end.shape or start.shape[-1] != charges.shape[0]:
            raise ValueError(
                f"paths from {tuple(start.shape)} to {tuple(end.shape)} for {charges.shape[0]} charges"
            )
        kernel(start, end, charges, edges, *grid.geometry)

    @staticmethod
    def gradient_block(nodes: torch.Tensor, grid: BlockGrid) -> torch.Tensor:
        """``G phi``: the difference of a node field along every edge (zero past a bounded end)."""
        ndim = len(grid.periodic)
        result = torch.zeros((*nodes.shape, ndim), dtype=nodes.dtype, device=nodes.device)
        for axis, periodic in enumerate(grid.periodic):
            if periodic:
                result[..., axis] = torch.roll(nodes, -1, dims=axis) - nodes
            else:
                n = nodes.shape[axis]
                result[..., axis].narrow(axis, 0, n - 1).copy_(
                    nodes.narrow(axis, 1, n - 1) - nodes.narrow(axis, 0, n - 1))
        return result

    @staticmethod
    def divergence_block(edges: torch.Tensor, grid: BlockGrid) -> torch.Tensor:
        """``G^T j``: the transpose of `gradient_block` (the change of the node charge)."""
        result = torch.zeros(edges.shape[:-1], dtype=edges.dtype, device=edges.device)
        for axis, periodic in enumerate(grid.periodic):
            flow = edges[..., axis]
            if periodic:
                result += torch.roll(flow, 1, dims=axis) - flow
            else:
                n = flow.shape[axis]
                result.narrow(axis, 0, n - 1).sub_(flow.narrow(axis, 0, n - 1))
                result.narrow(axis, 1, n - 1).add_(flow.narrow(axis, 0, n - 1))
        return result

    def __repr__(self) -> str:
        dims = sorted(set(self.gather) | set(self.deposit_paths))
        degree = "" if self.degree is None else f", degree={self.degree}"
        return f"EdgeWeighting({self.name!r}, ndim={tuple(dims)}, halo={self.halo}{degree})"


#: The lowest-order edge (Whitney) gather and path deposit, whose node space is LINEAR's.
WHITNEY = EdgeWeighting(
    "whitney",
    gather={n: EdgeGatherKernel(_lib.LINEAR, n, False) for n in (1, 2, 3)},
    deposit_paths={n: PathKernel(_lib.LINEAR, n, False) for n in (1, 2, 3)},
    halo=1,
    degree=1,
)


def _spline_edges(name: str, degree: int) -> EdgeWeighting:
    return EdgeWeighting(
        name,
        gather={n: _WithDegree(EdgeGatherKernel(_lib.SPLINE, n, True), degree) for n in (1, 2, 3)},
        deposit_paths={n: _WithDegree(PathKernel(_lib.SPLINE, n, True), degree) for n in (1, 2, 3)},
        halo=2,
        degree=degree,
        clamps=True,
    )


#: The edge weighting that goes with QUADRATIC (linear along an edge, quadratic across).
QUADRATIC_EDGES = _spline_edges("quadratic", 2)
#: The edge weighting that goes with CUBIC (quadratic along an edge, cubic across).
CUBIC_EDGES = _spline_edges("cubic", 3)
