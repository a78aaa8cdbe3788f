"""Node weightings on the B200 kernels: `Weighting`, `LINEAR`, `QUADRATIC`, `CUBIC`.

A `Weighting` is mpifield's plug-in type for deposits and gathers on the nodes
(src/mpifield/weighting.py:119-253): ``Weighting(name, scatter={ndim: kernel},
gather={ndim: kernel}, halo, degree, clamps)``, run on a block by `scatter_block` and
`gather_block`. The built-ins are backed by this package's kernels (`kernels.NodeKernel`),
whose arithmetic is that of mpifield's linear_cell.cuh (LINEAR), quadratic_cell.cuh
(QUADRATIC) and spline_cell.cuh (CUBIC and `spline_weighting`). The same kernels plug
into mpifield's own ``Weighting`` through `KERNELS`.
"""

from __future__ import annotations

from collections.abc import Callable, Mapping
from dataclasses import dataclass
from typing import Any

from mpifield_b200 import _lib
from mpifield_b200._plugins import KernelTable, is_device_array, on_device_of
from mpifield_b200._types import BlockGrid
from mpifield_b200.kernels import NodeKernel

__all__ = ["CUBIC", "LINEAR", "QUADRATIC", "Weighting", "spline_weighting"]

KernelFunction = Callable[..., Any]


@dataclass(frozen=True, eq=False, repr=False)
class Weighting(KernelTable):
    """Deposit (``scatter``) and gather kernels by number of dimensions.

    Kernels follow the convention ``scatter(positions, values, field, *geometry)``
    (adding) and ``gather(positions, field, result, *geometry)`` (overwriting).
    ``halo`` is the halo width a split field needs, ``(s + 1) // 2`` for ``s`` stencil
    nodes per axis; ``degree`` the B-spline degree, None for other shapes; ``clamps``
    whether the kernels take clamped axes (boundary code 2).
    """

    ROLES = ("scatter", "gather")

    name: str
    scatter: Mapping[int, KernelFunction]
    gather: Mapping[int, KernelFunction]
    halo: int = 1
    degree: int | None = None
    clamps: bool = False

    def scatter_kernel(self, ndim: int) -> KernelFunction:
        return self.kernel("scatter", ndim)

    def gather_kernel(self, ndim: int) -> KernelFunction:
        return self.kernel("gather", ndim)

    def scatter_block(self, positions, values, field, grid: BlockGrid) -> None:
        """Add the deposit of ``values`` (ncomp, N), or (N,) for one component, at
        ``positions`` (ndim, N) to ``field``, a device array on ``grid``."""
        run = self.scatter_kernel(self.accept_grid(grid))
        run(on_device_of(positions, field), on_device_of(values, field), field, *grid.geometry)

    def gather_block(self, positions, field, result, grid: BlockGrid) -> None:
        """Write ``field`` (a device array on ``grid``) interpolated at ``positions`` into
        ``result`` (ncomp, N), which may be on the host or the device."""
        run = self.gather_kernel(self.accept_grid(grid))
        positions = on_device_of(positions, field)
        if is_device_array(result):
            run(positions, field, result, *grid.geometry)
            return
        import numpy as np
        import torch

        shape = tuple(np.shape(result))
        staged = on_device_of(torch.empty(shape, dtype=torch.float64), field)
        run(positions, field, staged, *grid.geometry)
        host = staged.cpu()
        if isinstance(result, torch.Tensor):
            result.copy_(host)
        else:
            np.copyto(result, host.numpy())


def _node_tables(kind: int, degree: int) -> tuple[dict, dict]:
    """The scatter and gather tables of a stencil kind at a fixed degree, 1D to 3D."""
    return ({n: NodeKernel("scatter", kind, n, False, degree) for n in (1, 2, 3)},
            {n: NodeKernel("gather", kind, n, False, degree) for n in (1, 2, 3)})


def spline_weighting(degree: int, name: str | None = None) -> Weighting:
    """The B-spline weighting of degree 0-3 on the spline kernels (every boundary code,
    clamped axes from degree 1 on)."""
    if degree not in (0, 1, 2, 3):
        raise ValueError(f"spline degrees are (0, 1, 2, 3), got {degree}")
    scatter, gather = _node_tables(_lib.SPLINE, degree)
    return Weighting(name or f"spline{degree}", scatter=scatter, gather=gather, halo=(degree + 2) // 2,
                     degree=degree, clamps=degree >= 1)


#: Cloud-in-cell: the two nearest nodes per axis (linear_cell.cuh).
LINEAR = Weighting("linear", *_node_tables(_lib.LINEAR, 1), halo=1, degree=1)
#: The quadratic B-spline: the nearest node and its two neighbours per axis (quadratic_cell.cuh).
QUADRATIC = Weighting("quadratic", *_node_tables(_lib.QUADRATIC, 2), halo=2, degree=2)
#: The cubic B-spline on the spline kernels (spline_cell.cuh, degree 3); takes clamped axes.
CUBIC = spline_weighting(3, "cubic")
