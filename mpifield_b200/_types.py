"""The grid of a block as the kernels see it: `Bounds` and `BlockGrid`.

Code written against mpifield reads a grid through the fields of its ``BlockGrid``
(src/mpifield/_types.py:27-96): the same names in the same order, and the same
``from_geometry`` arguments and errors, are kept here. The grid is built from one
`_Axis` record per axis; ``geometry`` is what the kernels take after their arrays,
``(*lower, *cell_size, *num_nodes, *code)`` with the boundary codes 0 (bounded),
1 (periodic) and 2 (clamped spline knots).
"""

from __future__ import annotations

from itertools import zip_longest
from typing import NamedTuple

import numpy as np

BOUNDED, PERIODIC, CLAMPED = 0, 1, 2


class Bounds(NamedTuple):
    """Positions of a block's first node (``lower_bound``) and last node (``upper_bound``)
    along every axis."""

    lower_bound: np.ndarray
    upper_bound: np.ndarray


class _Axis(NamedTuple):
    """One axis of a grid: first node, spacing, node count and boundary code."""

    first: float
    step: float
    count: int
    code: int

    @property
    def last(self) -> float:
        return self.first + (self.count - 1) * self.step


def _flags(values, ndim: int) -> tuple[bool, ...]:
    return (False,) * ndim if values is None else tuple(bool(v) for v in values)


def _axes(lower, cell_size, num_nodes, periodic, clamped) -> list[_Axis]:
    counts = [int(n) for n in num_nodes]
    ndim = len(counts)
    rows = list(zip_longest(lower, cell_size, counts, _flags(periodic, ndim), _flags(clamped, ndim)))
    if any(None in row for row in rows):
        raise ValueError("lower, cell_size, num_nodes, periodic and clamped differ in length")
    axes = []
    for first, step, count, wraps, knots in rows:
        if wraps and knots:
            raise ValueError("an axis is either periodic or clamped")
        code = CLAMPED if knots else (PERIODIC if wraps else BOUNDED)
        axes.append(_Axis(float(first), float(step), count, code))
    return axes


class BlockGrid(NamedTuple):
    """The nodes of a block, halo nodes included, as the kernels address them.

    ``geometry`` is the kernels' trailing arguments; ``index`` picks the grid's nodes out
    of a stored array with halos; ``clamped`` flags the axes with clamped spline knots,
    along which an array of degree p holds ``num_nodes + p - 1`` coefficients.
    """

    bounds: Bounds
    grid_spacing: np.ndarray
    num_gridpoints: np.ndarray
    periodic: tuple[bool, ...]
    geometry: tuple[float | int, ...]
    index: tuple[slice, ...]
    clamped: tuple[bool, ...] = ()

    @classmethod
    def from_geometry(cls, lower, cell_size, num_nodes, periodic=None, clamped=None) -> BlockGrid:
        """The grid of a whole array: ``num_nodes`` nodes per axis from ``lower`` on,
        ``cell_size`` apart; axes bounded unless ``periodic`` or ``clamped`` flags them."""
        axes = _axes(lower, cell_size, num_nodes, periodic, clamped)
        first = np.array([a.first for a in axes], dtype=float)
        return cls(
            bounds=Bounds(first, np.array([a.last for a in axes], dtype=float)),
            grid_spacing=np.array([a.step for a in axes], dtype=float),
            num_gridpoints=np.array([a.count for a in axes], dtype=int),
            periodic=tuple(a.code == PERIODIC for a in axes),
            geometry=(*(a.first for a in axes), *(a.step for a in axes), *(a.count for a in axes),
                      *(a.code for a in axes)),
            index=tuple(slice(None) for _ in axes),
            clamped=tuple(a.code == CLAMPED for a in axes),
        )
