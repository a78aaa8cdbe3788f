"""`BlockGrid`: the grid of a block as the kernels see it.

The same value type as mpifield's ``BlockGrid`` (src/mpifield/_types.py:27-96): bounds,
spacing, node counts, periodic and clamped flags, and ``geometry``, the kernels' trailing
arguments ``(*lower, *cell_size, *num_nodes, *code)`` with code 0 bounded, 1 periodic,
2 clamped.
"""

from __future__ import annotations

from typing import NamedTuple

import numpy as np


class Bounds(NamedTuple):
    """The lower and upper corner of a grid block, one entry per axis."""

    lower_bound: np.ndarray
    upper_bound: np.ndarray


class BlockGrid(NamedTuple):
    """The grid of a block (halo nodes included), for the kernels.

    ``geometry`` is ``(*lower, *cell_size, *num_nodes, *code)``; ``index`` selects the
    nodes of the grid in a field's ``local_with_halos``; ``clamped`` marks the axes with
    clamped spline knots, where an array of degree p holds ``num_nodes + p - 1`` entries.
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
        """The grid of a whole array of ``num_nodes`` nodes from ``lower`` on."""
        lower = tuple(float(v) for v in lower)
        cell_size = tuple(float(v) for v in cell_size)
        num_nodes = tuple(int(n) for n in num_nodes)
        ndim = len(num_nodes)
        flags = (False,) * ndim if periodic is None else tuple(map(bool, periodic))
        ends = (False,) * ndim if clamped is None else tuple(map(bool, clamped))
        if not len(lower) == len(cell_size) == len(flags) == len(ends) == ndim:
            raise ValueError("lower, cell_size, num_nodes, periodic and clamped differ in length")
        if any(f and e for f, e in zip(flags, ends)):
            raise ValueError("an axis is either periodic or clamped")
        lower_bound = np.asarray(lower, dtype=float)
        spacing = np.asarray(cell_size, dtype=float)
        nodes = np.asarray(num_nodes, dtype=int)
        codes = tuple(2 if end else int(flag) for flag, end in zip(flags, ends))
        return cls(
            bounds=Bounds(lower_bound, lower_bound + (nodes - 1) * spacing),
            grid_spacing=spacing,
            num_gridpoints=nodes,
            periodic=flags,
            geometry=(*lower, *cell_size, *num_nodes, *codes),
            index=(slice(None),) * ndim,
            clamped=ends,
        )
