"""`Field`: a grid field on one GPU, with the particle-grid calls of mpifield's ``Field``.

The hot-path part of src/mpifield/field.py on one block (no decomposition across
GPUs): node storage with optional halo layers (``num_ghost_points``), `block_grid`
(field.py:150-245), `gather` (:1097-1126), `scatter` (:1128-1180), `deposit_density`
(:1182-1218), `node_volumes` (:563-588), `fill_halos` (:601-613) and `exchange_halos`
(:615-630). Node ``k`` of axis ``d`` is at ``lower[d] + k * h[d]``, with
``h = (upper - lower) / (N - 1)`` on a bounded axis and ``(upper - lower) / N`` on a
periodic one (the last node neighbours node 0). Storage is a torch tensor
``num_gridpoints + 2 h + (ncomp,)`` on a CUDA device; with halo layers the kernels see
the stored block as a bounded grid and a periodic axis is closed by `fill_halos` (before
a gather) and `exchange_halos` (after a deposit).
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from mpifield_b200 import _lib
from mpifield_b200._types import BlockGrid, Bounds
from mpifield_b200.weighting import LINEAR, Weighting

__all__ = ["Field"]


def _markers_on(array, like: torch.Tensor) -> torch.Tensor:
    """A marker array as a torch tensor on ``like``'s device in its dtype (no copy when it
    is one already; device arrays of other producers are viewed, host arrays copied)."""
    if isinstance(array, torch.Tensor):
        return array if (array.device, array.dtype) == (like.device, like.dtype) else array.to(like.device, like.dtype)
    return torch.as_tensor(array, dtype=like.dtype, device=like.device)


def _per_axis(value, ndim: int, name: str) -> tuple:
    if np.isscalar(value):
        return (value,) * ndim
    value = tuple(value)
    if len(value) != ndim:
        raise ValueError(f"{name} needs {ndim} entries, got {len(value)}")
    return value


class Field:
    """A field of ``num_components`` values per node on a uniform grid, on one GPU."""

    def __init__(self, ndim: int, lower_bound, upper_bound, num_gridpoints, num_components: int = 1,
                 periodic=None, num_ghost_points: int = 0, dtype: torch.dtype = torch.float64,
                 device: torch.device | str | None = None) -> None:
        if ndim not in (1, 2, 3):
            raise ValueError(f"ndim must be 1, 2 or 3, got {ndim}")
        if num_components < 1:
            raise ValueError(f"num_components must be >= 1, got {num_components}")
        if num_ghost_points < 0:
            raise ValueError(f"num_ghost_points must be >= 0, got {num_ghost_points}")
        self.ndim = ndim
        self.lower = np.asarray(_per_axis(lower_bound, ndim, "lower_bound"), dtype=float)
        self.upper = np.asarray(_per_axis(upper_bound, ndim, "upper_bound"), dtype=float)
        self.num_gridpoints = tuple(int(n) for n in _per_axis(num_gridpoints, ndim, "num_gridpoints"))
        flags = (False,) * ndim if periodic is None else _per_axis(periodic, ndim, "periodic")
        self.periodic = tuple(bool(f) for f in flags)
        self.num_components = int(num_components)
        self.num_ghost_points = int(num_ghost_points)
        self.dtype = dtype
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        n = np.asarray(self.num_gridpoints, dtype=float)
        self.grid_spacing = np.where(self.periodic, (self.upper - self.lower) / n,
                                     (self.upper - self.lower) / np.maximum(n - 1, 1))
        h = self.num_ghost_points
        shape = tuple(m + 2 * h for m in self.num_gridpoints) + (self.num_components,)
        self.local_with_halos = torch.zeros(shape, dtype=dtype, device=self.device)
        # a field split over ranks: its block's halo exchange (mpifield_b200.exchange), which
        # fill_halos / exchange_halos then run instead of the one-process kernels
        self.exchange = None

    # ------------------------------------------------------------------ storage --

    @property
    def distributed(self) -> bool:
        """Always False: one block on one GPU."""
        return False

    @property
    def local(self) -> torch.Tensor:
        """The owned nodes, without halo layers: a writable view."""
        h = self.num_ghost_points
        index = tuple(slice(h, h + m) for m in self.num_gridpoints)
        return self.local_with_halos[index]

    @property
    def bounds(self) -> Bounds:
        return Bounds(self.lower, self.upper)

    def set_field_data(self, data) -> None:
        """Set the owned nodes from a scalar or a ``num_gridpoints (+ (ncomp,))`` array; zero the halos."""
        self.local_with_halos.zero_()
        if np.isscalar(data):
            self.local.fill_(float(data))
            return
        data = torch.as_tensor(data, dtype=self.dtype, device=self.device)
        if data.dim() == self.ndim:
            data = data.unsqueeze(-1)
        self.local.copy_(data.expand_as(self.local))

    def _like(self, num_components: int | None = None) -> Field:
        return Field(self.ndim, self.lower, self.upper, self.num_gridpoints,
                     num_components or self.num_components, self.periodic, self.num_ghost_points,
                     self.dtype, self.device)

    def block_grid(self, inside_domain: bool = False) -> BlockGrid:
        """The grid of the stored block, halo layers included, for the kernels.

        With halo layers the block starts ``h`` nodes before node 0 and is bounded for the
        kernels; with ``inside_domain`` the halo layers beyond a bounded edge are left out
        (field.py:150-202).
        """
        h = self.num_ghost_points
        first, last = [], []
        for axis in range(self.ndim):
            trim = inside_domain and not self.periodic[axis]
            low = h if trim else 0
            high = h if trim else 0
            first.append(low)
            last.append(self.num_gridpoints[axis] + 2 * h - high)
        spacing = self.grid_spacing
        lower = self.lower + (np.asarray(first) - h) * spacing
        nodes = np.asarray([b - a for a, b in zip(first, last)], dtype=int)
        periodic = tuple(p and h == 0 for p in self.periodic)
        return BlockGrid(
            bounds=Bounds(lower, lower + (nodes - 1) * spacing),
            grid_spacing=spacing,
            num_gridpoints=nodes,
            periodic=periodic,
            geometry=(*(float(v) for v in lower), *(float(v) for v in spacing), *(int(n) for n in nodes),
                      *(int(p) for p in periodic)),
            index=tuple(slice(a, b) for a, b in zip(first, last)),
        )

    # --------------------------------------------------------- gather / scatter --

    def _marker_positions(self, positions) -> torch.Tensor:
        positions = _markers_on(positions, self.local_with_halos)
        if positions.dim() == 1:
            if self.ndim == 1:
                return positions.reshape(1, -1)
            if positions.shape[0] != self.ndim:
                raise ValueError(f"Expected {self.ndim} coordinates, got {positions.shape[0]}")
            return positions.reshape(self.ndim, 1)
        if positions.dim() != 2 or positions.shape[0] != self.ndim:
            raise ValueError(f"Expected positions with shape ({self.ndim}, N), got {tuple(positions.shape)}")
        return positions

    def _marker_values(self, values, count: int) -> torch.Tensor:
        if isinstance(values, (int, float)):
            return torch.full((self.num_components, count), float(values), dtype=self.dtype, device=self.device)
        values = _markers_on(values, self.local_with_halos)
        if values.dim() == 1:
            if values.shape[0] == count:
                values = values.reshape(1, count)
            elif count == 1 and values.shape[0] == self.num_components:
                values = values.reshape(self.num_components, 1)
            else:
                raise ValueError(f"Expected {count} values (or {self.num_components} components of one marker), "
                                 f"got {tuple(values.shape)}")
        elif values.dim() != 2 or values.shape[1] != count:
            raise ValueError(f"Expected values with shape ({self.num_components}, {count}), got {tuple(values.shape)}")
        if values.shape[0] != self.num_components:
            raise ValueError(f"Expected {self.num_components} components, got {values.shape[0]}")
        return values

    def gather(self, positions, weighting: Weighting = LINEAR) -> torch.Tensor:
        """Interpolate the field at ``positions`` (ndim, N): a new ``(ncomp, N)`` tensor.

        With halo layers, fill them first (`fill_halos`) for markers near a periodic seam.
        """
        positions = self._marker_positions(positions)
        grid = self.block_grid(inside_domain=True)
        result = torch.empty((self.num_components, positions.shape[1]), dtype=self.dtype, device=self.device)
        weighting.gather_block(positions, self.local_with_halos[grid.index], result, grid)
        return result

    def scatter(self, positions, values, weighting: Weighting = LINEAR) -> None:
        """Add marker values into the stored block (halo layers included); dead markers skipped.

        With halo layers, call `exchange_halos` afterwards to fold the halos back.
        """
        positions = self._marker_positions(positions)
        values = self._marker_values(values, positions.shape[1])
        grid = self.block_grid(inside_domain=True)
        target = self.local_with_halos[grid.index]
        weighting.scatter_block(positions, values, target, grid)

    def deposit_density(self, positions, values, weighting: Weighting = LINEAR) -> None:
        """Add the density of the marker values: a deposit divided by the node volumes.

        The deposit goes into a zero field like this one; with halo layers they are folded
        back (`exchange_halos`); then ``local += deposit / volume`` in one kernel.
        """
        deposit = self._like()
        deposit.scatter(positions, values, weighting)
        if self.num_ghost_points > 0:
            deposit.exchange_halos()
        h = self.num_ghost_points
        num = (C.c_int32 * self.ndim)(*self.num_gridpoints)
        cell = (C.c_double * self.ndim)(*(float(v) for v in self.grid_spacing))
        per = (C.c_int32 * self.ndim)(*(int(p) for p in self.periodic))
        status = _lib.library().mpf_add_density(
            self.local_with_halos.data_ptr(), deposit.local_with_halos.data_ptr(), self.ndim, num, h,
            self.num_components, cell, per, _lib.dtype_code(self.dtype), _lib.stream_of(self.device))
        _lib.check(status, "deposit_density")

    def node_volumes(self) -> Field:
        """The volume each node collects: prod(h), halved on the ends of a bounded axis."""
        volumes = self._like(num_components=1)
        local = torch.ones(self.num_gridpoints, dtype=self.dtype, device=self.device)
        for axis in range(self.ndim):
            factor = torch.full((self.num_gridpoints[axis],), float(self.grid_spacing[axis]),
                                dtype=self.dtype, device=self.device)
            if not self.periodic[axis]:
                factor[0] *= 0.5
                factor[-1] *= 0.5
            shape = [1] * self.ndim
            shape[axis] = -1
            local = local * factor.reshape(shape)
        volumes.local[..., 0] = local
        if self.num_ghost_points > 0:
            volumes.fill_halos()
        return volumes

    # --------------------------------------------------------------------- halos --

    def _halo_call(self, name: str) -> None:
        h = self.num_ghost_points
        if h == 0:
            return
        stored = (C.c_int32 * self.ndim)(*(m + 2 * h for m in self.num_gridpoints))
        per = (C.c_int32 * self.ndim)(*(int(p) for p in self.periodic))
        fn = getattr(_lib.library(), name)
        status = fn(self.local_with_halos.data_ptr(), self.ndim, stored, self.num_components, h, per,
                    _lib.dtype_code(self.dtype), _lib.stream_of(self.device))
        _lib.check(status, name)

    def fill_halos(self) -> None:
        """Fill the halo layers of periodic axes from the wrapped owned nodes (update_halos);
        for a field split over ranks, from the neighbours' owned nodes."""
        if self.exchange is not None:
            self.exchange.fill(self.local_with_halos)
            return
        self._halo_call("mpf_halo_fill")

    def exchange_halos(self) -> None:
        """Add the halo layers onto their wrapped owners and clear them (accumulate_halos)."""
        if self.exchange is not None:
            self.exchange.fold(self.local_with_halos)
            return
        self._halo_call("mpf_halo_fold")

    def __repr__(self) -> str:
        return (f"Field(ndim={self.ndim}, num_gridpoints={self.num_gridpoints}, "
                f"num_components={self.num_components}, periodic={self.periodic}, "
                f"num_ghost_points={self.num_ghost_points}, dtype={self.dtype})")
