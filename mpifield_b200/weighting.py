"""Weightings: a deposit (scatter) and its gather per number of dimensions.

The same plug-in type as mpifield's ``Weighting`` (src/mpifield/weighting.py:119-253):
``Weighting(name, scatter={ndim: kernel}, gather={ndim: kernel}, halo, degree, clamps)``
with ``scatter_block`` / ``gather_block`` on a `BlockGrid`, and the built-ins `LINEAR`,
`QUADRATIC` and `CUBIC` backed by the sm_100a kernels of this package. A weighting of
mpifield whose kernels are these (``mpifield.Weighting("linear", scatter=KERNELS...)``)
works the same; these objects take torch tensors on a CUDA device.
"""

from __future__ import annotations

from collections.abc import Callable, Mapping
from dataclasses import dataclass
from types import MappingProxyType
from typing import Any

import torch

from mpifield_b200 import _lib
from mpifield_b200._types import BlockGrid
from mpifield_b200.kernels import NodeKernel

__all__ = ["CUBIC", "LINEAR", "QUADRATIC", "Weighting"]

KernelFunction = Callable[..., Any]


def _frozen(kernels: Mapping[int, KernelFunction], role: str) -> Mapping[int, Any]:
    for ndim in kernels:
        if ndim not in (1, 2, 3):
            raise ValueError(f"{role} kernels are for 1, 2 or 3 dimensions, got {ndim}")
    return MappingProxyType(dict(kernels))


def _check_clamps(weighting: Any, grid: BlockGrid) -> None:
    """Raise if ``grid`` has a clamped axis that ``weighting``'s kernels do not take."""
    if any(grid.clamped) and not weighting.clamps:
        raise ValueError(
            f"the {weighting.name} weighting does not take clamped axes; use "
            "mpifield_b200.splines(degree, clamped=True)"
        )


@dataclass(frozen=True, eq=False, repr=False)
class Weighting:
    """A deposit and its gather, for each number of dimensions they cover.

    ``scatter`` and ``gather`` map 1, 2, 3 to kernels of the convention
    ``scatter(positions, values, field, *geometry)`` / ``gather(positions, field, result,
    *geometry)``; ``halo`` is ``(s + 1) // 2`` for a stencil of ``s`` nodes per axis,
    ``degree`` the B-spline degree, ``clamps`` whether the kernels take clamped axes.
    """

    name: str
    scatter: Mapping[int, KernelFunction]
    gather: Mapping[int, KernelFunction]
    halo: int = 1
    degree: int | None = None
    clamps: bool = False

    def __post_init__(self) -> None:
        if self.halo < 0:
            raise ValueError(f"halo must be >= 0, got {self.halo}")
        if self.degree is not None and self.degree < 0:
            raise ValueError(f"degree must be >= 0, got {self.degree}")
        object.__setattr__(self, "scatter", _frozen(self.scatter, "scatter"))
        object.__setattr__(self, "gather", _frozen(self.gather, "gather"))

    def _kernel(self, kernels: Mapping[int, KernelFunction], ndim: int, role: str):
        try:
            return kernels[ndim]
        except KeyError:
            have = ", ".join(f"{n}D" for n in sorted(kernels)) or "none"
            raise ValueError(f"the {self.name} weighting has no {ndim}D {role} kernel (has {have})") from None

    def scatter_kernel(self, ndim: int) -> KernelFunction:
        return self._kernel(self.scatter, ndim, "scatter")

    def gather_kernel(self, ndim: int) -> KernelFunction:
        return self._kernel(self.gather, ndim, "gather")

    def scatter_block(self, positions: torch.Tensor, values: torch.Tensor, field: torch.Tensor,
                      grid: BlockGrid) -> None:
        """Deposit ``values`` (ncomp, N) at ``positions`` (ndim, N) into ``field``, a block on ``grid``.

        A 1-D ``values`` is one component. The markers are moved to the field's device
        and dtype when they differ.
        """
        _check_clamps(self, grid)
        kernel = self.scatter_kernel(len(grid.periodic))
        positions = _as_marker_tensor(positions, field)
        values = _as_marker_tensor(values, field).reshape(-1, positions.shape[-1])
        kernel(positions, values, field, *grid.geometry)

    def gather_block(self, positions: torch.Tensor, field: torch.Tensor, result: torch.Tensor,
                     grid: BlockGrid) -> None:
        """Interpolate ``field``, a block on ``grid``, at ``positions`` into ``result`` (ncomp, N)."""
        _check_clamps(self, grid)
        kernel = self.gather_kernel(len(grid.periodic))
        positions = _as_marker_tensor(positions, field)
        if result.device != field.device or result.dtype != field.dtype:
            out = torch.empty(result.shape, dtype=field.dtype, device=field.device)
            kernel(positions, field, out, *grid.geometry)
            result.copy_(out)
            return
        kernel(positions, field, result, *grid.geometry)

    def __repr__(self) -> str:
        dims = sorted(set(self.scatter) | set(self.gather))
        degree = "" if self.degree is None else f", degree={self.degree}"
        return f"Weighting({self.name!r}, ndim={tuple(dims)}, halo={self.halo}{degree})"


def _as_marker_tensor(array, like: torch.Tensor) -> torch.Tensor:
    """A marker array as a tensor on ``like``'s device and dtype (no copy when it is one)."""
    if isinstance(array, torch.Tensor):
        if array.device == like.device and array.dtype == like.dtype:
            return array
        return array.to(device=like.device, dtype=like.dtype)
    return torch.as_tensor(array, dtype=like.dtype, device=like.device)


def _node_kernels(kind: int, degree: int, takes_degree: bool) -> tuple[dict, dict]:
    scatter, gather = {}, {}
    for n in (1, 2, 3):
        scatter[n] = NodeKernel("scatter", kind, n, False, degree)
        gather[n] = NodeKernel("gather", kind, n, False, degree)
    return scatter, gather


def spline_weighting(degree: int, name: str | None = None) -> Weighting:
    """The weighting of B-spline degree 0-3 on the spline kernels (codes 0, 1, 2)."""
    if degree not in (0, 1, 2, 3):
        raise ValueError(f"spline degrees are (0, 1, 2, 3), got {degree}")
    scatter, gather = _node_kernels(_lib.SPLINE, degree, False)
    return Weighting(name or f"spline{degree}", scatter=scatter, gather=gather,
                     halo=(degree + 2) // 2, degree=degree, clamps=degree >= 1)


_s, _g = _node_kernels(_lib.LINEAR, 1, False)
#: Linear (cloud-in-cell) weights: two nodes per axis (linear_cell.cuh arithmetic).
LINEAR = Weighting("linear", scatter=_s, gather=_g, halo=1, degree=1)

_s, _g = _node_kernels(_lib.QUADRATIC, 2, False)
#: Quadratic B-spline weights: the nearest node and its two neighbours (quadratic_cell.cuh).
QUADRATIC = Weighting("quadratic", scatter=_s, gather=_g, halo=2, degree=2)

_s, _g = _node_kernels(_lib.SPLINE, 3, False)
#: Cubic B-spline weights on the spline kernels (spline_cell.cuh, degree 3); takes clamped axes.
CUBIC = Weighting("cubic", scatter=_s, gather=_g, halo=2, degree=3, clamps=True)
del _s, _g
