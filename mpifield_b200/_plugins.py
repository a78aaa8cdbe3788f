"""What the plug-in types `Weighting` and `EdgeWeighting` have in common.

Both are named tables of kernels: for every role (``scatter`` and ``gather``, or
``gather`` and ``deposit_paths``) a read-only map from the number of dimensions (1, 2, 3)
to a kernel of mpifield's convention, plus the halo a split field needs, the B-spline
degree and whether the kernels take clamped axes. The argument checks and their
`ValueError` messages are those mpifield's types raise (src/mpifield/weighting.py:
83-97,150-164, src/mpifield/edges.py:66-135), so callers that catch or match them keep
working. Arrays on the host (markers given as NumPy arrays, lists or CPU tensors) are
moved to the field's device before a kernel runs, as mpifield moves markers to its
field's side.
"""

from __future__ import annotations

from types import MappingProxyType
from typing import Any

from mpifield_b200._arrays import as_device_array

DIMENSIONS = (1, 2, 3)


class KernelTable:
    """Mixin of the plug-in dataclasses: subclasses name their ``ROLES``, the noun of
    their messages and the lowest degree they accept."""

    ROLES: tuple[str, ...] = ()
    NOUN = "weighting"
    LOWEST_DEGREE = 0

    def __post_init__(self) -> None:
        if self.halo < 0:
            raise ValueError(f"halo must be >= 0, got {self.halo}")
        if self.degree is not None and self.degree < self.LOWEST_DEGREE:
            raise ValueError(f"degree must be >= {self.LOWEST_DEGREE}, got {self.degree}")
        for role in self.ROLES:
            table = dict(getattr(self, role))
            for ndim in table:
                if ndim not in DIMENSIONS:
                    raise ValueError(f"{role} kernels are for 1, 2 or 3 dimensions, got {ndim}")
            object.__setattr__(self, role, MappingProxyType(table))

    def kernel(self, role: str, ndim: int) -> Any:
        """The ``role`` kernel for ``ndim`` dimensions; ValueError when there is none."""
        table = getattr(self, role)
        found = table.get(ndim)
        if found is None:
            have = ", ".join(f"{n}D" for n in sorted(table)) or "none"
            raise ValueError(f"the {self.name} {self.NOUN} has no {ndim}D {role} kernel (has {have})")
        return found

    def dimensions(self) -> tuple[int, ...]:
        """The numbers of dimensions any role covers."""
        return tuple(sorted({n for role in self.ROLES for n in getattr(self, role)}))

    def accept_grid(self, grid) -> int:
        """The number of dimensions of ``grid``; ValueError for a clamped axis the kernels
        do not take."""
        if any(grid.clamped) and not self.clamps:
            raise ValueError(
                f"the {self.name} weighting does not take clamped axes; use "
                "mpifield_b200.splines(degree, clamped=True)")
        return len(grid.periodic)

    def __repr__(self) -> str:
        roles = "; ".join(f"{role} {'/'.join(f'{n}D' for n in sorted(getattr(self, role))) or '-'}"
                          for role in self.ROLES)
        degree = "" if self.degree is None else f", degree {self.degree}"
        clamps = ", takes clamped axes" if self.clamps else ""
        return f"{type(self).__name__}({self.name!r}: {roles}; halo {self.halo}{degree}{clamps})"


def on_device_of(array, like):
    """``array`` as a device array on the device of ``like`` (a device array): device
    arrays pass as they are; host arrays are copied to the device in ``like``'s type."""
    try:
        as_device_array(array)
        return array
    except TypeError:
        pass
    import torch

    target = as_device_array(like, "field").torch()
    return torch.as_tensor(array, dtype=target.dtype, device=target.device)


def is_device_array(array) -> bool:
    try:
        as_device_array(array)
    except TypeError:
        return False
    return True
