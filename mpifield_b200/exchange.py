"""The halo exchange of a field split over ranks, one GPU each.

mpifield decomposes a field over MPI ranks with mpiarray: every rank stores its block of
the grid with ``h`` halo layers per side, and ``Field.fill_halos`` / ``Field.exchange_halos``
(src/mpifield/field.py:601-630) call mpiarray's ``update_halos`` (a halo takes the owned
layers of the neighbour it overlaps) and ``accumulate_halos`` (a halo adds onto the
neighbour's owned layers it overlaps, then is cleared). Here the ranks are the processes of
a ``torch.distributed`` group (NCCL over NVLink between GPUs; gloo in the CPU tests), the
face slabs are packed and unpacked by the library's kernels (``mpf_halo_pack``,
``mpf_halo_unpack``) and travel as point-to-point messages.

The grid is cut into a Cartesian grid of blocks, ``dims[d]`` along axis d, as evenly as
possible (the first ``num % dims`` blocks one node longer); rank r holds the block whose
coordinates are r unravelled row-major over ``dims``. Axis by axis, in order, over the whole
storage (halos of the earlier axes included, so that corners take two steps, as on one
process), the exchange is two shifts: towards the upper neighbour, then towards the lower.

- fill: a rank sends its last ``h`` owned layers up (the upper neighbour's low halo) and its
  first ``h`` down (the lower neighbour's high halo), and writes what it receives into its
  halos.
- fold: a rank sends its high halo up (added onto the upper neighbour's first owned layers)
  and its low halo down (onto the lower neighbour's last), adds what it receives onto its
  own owned layers, and clears its halos.

On a periodic axis the neighbours wrap around (a rank alone along the axis is its own
neighbour, and the exchange is the one-process fill and fold of ``mpf_halo_fill`` /
``mpf_halo_fold``); at the wall of a bounded axis there is no neighbour: fill leaves the
halo as it is and fold drops it. Every rank takes the same steps in the same order.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from mpifield_b200 import _lib


@dataclass(frozen=True)
class Decomposition:
    """The block of ``rank`` in a Cartesian split of ``num_gridpoints`` over ``dims``."""

    num_gridpoints: tuple
    periodic: tuple
    dims: tuple
    rank: int

    def __post_init__(self) -> None:
        n = len(self.num_gridpoints)
        if not 1 <= n <= 3 or len(self.periodic) != n or len(self.dims) != n:
            raise ValueError(f"num_gridpoints, periodic and dims must have 1-3 equal lengths, got "
                             f"{self.num_gridpoints}, {self.periodic}, {self.dims}")
        for num, d in zip(self.num_gridpoints, self.dims):
            if d < 1 or num < d:
                raise ValueError(f"cannot split {num} nodes into {d} blocks")
        if not 0 <= self.rank < self.size:
            raise ValueError(f"rank {self.rank} outside a grid of {self.size} blocks")

    @property
    def ndim(self) -> int:
        return len(self.dims)

    @property
    def size(self) -> int:
        total = 1
        for d in self.dims:
            total *= d
        return total

    def coords_of(self, rank: int) -> tuple:
        coords = []
        for d in reversed(self.dims):
            coords.append(rank % d)
            rank //= d
        return tuple(reversed(coords))

    def rank_of(self, coords) -> int:
        rank = 0
        for c, d in zip(coords, self.dims):
            rank = rank * d + c
        return rank

    @property
    def coords(self) -> tuple:
        return self.coords_of(self.rank)

    def _cut(self, axis: int, c: int) -> tuple[int, int]:
        num, d = self.num_gridpoints[axis], self.dims[axis]
        base, extra = divmod(num, d)
        return c * base + min(c, extra), base + (1 if c < extra else 0)

    @property
    def offset(self) -> tuple:
        """The global index of the block's first owned node, per axis."""
        return tuple(self._cut(a, c)[0] for a, c in enumerate(self.coords))

    @property
    def owned(self) -> tuple:
        """The block's owned nodes per axis."""
        return tuple(self._cut(a, c)[1] for a, c in enumerate(self.coords))

    def neighbours(self, axis: int) -> tuple:
        """The ranks below and above along ``axis`` (None at the wall of a bounded axis)."""
        coords = list(self.coords)
        out = []
        for step in (-1, 1):
            c = coords[axis] + step
            if not 0 <= c < self.dims[axis]:
                if not self.periodic[axis]:
                    out.append(None)
                    continue
                c %= self.dims[axis]
            moved = list(coords)
            moved[axis] = c
            out.append(self.rank_of(moved))
        return tuple(out)


def kernel_pack(storage: torch.Tensor, halo: int, axis: int, first: int, buffer: torch.Tensor) -> None:
    """buffer <- the layers [first, first + halo) along ``axis`` of ``storage`` (mpf_halo_pack)."""
    ndim, stored, ncomp = _layout(storage)
    status = _lib.library().mpf_halo_pack(storage.data_ptr(), ndim, stored, ncomp, halo, axis, first,
                                          buffer.data_ptr(), _lib.dtype_code(storage.dtype),
                                          _lib.stream_of(storage.device))
    _lib.check(status, "halo_pack")


def kernel_unpack(storage: torch.Tensor, halo: int, axis: int, first: int, buffer: torch.Tensor,
                  accumulate: bool) -> None:
    """The layers [first, first + halo) along ``axis`` <- (or +=) buffer (mpf_halo_unpack)."""
    ndim, stored, ncomp = _layout(storage)
    status = _lib.library().mpf_halo_unpack(storage.data_ptr(), ndim, stored, ncomp, halo, axis, first,
                                            buffer.data_ptr(), int(accumulate), _lib.dtype_code(storage.dtype),
                                            _lib.stream_of(storage.device))
    _lib.check(status, "halo_unpack")


def _layout(storage: torch.Tensor):
    if storage.dim() < 2 or not storage.is_contiguous():
        raise ValueError(f"a block's storage is a contiguous (stored..., ncomp) tensor, got {tuple(storage.shape)}")
    ndim = storage.dim() - 1
    return ndim, (C.c_int32 * ndim)(*storage.shape[:-1]), int(storage.shape[-1])


class HaloExchange:
    """fill / fold of the halos of this rank's block, exchanged with its neighbours.

    ``group``: the process group whose ranks hold the blocks (the default group when None);
    its rank r holds block r of ``decomposition``. ``pack`` / ``unpack``: the slab copies,
    the library's kernels unless given (tests on CPU ranks give their own).
    """

    def __init__(self, decomposition: Decomposition, halo: int, group=None, pack=None, unpack=None) -> None:
        if halo < 1:
            raise ValueError(f"halo must be >= 1, got {halo}")
        if any(m < halo for m in decomposition.owned):
            raise ValueError(f"blocks of {decomposition.owned} owned nodes are thinner than the halo {halo}")
        self.decomposition = decomposition
        self.halo = halo
        self.group = group
        self._pack = pack or kernel_pack
        self._unpack = unpack or kernel_unpack

    def _check(self, storage: torch.Tensor) -> None:
        stored = tuple(m + 2 * self.halo for m in self.decomposition.owned)
        if tuple(storage.shape[:-1]) != stored:
            raise ValueError(f"this rank's storage is {stored} + (ncomp,), got {tuple(storage.shape)}")

    def _slab(self, storage: torch.Tensor, axis: int) -> torch.Tensor:
        count = storage.numel() // storage.shape[axis] * self.halo
        return torch.empty(count, dtype=storage.dtype, device=storage.device)

    def _shift(self, send: torch.Tensor | None, to, receive: torch.Tensor | None, source) -> None:
        """One shift along an axis: at most one slab out and one in per rank."""
        me = self.decomposition.rank
        if to == me and source == me:
            receive.copy_(send)
            return
        import torch.distributed as dist

        ops = []
        if to is not None:
            peer = to if self.group is None else dist.get_global_rank(self.group, to)
            ops.append(dist.P2POp(dist.isend, send, peer, self.group))
        if source is not None:
            peer = source if self.group is None else dist.get_global_rank(self.group, source)
            ops.append(dist.P2POp(dist.irecv, receive, peer, self.group))
        if ops:
            for request in dist.batch_isend_irecv(ops):
                request.wait()

    def fill(self, storage: torch.Tensor) -> None:
        """Halos <- the neighbours' owned layers they overlap (update_halos)."""
        self._check(storage)
        h = self.halo
        for axis in range(self.decomposition.ndim):
            lower, upper = self.decomposition.neighbours(axis)
            if lower is None and upper is None:
                continue
            owned = storage.shape[axis] - 2 * h
            up = down = None
            if upper is not None:  # my last owned layers: the upper neighbour's low halo
                up = self._slab(storage, axis)
                self._pack(storage, h, axis, owned, up)
            if lower is not None:  # my first owned layers: the lower neighbour's high halo
                down = self._slab(storage, axis)
                self._pack(storage, h, axis, h, down)
            got_low = self._slab(storage, axis) if lower is not None else None
            got_high = self._slab(storage, axis) if upper is not None else None
            self._shift(up, upper, got_low, lower)
            self._shift(down, lower, got_high, upper)
            if got_low is not None:
                self._unpack(storage, h, axis, 0, got_low, False)
            if got_high is not None:
                self._unpack(storage, h, axis, owned + h, got_high, False)

    def fold(self, storage: torch.Tensor) -> None:
        """Halos added onto the neighbours' owned layers they overlap, then cleared
        (accumulate_halos); at a wall they are dropped."""
        self._check(storage)
        h = self.halo
        for axis in range(self.decomposition.ndim):
            lower, upper = self.decomposition.neighbours(axis)
            owned = storage.shape[axis] - 2 * h
            up = down = None
            if upper is not None:  # my high halo: onto the upper neighbour's first owned layers
                up = self._slab(storage, axis)
                self._pack(storage, h, axis, owned + h, up)
            if lower is not None:  # my low halo: onto the lower neighbour's last owned layers
                down = self._slab(storage, axis)
                self._pack(storage, h, axis, 0, down)
            got_low = self._slab(storage, axis) if lower is not None else None
            got_high = self._slab(storage, axis) if upper is not None else None
            if lower is not None or upper is not None:
                self._shift(up, upper, got_low, lower)
                self._shift(down, lower, got_high, upper)
            storage.narrow(axis, 0, h).zero_()
            storage.narrow(axis, owned + h, h).zero_()
            if got_low is not None:
                self._unpack(storage, h, axis, h, got_low, True)
            if got_high is not None:
                self._unpack(storage, h, axis, owned, got_high, True)
