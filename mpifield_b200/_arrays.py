"""Device arrays of any CUDA producer, seen without a copy, and the stream a call runs on.

mpifield hands its kernels CuPy arrays on the GPU (``cunumpy.kernels.as_kernel_array``,
src/mpifield/weighting.py:205-213) and launches them on CuPy's current stream. This
backend's kernels take what a caller has: a torch tensor on a CUDA device, any object
with ``__cuda_array_interface__`` (versions 2 and 3: CuPy, Numba, JAX, ...) or with
``__dlpack__``. Each is read into a `DeviceArray` -- its address, shape, strides in
elements and element type -- and the kernels work on those, so a layout the C calls take
as it is (unit column stride, rows any distance apart, C-contiguous grids) is never
copied. Only a layout they do not take is copied, through torch, on the launch stream.

The launch stream is, in this order: the stream of an active `use_stream` block; the
``stream`` an array interface (version 3) names, the one its producer works on (1 and 2
are CUDA's legacy and per-thread default streams); CuPy's current stream for interface
arrays when CuPy is importable; the legacy default stream for other interface arrays;
torch's current stream for torch tensors.
"""

from __future__ import annotations

import contextlib
import threading
from functools import lru_cache

_TYPES = {"<f8": "f8", "<f4": "f4", "<i4": "i4", "<u4": "u4", "<i8": "i8", "|u1": "u1", "<u1": "u1",
          "|i1": "i1"}
_SIZES = {"f8": 8, "f4": 4, "i4": 4, "u4": 4, "i8": 8, "u1": 1, "i1": 1}
_TORCH_NAMES = {"float64": "f8", "float32": "f4", "int32": "i4", "int64": "i8", "uint8": "u1", "int8": "i1",
                "uint32": "u4"}

_local = threading.local()


class DeviceArray:
    """A strided view of device memory: ``ptr`` is the address of element (0, ..., 0),
    ``strides`` are in elements. ``source`` is the object it was read from, ``stream``
    the stream its producer named (None: none named), ``device`` the CUDA device index
    (None: the current one). A plain slotted record: one is made per array and call."""

    __slots__ = ("ptr", "shape", "strides", "dtype", "source", "stream", "device")

    def __init__(self, ptr: int, shape: tuple, strides: tuple, dtype: str, source: object,
                 stream: int | None = None, device: int | None = None) -> None:
        self.ptr, self.shape, self.strides, self.dtype = ptr, shape, strides, dtype
        self.source, self.stream, self.device = source, stream, device

    @property
    def ndim(self) -> int:
        return len(self.shape)

    @property
    def itemsize(self) -> int:
        return _SIZES[self.dtype]

    @property
    def size(self) -> int:
        total = 1
        for n in self.shape:
            total *= n
        return total

    def is_contiguous(self) -> bool:
        """C-contiguous (axes of length 1 may have any stride)."""
        expected = 1
        for n, s in zip(reversed(self.shape), reversed(self.strides)):
            if n != 1 and s != expected:
                return False
            expected *= n
        return True

    def reshaped(self, shape: tuple[int, ...]) -> DeviceArray:
        """The same memory with another shape (C-contiguous arrays only)."""
        if not self.is_contiguous():
            raise ValueError("only a C-contiguous array can be reshaped without a copy")
        total = 1
        for n in shape:
            total *= n
        if total != self.size:
            raise ValueError(f"cannot view {self.shape} as {shape}")
        strides, step = [], 1
        for n in reversed(shape):
            strides.append(step)
            step *= n
        return DeviceArray(self.ptr, tuple(shape), tuple(reversed(strides)), self.dtype, self.source, self.stream,
                           self.device)

    def torch(self):
        """A torch tensor over the same memory (for the copies of layouts the C calls do
        not take; needs a CUDA device)."""
        import torch

        src = self.source
        if isinstance(src, torch.Tensor) and src.data_ptr() == self.ptr and tuple(src.shape) == self.shape \
                and tuple(src.stride()) == self.strides:
            return src
        base = torch.as_tensor(src, device="cuda" if self.device is None else f"cuda:{self.device}")
        offset = base.storage_offset() + (self.ptr - base.data_ptr()) // self.itemsize
        return base.as_strided(self.shape, self.strides, offset)


@lru_cache(maxsize=256)
def _c_strides(shape: tuple) -> tuple:
    """The element strides of a C-contiguous array of ``shape``."""
    strides, step = [], 1
    for n in reversed(shape):
        strides.append(step)
        step *= n
    return tuple(reversed(strides))


def _from_interface(obj, iface: dict) -> DeviceArray:
    dtype = _TYPES.get(iface["typestr"])
    if dtype is None:
        raise TypeError(f"mpifield_b200 kernels take float64 or float32 arrays, got type {iface['typestr']!r}")
    if iface.get("mask") is not None:
        raise TypeError("masked device arrays are not supported")
    size = _SIZES[dtype]
    shape = tuple(iface["shape"])
    raw = iface.get("strides")
    if raw is None:
        strides = _c_strides(shape)
    else:
        if any(s % size for s in raw):
            raise ValueError(f"strides {tuple(raw)} are not whole elements of {size} bytes")
        strides = tuple(s // size for s in raw)
    ptr = int(iface["data"][0] or 0)
    stream = iface.get("stream") if int(iface.get("version", 2)) >= 3 else None
    return DeviceArray(ptr, shape, strides, dtype, obj, None if stream is None else int(stream))


def as_device_array(obj, name: str = "array") -> DeviceArray:
    """``obj`` as a `DeviceArray`; raises TypeError for host memory (there is no CPU
    fallback) and for objects that are not device arrays."""
    if isinstance(obj, DeviceArray):
        return obj
    torch = _torch_module()
    if torch is not None and isinstance(obj, torch.Tensor):
        if not obj.is_cuda:
            raise TypeError(
                f"mpifield_b200 runs on CUDA device arrays only (no CPU fallback); {name} is on {obj.device}")
        dtype = _TORCH_DTYPES.get(obj.dtype)
        if dtype is None:
            raise TypeError(f"mpifield_b200 kernels take float64 or float32 arrays, got {obj.dtype}")
        return DeviceArray(obj.data_ptr(), tuple(obj.shape), obj.stride(), dtype, obj, None, obj.get_device())
    iface = getattr(obj, "__cuda_array_interface__", None)
    if iface is not None:
        return _from_interface(obj, iface)
    if hasattr(obj, "__dlpack__") and torch is not None:
        device = getattr(obj, "__dlpack_device__", lambda: (0, 0))()
        if device[0] != 2:  # kDLCUDA
            raise TypeError(f"mpifield_b200 runs on CUDA device arrays only (no CPU fallback); {name} is not")
        return as_device_array(torch.from_dlpack(obj), name)
    raise TypeError(
        f"mpifield_b200 runs on CUDA device arrays only (a torch tensor on a CUDA device, or an object with "
        f"__cuda_array_interface__ or __dlpack__); {name} is a {type(obj).__name__}")


_TORCH = None
_TORCH_DTYPES: dict = {}
_RAW_STREAM = None


def _torch_module():
    """torch (imported once), with its dtype table and its raw current-stream query."""
    global _TORCH, _RAW_STREAM
    if _TORCH is None:
        try:
            import torch
        except ImportError:  # pragma: no cover
            return None
        for name, code in _TORCH_NAMES.items():
            _TORCH_DTYPES[getattr(torch, name)] = code
        _RAW_STREAM = getattr(torch._C, "_cuda_getCurrentRawStream", None)
        _TORCH = torch
    return _TORCH


def _cupy_stream() -> int | None:
    try:
        import cupy
    except ImportError:
        return None
    return int(cupy.cuda.get_current_stream().ptr)


def launch_stream(*arrays: DeviceArray) -> int:
    """The raw cudaStream_t a call on ``arrays`` runs on (see the module docstring)."""
    chosen = getattr(_local, "stream", None)
    if chosen is not None:
        return chosen
    for a in arrays:
        if a.stream is not None:
            return a.stream
    torch = _torch_module()
    if torch is None or any(not isinstance(a.source, torch.Tensor) for a in arrays):
        cupy = _cupy_stream()
        return 0 if cupy is None else cupy
    torch = _torch_module()
    device = next((a.device for a in arrays if a.device is not None), None)
    if _RAW_STREAM is not None:
        return int(_RAW_STREAM(torch.cuda.current_device() if device is None else device))
    return int(torch.cuda.current_stream(device).cuda_stream)


def _is_torch(obj) -> bool:
    torch = _torch_module()
    return torch is not None and isinstance(obj, torch.Tensor)


@contextlib.contextmanager
def use_stream(stream):
    """Run the calls of this block on ``stream``: a raw cudaStream_t (int), or an object
    with ``.cuda_stream`` (torch) or ``.ptr`` (CuPy)."""
    handle = int(getattr(stream, "cuda_stream", getattr(stream, "ptr", stream)))
    previous = getattr(_local, "stream", None)
    _local.stream = handle
    try:
        yield handle
    finally:
        _local.stream = previous


@contextlib.contextmanager
def torch_on(stream: int):
    """torch work (the copies of layouts the C calls do not take) on the launch stream."""
    import torch

    # 0 and 1 are the legacy default stream, torch's default stream
    target = torch.cuda.default_stream() if stream in (0, 1) else torch.cuda.ExternalStream(stream)
    with torch.cuda.stream(target):
        yield
