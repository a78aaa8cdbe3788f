"""Loading of the CUDA backend (``libmpifield_b200.so``) and its C ABI.

The library is built in-tree by ``mpifield_b200/build.py``; there is no CPU fallback: if
the library is missing or no CUDA device is present, every call raises.
"""

from __future__ import annotations

import ctypes as C
import functools
import threading
from pathlib import Path

import torch

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "libmpifield_b200.so"

OK = 0
ERR_ARGUMENT = 1
ERR_SHAPE = 2
ERR_ALIGNMENT = 3
ERR_WORKSPACE = 4
ERR_CUDA = 5
ERR_UNSUPPORTED = 6
ERR_TIMEOUT = 7

LINEAR, QUADRATIC, SPLINE = 0, 1, 2
F64, F32 = 0, 1
PATH_AUTO, PATH_DIRECT, PATH_STAGED = 0, 1, 2


class BackendError(RuntimeError):
    """A status other than MPF_OK from the backend that is not an argument error."""


class Tuning(C.Structure):
    """``mpf_tuning``: the path, CTA size, shared memory, CTAs per SM, kernel variant and wait limit of a launch."""

    _fields_ = [("path", C.c_int32), ("block", C.c_int32), ("smem_bytes", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("variant", C.c_int32), ("wait_limit", C.c_int32)]


class BatchRequest(C.Structure):
    """``mpf_batch_request``: one request of a serving batch (a device table entry)."""

    _fields_ = [("op", C.c_int32), ("kind", C.c_int32), ("degree", C.c_int32), ("ndim", C.c_int32),
                ("ncomp", C.c_int32), ("reserved", C.c_int32), ("n", C.c_int64), ("first_tile", C.c_int64),
                ("positions", C.c_void_p), ("pos_stride", C.c_int64), ("values", C.c_void_p),
                ("val_stride", C.c_int64), ("field", C.c_void_p), ("out", C.c_void_p), ("out_stride", C.c_int64),
                ("lower", C.c_double * 3), ("cell", C.c_double * 3), ("inv", C.c_double * 3),
                ("num", C.c_int32 * 3), ("code", C.c_int32 * 3), ("ext", C.c_int32 * 3), ("pad", C.c_int32)]


class BatchHeader(C.Structure):
    """``mpf_batch_header``: table size, tiles, markers per tile and the work counters."""

    _fields_ = [("requests", C.c_int64), ("tiles", C.c_int64), ("tile_markers", C.c_int64),
                ("next_tile", C.c_int64), ("finished", C.c_int64), ("pad", C.c_int64 * 3)]


OP_GATHER, OP_SCATTER, OP_PATHS = 0, 1, 2

_P = C.c_void_p
_I = C.c_int
_L = C.c_int64
_SIGNATURES = {
    "mpf_version": ([], _I),
    "mpf_launch_count": ([], _L),
    "mpf_last_error": ([], C.c_char_p),
    "mpf_device_errors": ([_I, _P], _I),
    "mpf_status_string": ([_I], C.c_char_p),
    "mpf_gather": ([_I, _I, _I, _P, _L, _L, _P, _L, _P, _L, _P, _P, _P, _P, _I, _P, _P], _I),
    "mpf_scatter": ([_I, _I, _I, _P, _L, _P, _L, _L, _P, _L, _P, _P, _P, _P, _I, _P, _P], _I),
    "mpf_gather_tiles": ([_I, _I, _I, _P, _L, _L, _P, _L, _P, _L, _P, _P, _P, _P, _P, _P, _I, _P, _P], _I),
    "mpf_scatter_tiles": ([_I, _I, _I, _P, _L, _P, _L, _L, _P, _L, _P, _P, _P, _P, _P, _P, _I, _P, _P], _I),
    "mpf_gather_grad": ([_I, _I, _I, _P, _L, _L, _P, _L, _P, _L, _P, _L, _P, _P, _P, _P, _I, _P], _I),
    "mpf_deposit_paths": ([_I, _I, _I, _P, _L, _P, _L, _P, _L, _P, _P, _P, _P, _P, _I, _P, _P], _I),
    "mpf_gather_edges": ([_I, _I, _I, _P, _L, _L, _P, _P, _L, _P, _P, _P, _P, _I, _P], _I),
    "mpf_halo_fill": ([_P, _I, _P, _L, C.c_int32, _P, _I, _P], _I),
    "mpf_halo_fold": ([_P, _I, _P, _L, C.c_int32, _P, _I, _P], _I),
    "mpf_halo_pack": ([_P, _I, _P, _L, C.c_int32, _I, C.c_int32, _P, _I, _P], _I),
    "mpf_halo_unpack": ([_P, _I, _P, _L, C.c_int32, _I, C.c_int32, _P, _I, _I, _P], _I),
    "mpf_add_density": ([_P, _P, _I, _P, C.c_int32, _L, _P, _P, _I, _P], _I),
    "mpf_num_tiles": ([_I, _I, _I, _P, _P, _P, _P], _I),
    "mpf_sort_workspace_bytes": ([_L, _L, _P], _I),
    "mpf_sort_by_tile": ([_I, _I, _I, _P, _L, _P, _L, _L, _L, _P, _P, _P, _P, _P, _I, _P, _P, _P, _P,
                          C.c_size_t, _I, _P], _I),
    "mpf_sort_by_tile_noalloc": ([_I, _I, _I, _P, _L, _P, _L, _L, _L, _P, _P, _P, _P, _P, _I, _P, _P, _P, _I,
                                  _P], _I),
    "mpf_gather_forms": ([_I, _I, _I, _P, _L, _L, _P, _L, _P, _L, _P, _P, _P, _P, _I, _P], _I),
    "mpf_scatter_forms": ([_I, _I, _I, _P, _L, _P, _L, _L, _P, _L, _P, _P, _P, _P, _I, _P], _I),
    "mpf_resort_workspace_bytes": ([_I, _I, _I, _P, _P, _P, _I, _L, _P], _I),
    "mpf_resort_by_tile": ([_I, _I, _I, _P, _L, _P, _L, _L, _L, _P, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P,
                            C.c_size_t, _I, _P], _I),
    "mpf_permute_rows": ([_P, _L, _P, _L, _L, _P, _L, _I, _P], _I),
    "mpf_unpermute_rows": ([_P, _L, _P, _L, _L, _P, _L, _I, _P], _I),
    "mpf_scatter_deterministic_workspace_bytes": ([_L, _P], _I),
    "mpf_scatter_deterministic": ([_I, _I, _I, _P, _L, _P, _L, _L, _P, _L, _P, _P, _P, _P, _P, C.c_size_t, _P], _I),
    "mpf_scatter_deterministic_tiles": ([_I, _I, _I, _P, _L, _P, _L, _L, _P, _L, _P, _P, _P, _P, _P, _P, _P,
                                         C.c_size_t, _P], _I),
    "mpf_batch_request_size": ([], _L),
    "mpf_batch_request_init": ([_P, _I, _I, _I, _I, _P, _L, _P, _L, _L, _P, _P, _L, _I, _P, _P, _P, _P], _I),
    "mpf_batch_launch": ([_P, _P, _I, _I, _P], _I),
}

_lock = threading.Lock()
_handle: C.CDLL | None = None


def library() -> C.CDLL:
    """The loaded backend library; raises if it is not built."""
    global _handle
    if _handle is None:
        with _lock:
            if _handle is None:
                if not LIBRARY.exists():
                    raise RuntimeError(
                        f"the CUDA backend {LIBRARY.name} is not built: run "
                        "`python mpifield_b200/build.py` (nvcc, sm_100a); there is no CPU fallback"
                    )
                lib = C.CDLL(str(LIBRARY))
                for name, (args, res) in _SIGNATURES.items():
                    fn = getattr(lib, name)
                    fn.argtypes = args
                    fn.restype = res
                _handle = lib
    return _handle


def symbols() -> list[str]:
    """The entry points this module binds."""
    return list(_SIGNATURES)


def check(status: int, what: str) -> None:
    """Raise for a non-zero status: ValueError for bad arguments, BackendError otherwise."""
    if status == OK:
        return
    message = library().mpf_status_string(status).decode()
    if status in (ERR_ARGUMENT, ERR_SHAPE, ERR_ALIGNMENT, ERR_WORKSPACE, ERR_UNSUPPORTED):
        raise ValueError(f"{what}: {message} (status {status})")
    cuda = library().mpf_last_error().decode()
    raise BackendError(f"{what}: {message} (status {status}, last CUDA error {cuda})")


def require_cuda(*tensors: torch.Tensor) -> torch.device:
    """The common CUDA device of the tensors; raises for CPU tensors (no CPU fallback)."""
    device = None
    for t in tensors:
        if not isinstance(t, torch.Tensor):
            raise TypeError(f"expected a torch tensor on a CUDA device, got {type(t).__name__}")
        if t.device.type != "cuda":
            raise TypeError(
                "mpifield_b200 runs on CUDA tensors only (no CPU fallback); got a tensor on "
                f"{t.device}"
            )
        if device is None:
            device = t.device
        elif t.device != device:
            raise ValueError(f"tensors on different devices: {device} and {t.device}")
    assert device is not None
    return device


def dtype_code(dtype: torch.dtype) -> int:
    if dtype == torch.float64:
        return F64
    if dtype == torch.float32:
        return F32
    raise TypeError(f"mpifield_b200 kernels take float64 or float32, got {dtype}")


def stream_of(device: torch.device) -> int:
    """The raw cudaStream_t of torch's current stream on ``device``."""
    return torch.cuda.current_stream(device).cuda_stream


def geometry_arrays(geometry) -> tuple[C.Array, C.Array, C.Array, C.Array, int]:
    """``(*lower, *cell, *num, *code)`` as C arrays, and ndim (one set per geometry, kept:
    the calls only read them)."""
    return _geometry_arrays(tuple(geometry))


@functools.lru_cache(maxsize=1024)
def _geometry_arrays(geometry: tuple) -> tuple[C.Array, C.Array, C.Array, C.Array, int]:
    if len(geometry) % 4 != 0 or not 4 <= len(geometry) <= 12:
        raise ValueError(f"a geometry has 4 * ndim entries, got {len(geometry)}")
    ndim = len(geometry) // 4
    lower = (C.c_double * ndim)(*(float(v) for v in geometry[:ndim]))
    cell = (C.c_double * ndim)(*(float(v) for v in geometry[ndim : 2 * ndim]))
    num = (C.c_int32 * ndim)(*(int(v) for v in geometry[2 * ndim : 3 * ndim]))
    code = (C.c_int32 * ndim)(*(int(v) for v in geometry[3 * ndim :]))
    return lower, cell, num, code, ndim


def tuning_struct(path: int = PATH_AUTO, block: int = 0, smem_bytes: int = 0, ctas_per_sm: int = 0,
                  variant: int = 0, wait_limit: int = 0) -> Tuning:
    return Tuning(path, block, smem_bytes, ctas_per_sm, variant, wait_limit)


def device_errors(clear: bool = True) -> int:
    """The MPF_DEVICE_ERROR_* bits raised by kernels on the current device (synchronises)."""
    flags = C.c_uint32(0)
    check(library().mpf_device_errors(int(clear), C.byref(flags)), "device_errors")
    return int(flags.value)
