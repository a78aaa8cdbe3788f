"""Build recipe of the CUDA backend: every .cu of csrc/ compiled for sm_100a and linked
in-tree into mpifield_b200/libmpifield_b200.so (the library the Python layer loads)."""

from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
LIBRARY = HERE / "libmpifield_b200.so"
OBJDIR = HERE / "_build"
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         f"-I{INCLUDE}", f"-I{CSRC}"]


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def _compile(source: Path, extra: list[str]) -> Path:
    obj = OBJDIR / (source.stem + ".o")
    newest = max([source.stat().st_mtime] + [h.stat().st_mtime for h in _headers()] + [Path(__file__).stat().st_mtime])
    if obj.exists() and obj.stat().st_mtime >= newest:
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", str(source), "-o", str(obj)]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed on {source.name}:\n{result.stderr}")
    return obj


def build(verbose: bool = False, extra: list[str] | None = None) -> Path:
    """Compile the changed sources and link the shared library; returns its path."""
    OBJDIR.mkdir(exist_ok=True)
    extra = list(extra or [])
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        objects = list(pool.map(lambda s: _compile(s, extra), sources()))
    if not LIBRARY.exists() or any(o.stat().st_mtime > LIBRARY.stat().st_mtime for o in objects):
        cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", *map(str, objects), "-o", str(LIBRARY)]
        subprocess.run(cmd, check=True)
    if verbose:
        print(LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
