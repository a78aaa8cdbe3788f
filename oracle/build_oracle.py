"""Build recipe for the test oracle (TEST INFRASTRUCTURE, not part of the product).

Three libraries:

- ``oracle/libmpf_oracle.so``: the C restatement ``mpf_oracle.c`` (serial, no fused
  multiply-adds) and the OpenMP restatement ``cpu_baseline.c`` of the reference's
  Pyccel kernels. Built from this repository's files only.
- ``oracle/_ref/libref_host.so``: the reference's own CUDA kernel bodies
  (``src/mpifield/kernels/*/*_cuda.cu`` of the mpifield project) compiled as serial C++
  for the host, one emulated thread per marker, with the project-written stand-ins of
  ``oracle/ref_stubs`` for the two missing ``cunumpy`` headers -- the scheme of the
  reference's ``src/mpifield/tests/kernels/test_cuda_emulated.py:30-126``. Also the
  reference's two C kernels (``scatter_rows_3d_c.c``, ``scatter_linear_1d_c.c``) with
  OpenMP.
- ``oracle/_ref/libref_cuda.so``: the same ``.cu`` kernels compiled with nvcc for sm_100a
  with a one-thread-per-marker launcher (block size 256), the reference's GPU kernels as
  the GPU baseline.

The ``_ref`` libraries are compiled from the reference sources where they lie (they are
never copied into this repository); they need the mpifield source tree, so they are
built only where it is present and otherwise keep whatever was built before.
"""

from __future__ import annotations

import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_OUT = HERE / "_ref"
ORACLE_SO = HERE / "libmpf_oracle.so"
REF_HOST_SO = REF_OUT / "libref_host.so"
REF_C_SO = REF_OUT / "libref_c.so"
REF_CUDA_SO = REF_OUT / "libref_cuda.so"
# the mpifield sources: MPF_REFERENCE_SRC, else the reference/src folder beside this repository
REFERENCE_SRC = Path(os.environ.get("MPF_REFERENCE_SRC", Path(__file__).resolve().parents[2] / "reference" / "src"))
KERNELS = REFERENCE_SRC / "mpifield" / "kernels"

#: The reference kernels compiled into the _ref libraries: the hot path, the edge gathers and
#: the k-form kernels.
REF_KERNELS = [
    f"{op}_{kind}_{n}d"
    for op in ("gather", "scatter")
    for kind in ("linear", "quadratic", "spline")
    for n in (1, 2, 3)
] + [
    f"{name}_{n}d"
    for name in ("deposit_paths", "deposit_paths_spline", "gather_edges", "gather_edges_spline",
                 "gather_forms_spline", "scatter_forms_spline")
    for n in (1, 2, 3)
]


def _run(cmd: list[str]) -> None:
    subprocess.run(cmd, check=True)


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    built = target.stat().st_mtime
    return any(s.stat().st_mtime > built for s in sources if s.exists())


def build_oracle(force: bool = False) -> Path:
    """Compile the C restatement and the CPU baseline into ``libmpf_oracle.so``."""
    sources = [HERE / "mpf_oracle.c", HERE / "cpu_baseline.c"]
    if force or _stale(ORACLE_SO, sources + [Path(__file__)]):
        # cpu_baseline.c includes mpf_oracle.c: one translation unit, no fused multiply-adds
        _run(["gcc", "-std=gnu11", "-O3", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
              str(sources[1]), "-o", str(ORACLE_SO), "-lm"])
    return ORACLE_SO


# ------------------------------------------------------------------ reference builds --

_SIGNATURE = re.compile(r'extern\s+"C"\s+__global__\s+void\s+(\w+)\s*\(([^)]*)\)', re.S)


def kernel_parameters(name: str) -> list[tuple[str, str, int]]:
    """The parameters of a reference kernel: (kind, name, ndim) with kind array/double/int."""
    source = (KERNELS / name / f"{name}_cuda.cu").read_text()
    match = _SIGNATURE.search(source)
    if match is None:
        raise ValueError(f"no kernel signature in {name}")
    params = []
    for part in match.group(2).split(","):
        words = part.split()
        if not words:
            continue
        array = re.match(r"Array(\d)D<double>", words[0])
        if array:
            params.append(("array", words[-1], int(array.group(1))))
        elif words[0] in ("double", "int"):
            params.append((words[0], words[-1], 0))
        else:
            raise ValueError(f"unexpected parameter {part!r} in {name}")
    return params


def _wrapper(name: str, cuda: bool) -> str:
    """A C-ABI wrapper that builds the array views and runs the kernel."""
    params = kernel_parameters(name)
    formals = ["long long n_threads"]
    if cuda:
        formals += ["int block", "int shared_bytes", "void* stream"]
    views, actuals = [], []
    for kind, pname, ndim in params:
        if kind == "array":
            formals += [f"double* {pname}_data", f"const long long* {pname}_shape",
                        f"const long long* {pname}_strides"]
            shape = ", ".join(f"{pname}_shape[{i}]" for i in range(ndim))
            strides = ", ".join(f"{pname}_strides[{i}]" for i in range(ndim))
            views.append(f"    Array{ndim}D<double> {pname}{{{pname}_data, {{{shape}}}, {{{strides}}}}};")
            actuals.append(pname)
        else:
            formals.append(f"{kind} {pname}")
            actuals.append(pname)
    body = "\n".join(views)
    call = ", ".join(actuals)
    if cuda:
        return (
            f'extern "C" int refcuda_{name}({", ".join(formals)}) {{\n{body}\n'
            f"    if (n_threads <= 0) return 0;\n"
            f"    const long long blocks = (n_threads + block - 1) / block;\n"
            f"    {name}<<<(unsigned)blocks, block, shared_bytes, (cudaStream_t)stream>>>({call});\n"
            f"    return (int)cudaGetLastError();\n}}\n"
        )
    return (
        f'extern "C" void ref_{name}({", ".join(formals)}) {{\n{body}\n'
        f"    blockDim.x = 1; gridDim.x = (unsigned)n_threads;\n"
        f"    for (long long t = 0; t < n_threads; ++t) {{ blockIdx.x = (unsigned)t; threadIdx.x = 0; "
        f"{name}({call}); }}\n}}\n"
    )


def reference_available() -> bool:
    return KERNELS.is_dir()


def build_ref_host(force: bool = False) -> Path | None:
    """The reference .cu kernels as serial host C++, and its two OpenMP C kernels."""
    if not reference_available():
        return REF_HOST_SO if REF_HOST_SO.exists() else None
    REF_OUT.mkdir(exist_ok=True)
    sources = [KERNELS / k / f"{k}_cuda.cu" for k in REF_KERNELS]
    if force or _stale(REF_HOST_SO, sources + [Path(__file__)]):
        work = REF_OUT / "src_host"
        work.mkdir(exist_ok=True)
        objects = []
        for kernel in REF_KERNELS:
            tu = work / f"{kernel}.cpp"
            tu.write_text(
                '#include "host_cuda.h"\n'
                "static double block_field[1 << 16];\n"
                f'#include "mpifield/kernels/{kernel}/{kernel}_cuda.cu"\n\n'
                + _wrapper(kernel, cuda=False)
            )
            obj = work / f"{kernel}.o"
            _run(["g++", "-std=c++17", "-O1", "-fPIC", "-ffp-contract=off",
                  f"-I{HERE / 'ref_stubs'}", f"-I{REFERENCE_SRC}", "-c", str(tu), "-o", str(obj)])
            objects.append(obj)
        _run(["g++", "-shared", *map(str, objects), "-o", str(REF_HOST_SO)])
    c_sources = [KERNELS / "scatter_rows_3d" / "scatter_rows_3d_c.c",
                 KERNELS / "scatter_linear_1d" / "scatter_linear_1d_c.c"]
    if force or _stale(REF_C_SO, c_sources + [Path(__file__)]):
        _run(["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", *map(str, c_sources),
              "-o", str(REF_C_SO), "-lm"])
    return REF_HOST_SO


def build_ref_cuda(force: bool = False) -> Path | None:
    """The reference .cu kernels for sm_100a, one thread per marker, as the GPU baseline."""
    if not reference_available():
        return REF_CUDA_SO if REF_CUDA_SO.exists() else None
    REF_OUT.mkdir(exist_ok=True)
    sources = [KERNELS / k / f"{k}_cuda.cu" for k in REF_KERNELS]
    if force or _stale(REF_CUDA_SO, sources + [Path(__file__)]):
        work = REF_OUT / "src_cuda"
        work.mkdir(exist_ok=True)
        tu = work / "ref_cuda.cu"
        parts = ['#include <cuda_runtime.h>\n']
        for kernel in REF_KERNELS:
            parts.append(f"namespace ns_{kernel} {{}}\n")
        # every kernel in one translation unit: the headers have include guards
        for kernel in REF_KERNELS:
            parts.append(f'#include "mpifield/kernels/{kernel}/{kernel}_cuda.cu"\n')
        for kernel in REF_KERNELS:
            parts.append(_wrapper(kernel, cuda=True))
        tu.write_text("".join(parts))
        _run(["nvcc", "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
              "-Xcompiler", "-fPIC", "-shared", f"-I{HERE / 'ref_stubs'}", f"-I{REFERENCE_SRC}",
              str(tu), "-o", str(REF_CUDA_SO)])
    return REF_CUDA_SO


def build_all(force: bool = False) -> None:
    build_oracle(force)
    build_ref_host(force)
    build_ref_cuda(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print(ORACLE_SO, REF_HOST_SO, REF_CUDA_SO)
