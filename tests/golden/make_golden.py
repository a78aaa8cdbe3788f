"""Generate the golden fixtures of tests/golden from the reference's own NumPy kernels.

Run where the mpifield source tree is at hand (``MPF_REFERENCE_SRC``, by default the
``reference/src`` folder beside this repository)::

    python tests/golden/make_golden.py

The mpifield package itself cannot be imported here (its ``__init__`` needs cunumpy,
mpiarray and simgeometry, which are absent), so the kernel modules are loaded from
their files: ``mpifield`` and ``mpifield.kernels`` are registered as bare namespace
packages and ``methodcard`` (the reference's documentation decorator, absent too) is a
stub whose ``method(...)`` returns its function unchanged. Nothing else of the
reference is stubbed: the arithmetic is that of
``src/mpifield/kernels/<name>/<name>_numpy.py`` and the modules they import
(``linear_cell.py``, ``quadratic_cell.py``, ``spline_cell.py``, ``whitney_cell.py``,
``spline_edges.py``, ``spline_forms.py``).

The fixtures are small seeded cases (a few dozen markers or paths on grids of a few
nodes per axis) covering every weighting, dimension and boundary code, with markers
outside bounded grids, on nodes and on periodic seams, dead markers (zero values,
NaN positions) and dead or non-finite paths.
"""

from __future__ import annotations

import importlib
import itertools
import os
import sys
import types
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent
SRC = Path(os.environ.get("MPF_REFERENCE_SRC", Path(__file__).resolve().parents[3] / "reference" / "src"))


def _load_reference() -> None:
    """Register the namespace packages and the methodcard stub."""
    stub = types.ModuleType("methodcard")
    stub.method = lambda *args, **kwargs: (lambda function: function)
    stub.Rule = type("Rule", (), {})
    stub.ConvergenceProblem = type("ConvergenceProblem", (), {})
    sys.modules["methodcard"] = stub
    for name, path in (("mpifield", SRC / "mpifield"),
                       ("mpifield.kernels", SRC / "mpifield" / "kernels")):
        module = types.ModuleType(name)
        module.__path__ = [str(path)]
        sys.modules[name] = module


def kernel(name: str):
    """The NumPy version of reference kernel ``name``."""
    folder = f"mpifield.kernels.{name}"
    if folder not in sys.modules:  # its __init__ builds a cunumpy kernel object: skip it
        package = types.ModuleType(folder)
        package.__path__ = [str(SRC / "mpifield" / "kernels" / name)]
        sys.modules[folder] = package
    module = importlib.import_module(f"{folder}.{name}_numpy")
    return getattr(module, name)


SHAPES = {1: (9,), 2: (8, 7), 3: (7, 6, 5)}
LOWER = np.array([0.0, -1.0, 2.0])
CELL = np.array([0.25, 0.5, 0.1])
NODE_KINDS = [("linear", 1), ("quadratic", 2), ("spline", 0), ("spline", 1), ("spline", 2),
              ("spline", 3)]


def _codes(ndim: int, kind: str, degree: int) -> list[tuple[int, ...]]:
    sets = [(0,) * ndim, (1,) * ndim]
    if ndim > 1:
        sets.append((1,) + (0,) * (ndim - 1))
    if kind == "spline" and degree >= 1:
        sets.append((2,) + (1,) * (ndim - 1))
    return sets


def _positions(rng, ndim, num, codes, count):
    lower = LOWER[:ndim]
    cell = CELL[:ndim]
    upper = lower + cell * (np.array(num) - 1)
    pos = rng.uniform(lower - 2.2 * cell, upper + 2.2 * cell, (count, ndim)).T.copy()
    # on nodes, on the seam of periodic axes (one cell past the last node), at the edges
    k = rng.integers(0, np.array(num), (8, ndim)).T
    pos[:, :8] = lower[:, None] + k * cell[:, None]
    for d in range(ndim):
        pos[d, 8] = lower[d] + num[d] * cell[d]
        pos[d, 9] = lower[d]
        pos[d, 10] = upper[d]
        pos[d, 11] = lower[d] - 1e-17
    return pos


def node_cases(rng) -> dict[str, np.ndarray]:
    out = {}
    for (kind, degree), ndim in itertools.product(NODE_KINDS, (1, 2, 3)):
        for codes in _codes(ndim, kind, degree):
            tag = f"{kind}{degree}_{ndim}d_" + "".join(map(str, codes))
            num = SHAPES[ndim]
            ext = tuple(n + (degree - 1 if c == 2 else 0) for n, c in zip(num, codes))
            geometry = (*LOWER[:ndim], *CELL[:ndim], *num, *codes)
            count = 40
            pos = _positions(rng, ndim, num, codes, count)
            ncomp = 2 if ndim != 1 or kind != "linear" else 1
            field = rng.normal(size=(*ext, ncomp))
            values = rng.uniform(0.5, 1.5, (ncomp, count))
            values[:, -3:] = 0.0
            dead = pos.copy()
            dead[:, -3:] = np.nan  # dead markers: zero values, any position
            result = np.zeros((ncomp, count))
            deposit = np.zeros((*ext, ncomp))
            if kind == "linear":
                gname, sname = f"gather_linear_{ndim}d", f"scatter_linear_{ndim}d"
                if ndim == 3:
                    kernel(gname)(pos, field.reshape(-1, ncomp), result, *geometry)
                    kernel(sname)(dead, values, deposit.reshape(-1, ncomp), *geometry)
                elif ndim == 1:
                    kernel(gname)(pos, field, result, *geometry)
                    kernel(sname)(dead[0], values[0], deposit[:, 0], *geometry)
                else:
                    kernel(gname)(pos, field, result, *geometry)
                    kernel(sname)(dead, values, deposit, *geometry)
            elif kind == "quadratic":
                kernel(f"gather_quadratic_{ndim}d")(pos, field, result, *geometry)
                kernel(f"scatter_quadratic_{ndim}d")(dead, values, deposit, *geometry)
            else:
                kernel(f"gather_spline_{ndim}d")(pos, field, result, *geometry, degree)
                kernel(f"scatter_spline_{ndim}d")(dead, values, deposit, *geometry, degree)
            out[f"{tag}/geometry"] = np.array(geometry, dtype=float)
            out[f"{tag}/positions"] = pos
            out[f"{tag}/dead_positions"] = dead
            out[f"{tag}/field"] = field
            out[f"{tag}/values"] = values
            out[f"{tag}/gather"] = result
            out[f"{tag}/scatter"] = deposit
    return out


def path_cases(rng) -> dict[str, np.ndarray]:
    out = {}
    for degree, ndim in itertools.product((1, 2, 3), (1, 2, 3)):
        code_sets = [(0,) * ndim, (1,) * ndim]
        if ndim > 1:
            code_sets.append((1,) + (0,) * (ndim - 1))
        if degree >= 2:
            code_sets.append((2,) + (1,) * (ndim - 1))
        for codes in code_sets:
            tag = f"paths{degree}_{ndim}d_" + "".join(map(str, codes))
            num = SHAPES[ndim]
            ext = tuple(n + (degree - 1 if c == 2 else 0) for n, c in zip(num, codes))
            lower, cell = LOWER[:ndim], CELL[:ndim]
            upper = lower + cell * (np.array(num) - 1)
            count = 30
            start = rng.uniform(lower - 2 * cell, upper + 2 * cell, (count, ndim)).T.copy()
            end = start + rng.normal(scale=2.5 * cell[:, None], size=start.shape)
            end[:, :4] = start[:, :4] + rng.uniform(-0.9, 0.9, (ndim, 4)) * cell[:, None]
            end[:, 4:6] = start[:, 4:6] + 9.0 * cell[:, None]  # long paths (several stretches)
            charges = rng.uniform(0.5, 1.5, count)
            charges[-3] = 0.0
            start[:, -3] = np.nan  # a dead path: zero charge, any position
            end[0, -2] = np.inf  # a non-finite end deposits nothing
            geometry = (*lower, *cell, *num, *codes)
            current = np.zeros((*ext, ndim))
            if degree == 1 and 2 not in codes:
                kernel(f"deposit_paths_{ndim}d")(start, end, charges, current, *geometry)
                out[f"{tag}/whitney"] = current.copy()
                current[...] = 0.0
            kernel(f"deposit_paths_spline_{ndim}d")(start, end, charges, current, *geometry, degree)
            edges = rng.normal(size=(*ext, ndim))
            points = rng.uniform(lower - cell, upper + cell, (count, ndim)).T.copy()
            gathered = np.zeros((ndim, count))
            kernel(f"gather_edges_spline_{ndim}d")(points, edges, gathered, *geometry, degree)
            if degree == 1 and 2 not in codes:
                whitney_field = np.zeros((ndim, count))
                kernel(f"gather_edges_{ndim}d")(points, edges, whitney_field, *geometry)
                out[f"{tag}/whitney_gather"] = whitney_field
            out[f"{tag}/geometry"] = np.array(geometry, dtype=float)
            out[f"{tag}/start"] = start
            out[f"{tag}/end"] = end
            out[f"{tag}/charges"] = charges
            out[f"{tag}/spline"] = current
            out[f"{tag}/edges"] = edges
            out[f"{tag}/points"] = points
            out[f"{tag}/edge_gather"] = gathered
    return out


def form_cases(rng) -> dict[str, np.ndarray]:
    """The k-form gathers and scatters (gather_forms_spline_{n}d, scatter_forms_spline_{n}d):
    every form of 1D to 3D, degrees 1 to 3, bounded, periodic, mixed and clamped axes."""
    out = {}
    for degree, ndim in itertools.product((1, 2, 3), (1, 2, 3)):
        for form in range(1, ndim + 1):
            code_sets = [(0,) * ndim, (1,) * ndim]
            if ndim > 1:
                code_sets.append((1,) + (0,) * (ndim - 1))
            code_sets.append((2,) + (1,) * (ndim - 1))
            for codes in code_sets:
                tag = f"forms{degree}_{form}of{ndim}d_" + "".join(map(str, codes))
                num = SHAPES[ndim]
                ext = tuple(n + (degree - 1 if c == 2 else 0) for n, c in zip(num, codes))
                ncomp = {(1, 1): 1, (1, 2): 2, (2, 2): 1, (1, 3): 3, (2, 3): 3, (3, 3): 1}[(form, ndim)]
                geometry = (*LOWER[:ndim], *CELL[:ndim], *num, *codes)
                count = 30
                pos = _positions(rng, ndim, num, codes, count)
                field = rng.normal(size=(*ext, ncomp))
                values = rng.uniform(0.5, 1.5, (ncomp, count))
                values[:, -3:] = 0.0
                dead = pos.copy()
                dead[:, -3:] = np.nan  # dead markers: zero values, any position
                result = np.zeros((ncomp, count))
                deposit = np.zeros((*ext, ncomp))
                kernel(f"gather_forms_spline_{ndim}d")(pos, field, result, *geometry, degree, form)
                kernel(f"scatter_forms_spline_{ndim}d")(dead, values, deposit, *geometry, degree, form)
                out[f"{tag}/geometry"] = np.array(geometry, dtype=float)
                out[f"{tag}/positions"] = pos
                out[f"{tag}/dead_positions"] = dead
                out[f"{tag}/field"] = field
                out[f"{tag}/values"] = values
                out[f"{tag}/gather"] = result
                out[f"{tag}/scatter"] = deposit
    return out


def main() -> None:
    _load_reference()
    rng = np.random.default_rng(20240611)
    np.savez_compressed(OUT / "node_kernels.npz", **node_cases(rng))
    np.savez_compressed(OUT / "path_kernels.npz", **path_cases(rng))
    np.savez_compressed(OUT / "form_kernels.npz", **form_cases(np.random.default_rng(20261204)))
    for name in ("node_kernels.npz", "path_kernels.npz", "form_kernels.npz"):
        print(name, (OUT / name).stat().st_size, "bytes")


if __name__ == "__main__":
    main()
