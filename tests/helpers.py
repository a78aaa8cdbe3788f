"""Shared helpers of the tests: golden fixtures, random cases, tolerances."""

from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"

#: FP64 gather/scatter tolerance: max |a - b| / max |b| (atomic order and summation order only).
RTOL_F64 = 1e-12
#: Stated FP32-variant bound against the FP64 oracle, relative to max |b|, on the test grids.
RTOL_F32 = 2e-5

KIND_NAMES = {"linear": 0, "quadratic": 1, "spline": 2}


def load(name: str) -> dict[str, np.ndarray]:
    with np.load(GOLDEN / name) as z:
        return {k: z[k] for k in z.files}


def cases(data: dict[str, np.ndarray]) -> list[str]:
    return sorted({k.split("/")[0] for k in data})


def geometry(array: np.ndarray) -> tuple:
    """A stored geometry as the kernels' tuple: floats, then ints."""
    g = tuple(float(v) for v in array)
    nd = len(g) // 4
    return g[: 2 * nd] + tuple(int(v) for v in g[2 * nd :])


def node_case(tag: str) -> tuple[str, int]:
    """(kind, degree) of a node fixture tag such as ``spline3_2d_10``."""
    head = tag.split("_")[0]
    return head[:-1], int(head[-1])


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    scale = max(float(np.abs(b).max()) if b.size else 0.0, 1e-300)
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / scale) if b.size else 0.0


def random_case(rng, ndim, codes, degree=2, n=500, ncomp=2, spread=2.0, shape=None):
    """A random grid and markers partly outside it (bounded axes), and a field."""
    shape = shape or (11, 9, 7)[:ndim]
    lower = rng.uniform(-1.0, 1.0, ndim)
    cell = rng.uniform(0.1, 0.6, ndim)
    ext = tuple(s + (degree - 1 if c == 2 else 0) for s, c in zip(shape, codes))
    upper = lower + cell * (np.array(shape) - 1)
    pos = rng.uniform(lower - spread * cell, upper + spread * cell, (n, ndim)).T.copy()
    field = rng.normal(size=(*ext, ncomp))
    values = rng.uniform(0.5, 1.5, (ncomp, n))
    geom = (*lower, *cell, *shape, *codes)
    return geom, pos, field, values
