"""The node and edge weighting of each B-spline degree, paired (src/mpifield/splines.py:100-272).

Faces and cells (2-forms, top forms) are not part of this backend: `Splines` here holds
``nodes`` and ``edges`` only.
"""

from __future__ import annotations

from dataclasses import dataclass

from mpifield_b200.edges import CUBIC_EDGES, QUADRATIC_EDGES, WHITNEY, EdgeWeighting, _spline_edges
from mpifield_b200.weighting import CUBIC, LINEAR, QUADRATIC, Weighting, spline_weighting

__all__ = ["CLAMPED_SPLINES", "SPLINES", "Splines", "splines"]


@dataclass(frozen=True, eq=False, repr=False)
class Splines:
    """The node weighting of B-spline degree ``degree`` and the edge weighting that matches it."""

    degree: int
    nodes: Weighting
    edges: EdgeWeighting | None = None
    clamped: bool = False

    def __post_init__(self) -> None:
        if self.nodes.degree != self.degree:
            raise ValueError(
                f"the node weighting {self.nodes.name!r} has degree {self.nodes.degree}, not {self.degree}")
        if self.edges is not None and self.edges.degree != self.degree:
            raise ValueError(
                f"the edge weighting {self.edges.name!r} has degree {self.edges.degree}, not {self.degree}")
        if self.clamped:
            for weighting in (self.nodes, self.edges):
                if weighting is not None and not weighting.clamps:
                    raise ValueError(f"the {weighting.name} weighting does not take clamped axes")

    @property
    def halo(self) -> int:
        edges = 0 if self.edges is None else self.edges.halo
        return max(self.nodes.halo, edges)

    def require_edges(self) -> EdgeWeighting:
        if self.edges is None:
            have = ", ".join(str(s.degree) for s in SPLINES.values() if s.edges)
            raise ValueError(f"degree {self.degree} has no edge weighting yet (degrees with one: {have})")
        return self.edges

    def __repr__(self) -> str:
        edges = None if self.edges is None else self.edges.name
        clamped = ", clamped=True" if self.clamped else ""
        return f"Splines(degree={self.degree}, nodes={self.nodes.name!r}, edges={edges!r}{clamped})"


def _clamping_nodes(name: str, degree: int) -> Weighting:
    w = spline_weighting(degree, name)
    return Weighting(name, scatter=w.scatter, gather=w.gather, halo=2 if degree > 1 else 1,
                     degree=degree, clamps=True)


#: The built-in shapes, by degree.
SPLINES: dict[int, Splines] = {
    1: Splines(1, LINEAR, WHITNEY),
    2: Splines(2, QUADRATIC, QUADRATIC_EDGES),
    3: Splines(3, CUBIC, CUBIC_EDGES),
}

#: The built-in shapes whose weightings all take clamped axes (the spline kernels).
CLAMPED_SPLINES: dict[int, Splines] = {
    1: Splines(1, _clamping_nodes("linear", 1), _spline_edges("linear", 1), clamped=True),
    2: Splines(2, _clamping_nodes("quadratic", 2), QUADRATIC_EDGES, clamped=True),
    3: Splines(3, CUBIC, CUBIC_EDGES, clamped=True),
}


def splines(degree: int | Splines, clamped: bool = False) -> Splines:
    """The built-in `Splines` of a degree (a `Splines` is returned as is)."""
    if isinstance(degree, Splines):
        if clamped and not degree.clamped:
            raise ValueError(f"{degree!r} does not take clamped axes")
        return degree
    if isinstance(degree, bool) or int(degree) != degree:
        raise ValueError(f"a spline degree is an integer, got {degree!r}")
    try:
        return (CLAMPED_SPLINES if clamped else SPLINES)[int(degree)]
    except KeyError:
        raise ValueError(f"no built-in splines of degree {degree}; have {tuple(SPLINES)}") from None
