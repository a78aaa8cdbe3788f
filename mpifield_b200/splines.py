"""The B-spline families: the weightings of every form of one degree.

mpifield's ``Splines`` (src/mpifield/splines.py:100-272) names, for a degree, the
weighting of every form: ``nodes`` (0-forms), ``edges`` (1-forms), ``faces`` (2-forms,
3D) and ``cells`` (top forms, 1D to 3D), all on this backend's kernels; the faces and
cells run the k-form kernels (`kernels.FormKernel`, mpf_gather_forms / mpf_scatter_forms)
and take clamped axes. `SPLINES` holds the built-in families; `CLAMPED_SPLINES` those
whose weightings all take clamped axes (every one on the spline kernels), and `splines`
picks one.
"""

from __future__ import annotations

from dataclasses import dataclass

from mpifield_b200.edges import CUBIC_EDGES, QUADRATIC_EDGES, WHITNEY, EdgeWeighting, spline_edges
from mpifield_b200.kernels import FormKernel
from mpifield_b200.weighting import CUBIC, LINEAR, QUADRATIC, Weighting, spline_weighting

__all__ = ["CLAMPED_SPLINES", "SPLINES", "Splines", "splines"]


@dataclass(frozen=True, eq=False, repr=False)
class Splines:
    """The weightings of B-spline degree ``degree``, one per form; ``edges``, ``faces``
    and ``cells`` may be None. With ``clamped`` every weighting must take clamped axes."""

    degree: int
    nodes: Weighting
    edges: EdgeWeighting | None = None
    faces: Weighting | None = None
    cells: Weighting | None = None
    clamped: bool = False

    def __post_init__(self) -> None:
        for role, weighting in (("node", self.nodes), ("edge", self.edges)):
            if weighting is not None and weighting.degree != self.degree:
                raise ValueError(
                    f"the {role} weighting {weighting.name!r} has degree {weighting.degree}, not {self.degree}")
        if self.clamped:
            refusing = [w for w in self.forms() if not w.clamps]
            if refusing:
                raise ValueError(f"the {refusing[0].name} weighting does not take clamped axes")

    def forms(self) -> tuple:
        """The weightings present, nodes first."""
        return tuple(w for w in (self.nodes, self.edges, self.faces, self.cells) if w is not None)

    @property
    def halo(self) -> int:
        """The halo a split field needs for the node and edge weightings together."""
        return max(w.halo for w in (self.nodes, self.edges) if w is not None)

    def require_edges(self) -> EdgeWeighting:
        """The edge weighting; ValueError for a family without one."""
        if self.edges is not None:
            return self.edges
        have = ", ".join(str(d) for d, s in SPLINES.items() if s.edges is not None)
        raise ValueError(f"degree {self.degree} has no edge weighting yet (degrees with one: {have})")

    def __repr__(self) -> str:
        names = ", ".join(f"{label}={w.name!r}" for label, w in
                          (("nodes", self.nodes), ("edges", self.edges), ("faces", self.faces),
                           ("cells", self.cells)) if w is not None)
        return f"Splines(degree {self.degree}: {names}{', clamped' if self.clamped else ''})"


_NAMES = {1: "linear", 2: "quadratic", 3: "cubic"}


def _faces(degree: int) -> Weighting:
    """The 2-forms of a degree in 3D: one component per face normal."""
    fixed = (degree, 2)
    return Weighting(f"{_NAMES[degree]} faces", scatter={3: FormKernel("scatter", 3, fixed)},
                     gather={3: FormKernel("gather", 3, fixed)}, halo=2 if degree > 1 else 1, clamps=True)


def _cells(degree: int) -> Weighting:
    """The top forms of a degree in 1D to 3D: one component."""
    return Weighting(f"{_NAMES[degree]} cells",
                     scatter={n: FormKernel("scatter", n, (degree, n)) for n in (1, 2, 3)},
                     gather={n: FormKernel("gather", n, (degree, n)) for n in (1, 2, 3)},
                     halo=2 if degree > 1 else 1, clamps=True)


_FACES = {d: _faces(d) for d in (1, 2, 3)}
_CELLS = {d: _cells(d) for d in (1, 2, 3)}


def _family(degree: int, clamped: bool) -> Splines:
    if not clamped:
        nodes = {1: LINEAR, 2: QUADRATIC, 3: CUBIC}[degree]
        edges = {1: WHITNEY, 2: QUADRATIC_EDGES, 3: CUBIC_EDGES}[degree]
        return Splines(degree, nodes, edges, _FACES[degree], _CELLS[degree])
    # on clamped axes every weighting runs on the spline kernels (degree 3 already does)
    name = {1: "linear", 2: "quadratic", 3: "cubic"}[degree]
    nodes = CUBIC if degree == 3 else spline_weighting(degree, name)
    nodes = Weighting(nodes.name, nodes.scatter, nodes.gather, halo=2 if degree > 1 else 1, degree=degree,
                      clamps=True)
    edges = {1: spline_edges("linear", 1), 2: QUADRATIC_EDGES, 3: CUBIC_EDGES}[degree]
    return Splines(degree, nodes, edges, _FACES[degree], _CELLS[degree], clamped=True)


#: The built-in families, by degree.
SPLINES: dict[int, Splines] = {d: _family(d, False) for d in (1, 2, 3)}
#: The built-in families whose weightings all take clamped axes, by degree.
CLAMPED_SPLINES: dict[int, Splines] = {d: _family(d, True) for d in (1, 2, 3)}


def splines(degree: int | Splines, clamped: bool = False) -> Splines:
    """The built-in `Splines` of a degree (from `CLAMPED_SPLINES` with ``clamped``); a
    `Splines` is returned as it is, if it takes clamped axes where asked to."""
    if isinstance(degree, Splines):
        if clamped and not degree.clamped:
            raise ValueError(f"{degree!r} does not take clamped axes")
        return degree
    if isinstance(degree, bool) or int(degree) != degree:
        raise ValueError(f"a spline degree is an integer, got {degree!r}")
    table = CLAMPED_SPLINES if clamped else SPLINES
    if int(degree) not in table:
        raise ValueError(f"no built-in splines of degree {degree}; have {tuple(SPLINES)}")
    return table[int(degree)]
