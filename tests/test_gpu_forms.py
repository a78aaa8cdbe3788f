"""GPU parity of the k-form gathers and scatters with the oracle and the reference's fixtures.

The faces (2-forms of 3D) and cells (top forms) of every degree, and the 1-forms through
the same kernels: against the reference's own NumPy kernels on the golden fixtures
(tests/golden/form_kernels.npz: bounded, periodic, mixed and clamped axes, markers on
nodes, seams and outside the grid, dead markers with NaN positions), against the oracle
on random cases within 1e-12 of max, the adjoint identity <scatter(x, v), f> =
<v, gather(f, x)>, the float32 variant within its bound, and the block API of
`Splines.faces` / `Splines.cells`.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import mpifield_b200 as mf
from mpifield_b200.kernels import form_components, gather_forms, scatter_forms
from oracle import oracle as O
from tests.helpers import RTOL_F32, RTOL_F64, cases, geometry, load, rel_err

pytestmark = pytest.mark.gpu

FORMS = load("form_kernels.npz")


def _form_case(tag):
    head = tag.split("_")
    return int(head[0][5:]), int(head[1][0]), int(head[1][3])


@pytest.mark.parametrize("tag", cases(FORMS))
def test_forms_match_the_reference_fixtures(tag):
    degree, form, _ = _form_case(tag)
    geom = geometry(FORMS[f"{tag}/geometry"])
    field = torch.tensor(FORMS[f"{tag}/field"], device="cuda")
    pos = torch.tensor(FORMS[f"{tag}/positions"], device="cuda")
    out = torch.zeros(FORMS[f"{tag}/gather"].shape, dtype=torch.float64, device="cuda")
    gather_forms(degree, form, pos, field, out, geom)
    np.testing.assert_allclose(out.cpu().numpy(), FORMS[f"{tag}/gather"], rtol=0, atol=1e-13)
    deposit = torch.zeros_like(field)
    scatter_forms(degree, form, torch.tensor(FORMS[f"{tag}/dead_positions"], device="cuda"),
                  torch.tensor(FORMS[f"{tag}/values"], device="cuda"), deposit, geom)
    np.testing.assert_allclose(deposit.cpu().numpy(), FORMS[f"{tag}/scatter"], rtol=0, atol=1e-13)


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("degree", [1, 2, 3])
def test_forms_match_the_oracle_on_random_cases(ndim, degree):
    rng = np.random.default_rng(10 * ndim + degree)
    for form in range(1, ndim + 1):
        ncomp = form_components(form, ndim)
        for codes in ((0,) * ndim, (1,) * ndim, (2,) + (1,) * (ndim - 1), (1,) + (0,) * (ndim - 1)):
            shape = (12, 9, 7)[:ndim]
            ext = tuple(s + (degree - 1 if c == 2 else 0) for s, c in zip(shape, codes))
            geom = (*rng.uniform(-1, 1, ndim), *rng.uniform(0.1, 0.5, ndim), *shape, *codes)
            lower, cell = np.array(geom[:ndim]), np.array(geom[ndim:2 * ndim])
            n = 20_000
            pos = lower[:, None] + cell[:, None] * rng.uniform(-2, np.array(shape)[:, None] + 1, (ndim, n))
            pos[:, ::53] = lower[:, None] + cell[:, None] * 0.5  # a dense cell
            field = rng.normal(size=(*ext, ncomp))
            values = rng.uniform(0.5, 1.5, (ncomp, n))
            values[:, ::9] = 0.0
            out = torch.zeros((ncomp, n), dtype=torch.float64, device="cuda")
            p = torch.tensor(pos, device="cuda")
            gather_forms(degree, form, p, torch.tensor(field, device="cuda"), out, geom)
            assert rel_err(out.cpu().numpy(), O.gather_forms(degree, form, pos, field, geom)) <= RTOL_F64
            dep = torch.zeros((*ext, ncomp), dtype=torch.float64, device="cuda")
            scatter_forms(degree, form, p, torch.tensor(values, device="cuda"), dep, geom)
            expected = O.scatter_forms(degree, form, pos, values, np.zeros((*ext, ncomp)), geom)
            assert rel_err(dep.cpu().numpy(), expected) <= RTOL_F64
            # the adjoint identity
            lhs = float((dep.cpu().numpy() * field).sum())
            rhs = float((values * out.cpu().numpy()).sum())
            assert abs(lhs - rhs) <= 1e-10 * max(1.0, abs(lhs))
            # float32 within its bound, both on the positions rounded to float32; not for
            # degree 1, whose edge functions (B_0) jump at the cell faces, where a rounded
            # position may land on the other side
            if degree >= 2:
                p32 = p.float()
                ref64 = torch.zeros((ncomp, n), dtype=torch.float64, device="cuda")
                gather_forms(degree, form, p32.double(), torch.tensor(field, device="cuda"), ref64, geom)
                out32 = torch.zeros((ncomp, n), dtype=torch.float32, device="cuda")
                gather_forms(degree, form, p32, torch.tensor(field, device="cuda").float(), out32, geom)
                assert rel_err(out32.double().cpu().numpy(), ref64.cpu().numpy()) <= RTOL_F32


def test_faces_and_cells_through_the_block_api():
    rng = np.random.default_rng(3)
    grid = mf.BlockGrid.from_geometry((0.0, 0.0, 0.0), (0.1, 0.2, 0.25), (10, 6, 5), (True, False, True))
    pos = torch.tensor(rng.uniform(0.0, 0.9, (3, 5000)), device="cuda")
    for degree in (1, 2, 3):
        sp = mf.splines(degree)
        faces = torch.zeros((10, 6, 5, 3), dtype=torch.float64, device="cuda")
        v = torch.tensor(rng.uniform(0.5, 1.5, (3, 5000)), device="cuda")
        sp.faces.scatter_block(pos, v, faces, grid)
        expected = O.scatter_forms(degree, 2, pos.cpu().numpy(), v.cpu().numpy(), np.zeros((10, 6, 5, 3)),
                                   grid.geometry)
        assert rel_err(faces.cpu().numpy(), expected) <= RTOL_F64
        cells = torch.tensor(rng.normal(size=(10, 6, 5, 1)), device="cuda")
        out = torch.zeros((1, 5000), dtype=torch.float64, device="cuda")
        sp.cells.gather_block(pos, cells, out, grid)
        assert rel_err(out.cpu().numpy(), O.gather_forms(degree, 3, pos.cpu().numpy(), cells.cpu().numpy(),
                                                         grid.geometry)) <= RTOL_F64
