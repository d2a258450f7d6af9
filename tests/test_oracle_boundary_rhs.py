"""The oracle's boundary-data right-hand sides against the compiled reference
(tests/golden/bd_*.npz, made by tests/golden/make_golden.py --bd):
CalcHierarchicalBasisForRHS (MatrixVectorMultiplication/RHS.cpp:6-41) and
InHomoBoundaryRHSHierarchical::multiply / multiply_mass / multiply_mass_coeff
(RHS.cpp:697-1008).  The oracle evaluates the reference's integrals in the
reference's order, so the results are bit-exact."""
import os

import numpy as np
import pytest

from conftest import GOLDEN_BD
from oracle import OracleGrid

KINDS = [("y_stiff", 0), ("y_mass", 1), ("y_coeff", 2)]


@pytest.fixture(params=GOLDEN_BD, ids=[os.path.basename(p)[:-4] for p in GOLDEN_BD])
def bd(request):
    z = np.load(request.param)
    return {k: z[k] for k in z.files}


def grids(c):
    return OracleGrid(c["points"], c["active"]), OracleGrid(c["npoints"], c["nactive"])


def test_fixture_shapes(bd):
    d = int(bd["d"])
    assert bd["points"].shape[1] == d and bd["npoints"].shape[1] == d
    # the second grid holds boundary points, the first none
    assert (bd["npoints"] < 2).any(axis=1).any()
    assert not (bd["points"] < 2).any()
    boundary = (bd["npoints"] < 2).any(axis=1)
    assert not bd["g"][~boundary].any()


def test_hierarchize_boundary_bit_exact(bd):
    _, ng = grids(bd)
    assert np.array_equal(ng.hierarchize_boundary(bd["g"]), bd["g_hier"])


@pytest.mark.parametrize("name,kind", KINDS)
def test_boundary_rhs_bit_exact(bd, name, kind):
    g, ng = grids(bd)
    y = g.boundary_rhs(ng, kind, bd["g_hier"])
    assert np.array_equal(y, bd[name])


def test_constant_boundary_data():
    """g = 1 on the boundary: the hierarchical coefficients are 1 at the corners
    and 0 elsewhere, its extension is the constant 1, so the gradient form
    vanishes and the mass form is integral(psi_i): 2^-d at the root point,
    whose prewavelet is the level-1 hat (its stencil holds only itself)."""
    c = {k: v for k, v in np.load(GOLDEN_BD[0]).items()}
    g, ng = grids(c)
    one = (c["npoints"] < 2).any(axis=1).astype(np.float64)
    h = ng.hierarchize_boundary(one)
    corner = (c["npoints"] < 2).all(axis=1)
    assert np.array_equal(h != 0, corner) and np.all(h[corner] == 1.0)
    assert np.abs(g.boundary_rhs(ng, 0, h)).max() < 1e-12
    m = g.boundary_rhs(ng, 1, h)
    root = np.nonzero((c["points"] == 2).all(axis=1))[0][0]
    assert m[root] == 0.5 ** int(c["d"])


def test_missing_parent_is_an_error():
    c = {k: v for k, v in np.load(GOLDEN_BD[0]).items()}
    pts, act = c["npoints"], c["nactive"]
    # drop one boundary corner: the boundary points next to it lose a parent
    corner = np.nonzero((pts < 2).all(axis=1))[0][0]
    keep = np.arange(len(pts)) != corner
    ng = OracleGrid(pts[keep], act[keep])
    with pytest.raises(ValueError):
        ng.hierarchize_boundary(np.ones(keep.sum()))


# ---------------------------------------------------------------- PDE_*::SetUp
from conftest import GOLDEN_PDE  # noqa: E402


@pytest.fixture(params=GOLDEN_PDE, ids=[os.path.basename(p)[:-4] for p in GOLDEN_PDE])
def pde(request):
    z = np.load(request.param)
    return {k: z[k] for k in z.files}


def test_transforms_bit_exact(pde):
    """CalcHierarchicalBasis on the grid with boundary points and CalcNodalBasis
    on the interior grid (BasisTransformations.cpp:174-198,390-409)."""
    g, ng = grids(pde)
    assert np.array_equal(ng.hierarchize(pde["f"]), pde["f_hier"])
    assert np.array_equal(g.dehierarchize(pde["x"]), pde["x_nodal"])


@pytest.mark.parametrize("helmholtz", [False, True], ids=["poisson", "helmholtz"])
def test_pde_setup_rhs(pde, helmholtz):
    """PDE_Poisson_InHomRHS::SetUp / PDE_Helmholtz_VariableCoeff::SetUp
    composed from the oracle's pieces: 1e-14 relative to the reference (the
    inverse basis transform is a dense solve here)."""
    g, ng = grids(pde)
    y = g.pde_rhs(ng, pde["f"], pde["g"], helmholtz=helmholtz)
    ref = pde["rhs_helmholtz" if helmholtz else "rhs_poisson"]
    assert np.abs(y - ref).max() <= 1e-14 * np.abs(ref).max()
