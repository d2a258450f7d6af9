"""Boundary-data right-hand sides on the GPU (lsg_hierarchize_boundary,
lsg_boundary_rhs*): CalcHierarchicalBasisForRHS and
InHomoBoundaryRHSHierarchical::multiply / multiply_mass / multiply_mass_coeff
(MatrixVectorMultiplication/RHS.cpp:6-41,697-1008) against the compiled
reference's golden vectors (tests/golden/bd_*.npz) and the oracle.  The kernels
evaluate the reference's integrals in the reference's order with every
operation rounded on its own, so the results are bit-exact."""
import os

import numpy as np
import pytest

import loadsg_b200 as lsg
from conftest import GOLDEN_BD
from oracle import OracleGrid

pytestmark = pytest.mark.gpu

KINDS = [("y_stiff", "multiply", 0), ("y_mass", "multiply_mass", 1), ("y_coeff", "multiply_mass_coeff", 2)]


@pytest.fixture(params=GOLDEN_BD, ids=[os.path.basename(p)[:-4] for p in GOLDEN_BD])
def bd(request):
    z = np.load(request.param)
    return {k: z[k] for k in z.files}


def setup(c):
    g = lsg.AdaptiveSparseGrid(c["points"], c["active"])
    ng = lsg.AdaptiveSparseGrid(c["npoints"], c["nactive"])
    m = lsg.MatrixVectorHomogen(g)
    return g, ng, m, lsg.InHomoBoundaryRHSHierarchical(m, ng)


def test_hierarchize_matches_reference(bd):
    _, ng, _, _ = setup(bd)
    u = bd["g"].copy()
    lsg.CalcHierarchicalBasisForRHS(u, ng)
    assert np.array_equal(u, bd["g_hier"])


@pytest.mark.parametrize("key,method,kind", KINDS, ids=[k[1] for k in KINDS])
def test_boundary_rhs_matches_reference(bd, key, method, kind):
    g, ng, m, rhs = setup(bd)
    y = np.zeros(g.n)
    getattr(rhs, method)(bd["g_hier"], y)
    ref = bd[key]
    assert np.array_equal(y, ref), np.abs(y - ref).max() / max(np.abs(ref).max(), 1e-300)


def test_device_form_and_untouched_entries():
    """The device entry point on torch buffers gives the host result; entries
    at hanging points keep what the caller left there."""
    import torch
    c = {k: v for k, v in np.load(GOLDEN_BD[1]).items()}  # an adaptive grid with hanging points
    g, ng, m, rhs = setup(c)
    assert (g.active == 0).any()
    y_host = np.full(g.n, 7.0)
    rhs.multiply_mass(c["g_hier"], y_host)
    hier = torch.tensor(c["g_hier"], device="cuda")
    y = torch.full((g.n,), 7.0, dtype=torch.float64, device="cuda")
    rhs.multiply_device(lsg.BDRHS_MASS, hier.data_ptr(), y.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    yd = y.cpu().numpy()
    assert np.array_equal(yd, y_host)
    assert np.all(yd[g.active == 0] == 7.0)
    assert np.array_equal(yd[g.active > 0], c["y_mass"][g.active > 0])


def test_generated_grid_against_oracle():
    """A grid from the generators (regular level 5 in d = 3, 1023 points, and
    its boundary grid): hierarchization and all three forms equal the oracle."""
    g = lsg.AdaptiveSparseGrid.regular(3, 5)
    ng = lsg.AdaptiveSparseGrid.neumann(3, 5)
    x = ng.coordinates()
    gv = np.where(ng.boundary_mask(), np.exp(0.3 * np.sin(np.pi * x[:, 0]) - 0.2 * x[:, 1] + x[:, 2] ** 2), 0.0)
    o, on = OracleGrid(g.points, g.active), OracleGrid(ng.points, ng.active)
    h = gv.copy()
    lsg.CalcHierarchicalBasisForRHS(h, ng)
    assert np.array_equal(h, on.hierarchize_boundary(gv))
    m = lsg.MatrixVectorHomogen(g)
    rhs = lsg.InHomoBoundaryRHSHierarchical(m, ng)
    for _, method, kind in KINDS:
        y = np.zeros(g.n)
        getattr(rhs, method)(h, y)
        assert np.array_equal(y, o.boundary_rhs(on, kind, h)), method


def test_linearity_and_constant_data():
    """At a size the oracle would take minutes on (d = 4, level 5: 3,329
    points): the forms are linear in g to rounding, the gradient form of
    constant boundary data vanishes, and the mass form at the root is 2^-d."""
    d = 4
    g = lsg.AdaptiveSparseGrid.regular(d, 5)
    ng = lsg.AdaptiveSparseGrid.neumann(d, 5)
    m = lsg.MatrixVectorHomogen(g)
    rhs = lsg.InHomoBoundaryRHSHierarchical(m, ng)
    rng = np.random.default_rng(5)
    b = ng.boundary_mask()
    h1, h2 = rng.uniform(-1, 1, ng.n) * b, rng.uniform(-1, 1, ng.n) * b
    y1, y2, y12 = np.zeros(g.n), np.zeros(g.n), np.zeros(g.n)
    rhs.multiply(h1, y1)
    rhs.multiply(h2, y2)
    rhs.multiply(2.5 * h1 + h2, y12)
    assert np.abs(y12 - (2.5 * y1 + y2)).max() <= 1e-12 * np.abs(y12).max()
    one = b.astype(np.float64)
    lsg.CalcHierarchicalBasisForRHS(one, ng)
    corner = (ng.points < 2).all(axis=1)
    assert np.array_equal(one != 0, corner)
    ys, ym = np.zeros(g.n), np.zeros(g.n)
    rhs.multiply(one, ys)
    rhs.multiply_mass(one, ym)
    assert np.abs(ys).max() < 1e-9
    root = np.nonzero((g.points == 2).all(axis=1))[0][0]
    assert ym[root] == 0.5 ** d


def test_errors():
    c = {k: v for k, v in np.load(GOLDEN_BD[0]).items()}
    g, ng, m, rhs = setup(c)
    y = np.zeros(g.n)
    with pytest.raises(lsg.LsgError):
        rhs._run(3, c["g_hier"], y)  # no such form
    corner = np.nonzero((c["npoints"] < 2).all(axis=1))[0][0]
    keep = np.arange(ng.n) != corner
    broken = lsg.AdaptiveSparseGrid(c["npoints"][keep], c["nactive"][keep])
    u = np.ones(broken.n)
    with pytest.raises(lsg.LsgError):
        lsg.CalcHierarchicalBasisForRHS(u, broken)
    # a boundary grid without boundary points gives zero at every active point
    inner = lsg.AdaptiveSparseGrid(c["points"], c["active"])
    y = np.full(g.n, 3.0)
    lsg.InHomoBoundaryRHSHierarchical(m, inner).multiply(np.ones(inner.n), y)
    assert np.all(y[g.active > 0] == 0.0) and np.all(y[g.active == 0] == 3.0)


# ---------------------------------------------------------------- PDE_*::SetUp
from conftest import GOLDEN_PDE  # noqa: E402


@pytest.fixture(params=GOLDEN_PDE, ids=[os.path.basename(p)[:-4] for p in GOLDEN_PDE])
def pde(request):
    z = np.load(request.param)
    return {k: z[k] for k in z.files}


def test_transforms_match_reference(pde):
    """CalcHierarchicalBasis on the grid with boundary points, CalcNodalBasis
    on the interior grid: bit-exact."""
    g = lsg.AdaptiveSparseGrid(pde["points"], pde["active"])
    ng = lsg.AdaptiveSparseGrid(pde["npoints"], pde["nactive"])
    f = pde["f"].copy()
    lsg.CalcHierarchicalBasis(f, ng)
    assert np.array_equal(f, pde["f_hier"])
    x = pde["x"].copy()
    lsg.CalcNodalBasis(x, g)
    assert np.array_equal(x, pde["x_nodal"])
    lsg.CalcHierarchicalBasis(x, g)  # and back
    assert np.abs(x - pde["x"]).max() < 1e-13


@pytest.mark.parametrize("cls,key", [(lsg.PDE_Poisson_InHomRHS, "rhs_poisson"),
                                     (lsg.PDE_Helmholtz_VariableCoeff, "rhs_helmholtz")], ids=["poisson", "helmholtz"])
def test_pde_setup_matches_reference(pde, cls, key):
    """The whole SetUp against the reference's: 1e-12 relative (the inverse
    basis transform and the mass product carry the matvec's 1e-13 rounding);
    f and g come back transformed as the reference leaves them."""
    g = lsg.AdaptiveSparseGrid(pde["points"], pde["active"])
    ng = lsg.AdaptiveSparseGrid(pde["npoints"], pde["nactive"])
    m = lsg.MatrixVectorHomogen(g)
    p = cls(ng, g, m)
    f, gv = pde["f"].copy(), pde["g"].copy()
    p.SetUp(f, gv)
    ref = pde[key]
    assert np.abs(p.getRHS() - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.all(p.getRHS()[g.active == 0] == 0.0)
    # the active interior entries of f moved out (PDE.cpp:14-23); inactive
    # entries keep their values, which the hierarchization does not touch
    interior = (ng.points >= 2).all(axis=1) & (ng.active > 0)
    assert np.array_equal(f[~interior], pde["f_hier"][~interior]) and not f[interior].any()
    on = OracleGrid(ng.points, ng.active)
    assert np.array_equal(gv, on.hierarchize_boundary(pde["g"]))
