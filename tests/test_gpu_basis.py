"""Basis transforms on the GPU (lsg_calc_nodal_by_prew / lsg_calc_prew_by_nodal
through the C-ABI) against the compiled reference's golden vectors and the
oracle.  The surpluses of all depths are summed with atomic adds, so results
agree to rounding: 1e-13 relative (max norm) for calcNodalByPrew, 1e-12 for
calcPrewByNodal; on larger grids the round trip prew -> u -> prew holds to 1e-10."""
import numpy as np
import pytest

import loadsg_b200 as lsg
import oracle

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def mat(g):
    return lsg.MatrixVectorHomogen(g, lsg.MidpointDiffusion(lsg.COEF_CONST, [1.0]))


def test_nodal_by_prew_matches_reference(golden):
    if "prew2nodal_y" not in golden:
        pytest.skip("no transform vectors")
    g = lsg.AdaptiveSparseGrid(golden["points"], golden["active"])
    u = np.zeros(g.n)
    lsg.calcNodalByPrew(golden["x"], u, mat(g))
    assert rel(u, golden["prew2nodal_y"]) < 1e-13


def test_prew_by_nodal_matches_reference(golden):
    if "nodal2prew_y" not in golden:
        pytest.skip("no transform vectors")
    g = lsg.AdaptiveSparseGrid(golden["points"], golden["active"])
    p = np.zeros(g.n)
    x = golden["x"].copy()
    lsg.calcPrewByNodal(p, x, mat(g))
    assert rel(p, golden["nodal2prew_y"]) < 1e-12
    assert not np.any(p[golden["active"] == 0])
    assert np.array_equal(x, golden["x"])  # u is not modified


@pytest.mark.parametrize("grid", [("regular", 6, 5), ("adaptive", 5, 3, 2), ("adaptive", 3, 5, 3), ("regular", 2, 10)],
                         ids=lambda a: "-".join(map(str, a)))
def test_round_trip_and_oracle(grid):
    g = lsg.AdaptiveSparseGrid.regular(*grid[1:]) if grid[0] == "regular" else \
        lsg.AdaptiveSparseGrid.adaptive(*grid[1:], 0.6, "corner")
    m = mat(g)
    rng = np.random.default_rng(4)
    p = rng.uniform(-1, 1, g.n) * g.active
    u = np.zeros(g.n)
    lsg.calcNodalByPrew(p, u, m)
    og = oracle.OracleGrid(g.points, g.active)
    assert rel(u, og.nodal_by_prew(p)) < 1e-13
    p2 = np.zeros(g.n)
    lsg.calcPrewByNodal(p2, u, m)
    assert rel(p2, p) < 1e-10


def test_device_entry_points_match_host():
    import torch
    g = lsg.AdaptiveSparseGrid.adaptive(3, 4, 2, 0.6, "corner")
    m = mat(g)
    rng = np.random.default_rng(9)
    p = rng.uniform(-1, 1, g.n)
    u_h = np.zeros(g.n)
    lsg.calcNodalByPrew(p, u_h, m)
    pd = torch.tensor(p, device="cuda")
    ud = torch.zeros_like(pd)
    lsg.calcNodalByPrew_device(pd.data_ptr(), ud.data_ptr(), m)
    torch.cuda.synchronize()
    assert rel(ud.cpu().numpy(), u_h) < 1e-14
    q_h = np.zeros(g.n)
    lsg.calcPrewByNodal(q_h, u_h, m)
    qd = torch.zeros_like(pd)
    lsg.calcPrewByNodal_device(qd.data_ptr(), ud.data_ptr(), m)
    torch.cuda.synchronize()
    assert rel(qd.cpu().numpy(), q_h) < 1e-13


def test_norms_match_reference(golden):
    """lsg_h1_norm / lsg_l2_norm (H1::getValue, L2::getValue of applications/H1_Norm.cpp)."""
    if "h1norm_meta_value" not in golden:
        pytest.skip("no norms")
    g = lsg.AdaptiveSparseGrid(golden["points"], golden["active"])
    m = lsg.MatrixVectorHomogen(g, lsg.MidpointDiffusion(int(golden["coef_family"]), golden["coef_params"]))
    for cls, key in ((lsg.H1, "h1norm_meta_value"), (lsg.L2, "l2norm_meta_value")):
        ref = float(golden[key])
        assert abs(cls(m).getValue(golden["x"]) - ref) <= 1e-12 * ref
    # the operator's own coefficient and form are left in place
    y = np.zeros(g.n)
    m.multiplication(golden["x"], y, m._problem)
    assert rel(y, golden["matvec_y"]) < 1e-12
