"""The CPU oracle (oracle/lsg_oracle.c) against vectors produced by the compiled
reference (tests/golden, generated by tests/golden/make_golden.py)."""
import numpy as np

import oracle


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_matvec_matches_reference(golden):
    g = oracle.OracleGrid(golden["points"], golden["active"])
    y = g.matvec(int(golden["coef_family"]), golden["coef_params"], golden["x"])
    assert rel(y, golden["matvec_y"]) < 1e-13


def test_poisson_anchor(golden):
    """a == 1 through the plugin path equals the reference's built-in Poisson
    stencil (Stencil.h:1605-1793), the constant-coefficient anchor."""
    if "poisson_y" not in golden:
        return
    g = oracle.OracleGrid(golden["points"], golden["active"])
    y = g.matvec(0, [1.0], golden["x"])
    assert rel(y, golden["poisson_y"]) < 1e-12


def test_diag_matches_reference(golden):
    if "diag_diag" not in golden:
        return
    g = oracle.OracleGrid(golden["points"], golden["active"])
    dg = g.diag(int(golden["coef_family"]), golden["coef_params"])
    assert rel(dg, golden["diag_diag"]) < 1e-13
    act = golden["active"] > 0
    assert (dg[act] > 0).all()


def test_depth_tables_match_reference(golden):
    if "tables_depthlist" not in golden:
        return
    d = int(golden["d"])
    g = oracle.OracleGrid(golden["points"], golden["active"])
    assert np.array_equal(g.depths().ravel(), golden["tables_depthlist"])
    off = golden["tables_sorted_off"]
    srt = golden["tables_sorted"].reshape(-1, d)
    for c in range(1 << d):
        assert np.array_equal(g.sorted_depths(c), srt[off[c]:off[c + 1]])
    cells_off = golden["tables_cells_off"]
    for t, T in enumerate(g.depths()):
        assert g.num_cells(T) == cells_off[t + 1] - cells_off[t]


def test_cg_matches_reference(golden):
    if "cg_x" not in golden:
        return
    g = oracle.OracleGrid(golden["points"], golden["active"])
    x, it = g.cg(int(golden["coef_family"]), golden["coef_params"], golden["f"], 1e-20)
    # eps = 1e-20 stops on delta' < 1e-40, at the round-off floor of the
    # recursive residual, so the last iteration or two depend on rounding
    assert abs(it - int(golden["cg_meta_iterations"])) <= 2
    assert rel(x, golden["cg_x"]) < 1e-9


def test_mass_matches_reference(golden):
    """The midpoint plugin with the Q1 mass matrix (LocalStiffnessMatrices path
    of the reference) and, for a = 1, the reference's own HelmHoltz stencil."""
    if "mass_y" not in golden:
        return
    g = oracle.OracleGrid(golden["points"], golden["active"])
    y = g.matvec(int(golden["coef_family"]), golden["coef_params"], golden["x"], form=1)
    assert rel(y, golden["mass_y"]) < 1e-13
    y1 = g.matvec(0, [1.0], golden["x"], form=1)
    assert rel(y1, golden["helmholtz_y"]) < 1e-13


def test_mass_diag_matches_reference(golden):
    if "massdiag_diag" not in golden:
        return
    g = oracle.OracleGrid(golden["points"], golden["active"])
    dg = g.diag(int(golden["coef_family"]), golden["coef_params"], form=1)
    assert rel(dg, golden["massdiag_diag"]) < 1e-13
