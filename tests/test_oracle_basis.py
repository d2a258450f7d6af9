"""The oracle's basis transforms against the compiled reference's golden
vectors: calcNodalByPrew restated in C agrees bit for bit; calcPrewByNodal,
computed by the oracle as the exact inverse of calcNodalByPrew on the active
points (dense solve), agrees to rounding (the reference's pole-by-pole
algorithm is such an inverse: BasisTransformations.cpp:486-545)."""
import numpy as np

import oracle


def test_nodal_by_prew_bit_exact(golden):
    if "prew2nodal_y" not in golden:
        return
    g = oracle.OracleGrid(golden["points"], golden["active"])
    u = g.nodal_by_prew(golden["x"])
    assert np.array_equal(u, golden["prew2nodal_y"])


def test_prew_by_nodal_is_the_exact_inverse(golden):
    if "nodal2prew_y" not in golden:
        return
    g = oracle.OracleGrid(golden["points"], golden["active"])
    p = g.prew_by_nodal(golden["x"])
    ref = golden["nodal2prew_y"]
    assert np.abs(p - ref).max() <= 1e-13 * np.abs(ref).max()
    assert not np.any(ref[golden["active"] == 0])


def test_norms_match_reference(golden):
    """H1::getValue / L2::getValue of the fixture's x read as nodal values."""
    if "h1norm_meta_value" not in golden:
        return
    g = oracle.OracleGrid(golden["points"], golden["active"])
    for key, h1 in (("h1norm_meta_value", True), ("l2norm_meta_value", False)):
        ref = float(golden[key])
        assert abs(g.norm(golden["x"], h1) - ref) <= 1e-12 * ref
