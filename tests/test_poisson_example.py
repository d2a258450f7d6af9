"""Known-answer test: the convergence table of the reference's Poisson example
(examples_doxygen/poisson_regular.cpp; d = 3, regular levels 1..5, u = prod
sin(pi x_d), -lap u = f), recorded from the compiled reference in
tests/golden/ex_poisson_d3.npz.  Each level converts f to prewavelets
(calcPrewByNodal), forms the right-hand side with the HelmHoltz (mass) product,
solves with Jacobi CG at the reference's stopping rule (eps = 1e-10), converts
the solution back (calcNodalByPrew) and measures the error in the maximum,
L2 and L2 + H1 norms.  The DOF counts must be equal, the CG iteration counts
within one, and the error norms within 1e-10 relative for the oracle (it
follows the reference step by step) and 1e-4 for the GPU: there the dot
products are reduced in another order, and the reference's rule stops near
1e-6 relative residual, so the norms carry the solver's error."""
import os

import numpy as np
import pytest

import loadsg_b200 as lsg
from conftest import ROOT

REF = np.load(os.path.join(ROOT, "tests", "golden", "ex_poisson_d3.npz"))


def problem(level):
    g = lsg.AdaptiveSparseGrid.regular(3, level)
    x = g.coordinates()
    u = np.prod(np.sin(np.pi * x), axis=1) * (g.active > 0)
    return g, u, 3 * np.pi ** 2 * u


def check(level, dofs, it, linf, l2, h1, tol):
    k = level - 1
    assert dofs == REF["dofs"][k]
    assert abs(it - REF["iterations"][k]) <= 1
    for v, key in ((linf, "linfty"), (l2, "l2"), (h1, "h1")):
        assert abs(v - REF[key][k]) <= tol * REF[key][k], (level, key, v, REF[key][k])


@pytest.mark.parametrize("level", [1, 2, 3, 4])
def test_oracle_reproduces_the_example(level):
    from oracle import OracleGrid
    g, u, f = problem(level)
    o = OracleGrid(g.points, g.active)
    prew = o.prew_by_nodal(f)
    rhs = o.matvec(0, [1.0], prew, form=1)
    xs, it = o.cg(0, [1.0], rhs, 1e-10)
    d = u - o.nodal_by_prew(xs)
    l2 = o.norm(d, h1=False)
    # the oracle follows the reference step by step: equal to 1e-13 here
    check(level, int(g.active.sum()), it, np.abs(d).max(), l2, o.norm(d, h1=True) + l2, 1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("level", [1, 2, 3, 4, 5])
def test_gpu_reproduces_the_example(level):
    g, u, f = problem(level)
    m = lsg.MatrixVectorHomogen(g)
    prew = np.zeros(g.n)
    lsg.calcPrewByNodal(prew, f, m)
    rhs = np.zeros(g.n)
    m.multiplication(prew, rhs, lsg.MidpointMass(lsg.COEF_CONST, [1.0]))
    x = np.zeros(g.n)
    rep = lsg.CG.solveHomogen(1e-10, x, rhs, m, lsg.MidpointDiffusion(lsg.COEF_CONST, [1.0]))
    w = np.zeros(g.n)
    lsg.calcNodalByPrew(x, w, m)
    d = u - w
    l2 = lsg.L2(m).getValue(d)
    check(level, g.getDOFS(), rep["iterations"], np.abs(d).max(), l2, lsg.H1(m).getValue(d) + l2, 1e-4)
