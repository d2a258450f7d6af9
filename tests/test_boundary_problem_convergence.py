"""End to end with boundary data, against the mathematics: -lap u = f on
(0,1)^d with u = g on the boundary and the exact solution u = exp(prod_k x_k).
The right-hand side of the reduced problem comes from
PDE_Poisson_InHomRHS::SetUp (applications/PDE.cpp:9-52), CG solves for the
interior part u0, calcNodalByPrew gives its nodal values, and the extension of
g (the hierarchical boundary hats of the grid with boundary points, weighted
by CalcHierarchicalBasisForRHS's coefficients) is added back.  The nodal
error must fall by at least 2.5x per level (second order up to logarithms).
The oracle version runs on the CPU; the GPU version must agree with it."""
import numpy as np
import pytest

import loadsg_b200 as lsg


def exact(Y):
    return np.exp(np.prod(Y, axis=1))


def laplacian(Y):
    d = Y.shape[1]
    return exact(Y) * sum(np.prod(np.delete(Y, k, axis=1) ** 2, axis=1) for k in range(d))


def hat1(x, i):
    """Hierarchical 1D hat of index i; the boundary indices 0 and 1 carry 1 - x and x."""
    if i == 0:
        return 1.0 - x
    if i == 1:
        return x
    t = int(np.floor(np.log2(i)))
    h = 2.0 ** -t
    return np.maximum(0.0, 1.0 - np.abs(x - (2 * (i - 2 ** t) + 1) * h) / h)


def extension(bpoints, gh, X):
    out = np.zeros(len(X))
    for b in np.nonzero(gh)[0]:
        f = np.ones(len(X))
        for k in range(X.shape[1]):
            f *= hat1(X[:, k], bpoints[b, k])
        out += gh[b] * f
    return out


def data(d, level):
    g = lsg.AdaptiveSparseGrid.regular(d, level)
    ng = lsg.AdaptiveSparseGrid.neumann(d, level)
    NX = ng.coordinates()
    return g, ng, -laplacian(NX), np.where(ng.boundary_mask(), exact(NX), 0.0)


def oracle_solution(d, level):
    from oracle import OracleGrid
    g, ng, f, gv = data(d, level)
    o, on = OracleGrid(g.points, g.active), OracleGrid(ng.points, ng.active)
    c, _ = o.cg(0, [1.0], o.pde_rhs(on, f, gv), 1e-26, maxit=2000)
    X = g.coordinates()
    return g, o.nodal_by_prew(c) + extension(ng.points, on.hierarchize_boundary(gv), X), exact(X)


@pytest.mark.parametrize("d,levels", [(2, (2, 3, 4, 5)), (3, (2, 3))])
def test_oracle_converges(d, levels):
    errs = []
    for L in levels:
        _, uh, ue = oracle_solution(d, L)
        errs.append(np.abs(uh - ue).max())
    assert all(a / b >= 2.5 for a, b in zip(errs, errs[1:])), errs
    assert errs[-1] < 4e-4


@pytest.mark.gpu
@pytest.mark.parametrize("d,level", [(2, 4), (2, 5), (3, 3)])
def test_gpu_solves_the_boundary_problem(d, level):
    g, ng, f, gv = data(d, level)
    m = lsg.MatrixVectorHomogen(g)
    pde = lsg.PDE_Poisson_InHomRHS(ng, g, m)
    f_in, g_in = f.copy(), gv.copy()
    pde.SetUp(f_in, g_in)  # g_in comes back as hierarchical boundary coefficients
    c = np.zeros(g.n)
    lsg.CG.solveHomogen(1e-13, c, pde.getRHS(), m, lsg.MidpointDiffusion(lsg.COEF_CONST, [1.0]), criterion=1,
                        max_iter=2000)
    u0 = np.zeros(g.n)
    lsg.calcNodalByPrew(c, u0, m)
    uh = u0 + extension(ng.points, g_in, g.coordinates())
    _, uo, ue = oracle_solution(d, level)
    assert np.abs(uh - uo).max() <= 1e-9 * np.abs(ue).max()
    assert np.abs(uh - ue).max() < 2e-3
