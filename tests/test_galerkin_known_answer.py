"""Known answer from the mathematics, independent of the reference's code:
with a = 1 the prewavelet operator is the Galerkin product
A_prew = Psi^T K Psi, where K is the Q1 stiffness (or mass) matrix of the
full grid of the finest mesh width (zero Dirichlet values) and Psi holds the
prewavelets sampled at its nodes.  Each prewavelet of a point of depth T is
its 5^d stencil (nextFiveP, indices/index.cc:252-327) of level-T hats, so on a
regular sparse grid (which holds every stencil point) Psi is exact.  This is
the comparison the reference's checkgrid_dirichlet (tests/testing.cpp:129-249)
was written for, with its full-grid product switched off there."""
import numpy as np
import pytest

import loadsg_b200 as lsg


def hat(x, c, w):
    return np.maximum(0.0, 1.0 - np.abs(x - c) / w)


def galerkin(d, level, form):
    g = lsg.AdaptiveSparseGrid.regular(d, level)
    plan = lsg.Plan(g)
    D = int(np.floor(np.log2(g.points.max())))  # finest depth
    n1 = 2 ** D - 1
    h = 2.0 ** -D
    x1 = h * np.arange(1, n1 + 1)
    K1 = (np.diag(np.full(n1, 2.0)) - np.diag(np.ones(n1 - 1), 1) - np.diag(np.ones(n1 - 1), -1)) / h
    M1 = (np.diag(np.full(n1, 4.0)) + np.diag(np.ones(n1 - 1), 1) + np.diag(np.ones(n1 - 1), -1)) * h / 6

    def kron(ms):
        out = ms[0]
        for m in ms[1:]:
            out = np.kron(out, m)
        return out

    if form == 0:
        K = sum(kron([K1 if j == k else M1 for j in range(d)]) for k in range(d))
    else:
        K = kron([M1] * d)
    coords = g.coordinates()
    depth = np.floor(np.log2(g.points)).astype(int)
    Psi = np.zeros((n1 ** d, g.n))
    for i in range(g.n):
        idx, w = plan.stencil(i)
        assert (idx >= 0).all()  # a regular grid holds every stencil point
        col = np.zeros(n1 ** d)
        for j, wj in zip(idx, w):
            f = hat(x1, coords[j, 0], 2.0 ** -depth[i, 0])
            for k in range(1, d):
                f = np.multiply.outer(f, hat(x1, coords[j, k], 2.0 ** -depth[i, k]))
            col += wj * f.ravel()
        Psi[:, i] = col
    return g, Psi.T @ K @ Psi


CASES = [(2, 4, 0), (2, 4, 1), (3, 3, 0), (3, 3, 1)]


@pytest.mark.parametrize("d,level,form", CASES, ids=lambda v: str(v))
def test_oracle_is_the_galerkin_product(d, level, form):
    from oracle import OracleGrid
    g, A = galerkin(d, level, form)
    x = np.random.default_rng(d * 10 + level).uniform(-1, 1, g.n)
    y = OracleGrid(g.points, g.active).matvec(0, [1.0], x, form=form)
    ref = A @ x
    assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("d,level,form", CASES, ids=lambda v: str(v))
def test_gpu_is_the_galerkin_product(d, level, form):
    g, A = galerkin(d, level, form)
    x = np.random.default_rng(d * 10 + level).uniform(-1, 1, g.n)
    prob = (lsg.MidpointMass if form else lsg.MidpointDiffusion)(lsg.COEF_CONST, [1.0])
    m = lsg.MatrixVectorHomogen(g, prob)
    y = np.zeros(g.n)
    m.multiplication(x, y, prob)
    ref = A @ x
    assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()
