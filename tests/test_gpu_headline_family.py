"""The benchmark's grid family on the GPU: d = 5 / 6 grids refined toward the
corner and completed by the reference's rules (hanging nodes included), the
family of the mixed-precision configuration.

* Against the CPU oracle (the C restatement of the reference's
  MatrixVectorHomogen::multiplication, MatrixVectorMultiplication/
  MatrixVectorHomogen.h:659-759, pinned by the reference's golden vectors):
  FP64 matvec 1e-12, FP32 matvec 2e-5 (max-norm, relative to max |y|), FP64
  Jacobi diagonal 1e-12.  The reference's own golden vectors of the same
  family (d5_corner, d6_corner) are covered by test_gpu_parity.py.
* Run to run: two matvecs, and two FP32+IR solves, give the same bits (no
  atomics on the path: the cell operator and the convert stage write private
  slots that are summed in a fixed order).
"""
import numpy as np
import pytest

import loadsg_b200 as lsg
import oracle

pytestmark = pytest.mark.gpu

EXPSIN = [0.3, -0.2, 0.25, 0.1, -0.15, 0.2]


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def corner40k():
    """d = 6, regular level 5 refined toward the corner and completed: 40,811 points."""
    g = lsg.AdaptiveSparseGrid.adaptive(6, 5, 2, 0.6, "corner")
    assert g.n == 40811 and (g.active == 0).sum() > 0  # hanging nodes present
    return g


def _matvecs(g, fam, params, seed):
    import torch
    prob = lsg.MidpointDiffusion(fam, params)
    m = lsg.MatrixVectorHomogen(g, prob)
    x = np.random.default_rng(seed).uniform(-1, 1, g.n)
    y64 = np.zeros(g.n)
    m.multiplication(x, y64, prob)
    xd = torch.tensor(x, dtype=torch.float32, device="cuda")
    yd = torch.zeros_like(xd)
    m.multiplication_device(xd.data_ptr(), yd.data_ptr(), lsg.FP32)
    torch.cuda.synchronize()
    return m, prob, x, y64, yd.double().cpu().numpy()


def test_corner_d6_40k_matvec_vs_oracle(corner40k):
    g = corner40k
    m, prob, x, y64, y32 = _matvecs(g, lsg.COEF_EXPSIN, EXPSIN, 11)
    yo = oracle.OracleGrid(g.points, g.active).matvec(lsg.COEF_EXPSIN, EXPSIN, x)
    act = g.active > 0
    assert rel(y64[act], yo[act]) < 1e-12
    assert rel(y32[act], yo[act]) < 2e-5


@pytest.mark.parametrize("d,level,fam,params", [
    (5, 4, lsg.COEF_SINPROD, [1.0, 0.9, 2, 1, 3, 2, 1]),
    (6, 4, lsg.COEF_EXPSIN, EXPSIN),
])
def test_corner_matvec_and_diag_vs_oracle(d, level, fam, params):
    g = lsg.AdaptiveSparseGrid.adaptive(d, level, 2, 0.6, "corner")
    m, prob, x, y64, y32 = _matvecs(g, fam, params, d)
    o = oracle.OracleGrid(g.points, g.active)
    act = g.active > 0
    yo = o.matvec(fam, params, x)
    assert rel(y64[act], yo[act]) < 1e-12
    assert rel(y32[act], yo[act]) < 2e-5
    assert rel(m.diagonal(prob), o.diag(fam, params)) < 1e-12


def test_matvec_bitwise_repeatable(corner40k, golden):
    """Two products of the same vector are identical to the bit, FP64 and FP32,
    on every golden grid (sparse slabs included) and on the 40,811-point grid."""
    import torch
    for g, fam, params in ((corner40k, lsg.COEF_EXPSIN, EXPSIN),
                           (lsg.AdaptiveSparseGrid(golden["points"], golden["active"]), int(golden["coef_family"]),
                            golden["coef_params"])):
        m = lsg.MatrixVectorHomogen(g, lsg.MidpointDiffusion(fam, params))
        for dt, prec in ((torch.float64, lsg.FP64), (torch.float32, lsg.FP32)):
            x = torch.tensor(np.random.default_rng(5).uniform(-1, 1, g.n), dtype=dt, device="cuda")
            y1, y2 = torch.zeros_like(x), torch.zeros_like(x)
            m.multiplication_device(x.data_ptr(), y1.data_ptr(), prec)
            m.multiplication_device(x.data_ptr(), y2.data_ptr(), prec)
            torch.cuda.synchronize()
            assert torch.equal(y1, y2)


def test_fp32_ir_solve_bitwise_repeatable(corner40k):
    """FP32 matvec inside FP64 refinement to 1e-10: two solves take the same
    iterations and refinement steps and return the same bits."""
    import torch
    g = corner40k
    prob = lsg.MidpointDiffusion(lsg.COEF_EXPSIN, EXPSIN)
    m = lsg.MatrixVectorHomogen(g, prob)
    f = torch.tensor(np.random.default_rng(3).uniform(-1, 1, g.n) * g.active, device="cuda")
    o = lsg.SolverOpts(1e-10, 1, 3000, 0, lsg.FP32, 1000, 1e-5, 1)
    out = []
    for _ in range(2):
        x = torch.zeros_like(f)
        r = lsg.CG.solve_device(m, f.data_ptr(), x.data_ptr(), o)
        torch.cuda.synchronize()
        assert r["converged"] and r["rel_residual"] <= 1e-10
        out.append((r["iterations"], r["outer_iterations"], x.cpu().numpy()))
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1]
    assert np.array_equal(out[0][2], out[1][2])
