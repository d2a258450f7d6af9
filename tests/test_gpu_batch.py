"""Batched operators and solves (lsg_batch_* through the C-ABI): grids of
different dimension and size with their own coefficients, applied and solved
together, against the reference's golden vectors and against the same grids
run one at a time.  A grid's matvec inside a batch runs the same per-item
arithmetic as on its own; the cell operator and the conversion to prewavelets
accumulate with atomic adds, whose order is not fixed, so products agree to
rounding (1e-13 relative in FP64, 1e-6 in FP32) rather than bit for bit.  The
batched CG reduces its dot products in fixed chunks of its own, so solutions
agree to 1e-8 and iteration counts to within one."""
import numpy as np
import pytest

import loadsg_b200 as lsg
from conftest import GOLDEN, load_golden

pytestmark = pytest.mark.gpu

NAMES = ["d2_L6", "d3_adapt", "d4_L3", "d3_L5", "d6_L2", "d5_L2", "d2_adapt", "d4_plane", "d3_plane"]


def golden_batch():
    gold = {g["name"]: g for g in map(load_golden, GOLDEN)}
    cases = [gold[n] for n in NAMES]
    grids = [lsg.AdaptiveSparseGrid(c["points"], c["active"]) for c in cases]
    probs = [lsg.MidpointDiffusion(int(c["coef_family"]), c["coef_params"]) for c in cases]
    return cases, grids, probs


def generated_batch(seed=3):
    """Uneven sizes and dimensions; SINPROD coefficients a = 1 + 0.9 prod sin(pi m_i x_i)."""
    rng = np.random.default_rng(seed)
    grids = [lsg.AdaptiveSparseGrid.regular(2, 7), lsg.AdaptiveSparseGrid.adaptive(3, 3, 2, 0.6, "corner"),
             lsg.AdaptiveSparseGrid.regular(4, 4), lsg.AdaptiveSparseGrid.regular(3, 6),
             lsg.AdaptiveSparseGrid.adaptive(5, 3, 1, 0.6, "corner"), lsg.AdaptiveSparseGrid.regular(2, 4)]
    probs = []
    for g in grids:
        m = rng.integers(1, 4, g.d).astype(float)
        probs.append(lsg.MidpointDiffusion(lsg.COEF_SINPROD, [1.0, 0.9] + list(m)))
    return grids, probs


def to_dev(a, dtype=None):
    import torch
    return torch.tensor(a, device="cuda", dtype=dtype or torch.float64)


def test_batch_layout():
    grids, probs = generated_batch()
    b = lsg.Batch(grids, probs)
    assert b.size == sum(g.n for g in grids)
    ends = sorted((o, o + g.n) for o, g in zip(b.offsets, grids))
    assert ends[0][0] == 0 and ends[-1][1] == b.size
    assert all(ends[k][1] == ends[k + 1][0] for k in range(len(ends) - 1))


def test_batch_matvec_fp64_matches_reference_and_single():
    import torch
    cases, grids, probs = golden_batch()
    b = lsg.Batch(grids, probs)
    x = to_dev(b.gather([c["x"] for c in cases]))
    y = torch.zeros_like(x)
    b.matvec_device(x.data_ptr(), y.data_ptr(), lsg.FP64)
    torch.cuda.synchronize()
    parts = b.split(y.cpu().numpy())
    for c, g, p, yb in zip(cases, grids, probs, parts):
        ref = c["matvec_y"]
        act = g.active > 0
        assert np.abs(yb[act] - ref[act]).max() / np.abs(ref).max() < 1e-12, c["name"]
        m = lsg.MatrixVectorHomogen(g, p)
        xs = to_dev(c["x"])
        ys = torch.zeros_like(xs)
        m.multiplication_device(xs.data_ptr(), ys.data_ptr(), lsg.FP64)
        torch.cuda.synchronize()
        y1 = ys.cpu().numpy()[act]
        assert np.abs(y1 - yb[act]).max() <= 1e-13 * np.abs(y1).max(), c["name"]


def test_batch_matvec_fp32_matches_single():
    import torch
    grids, probs = generated_batch()
    b = lsg.Batch(grids, probs)
    rng = np.random.default_rng(0)
    xs = [rng.uniform(-1, 1, g.n) for g in grids]
    x = to_dev(b.gather(xs), torch.float32)
    y = torch.zeros_like(x)
    b.matvec_device(x.data_ptr(), y.data_ptr(), lsg.FP32)
    torch.cuda.synchronize()
    parts = b.split(y.cpu().numpy())
    for g, p, xi, yb in zip(grids, probs, xs, parts):
        m = lsg.MatrixVectorHomogen(g, p)
        x1 = to_dev(xi, torch.float32)
        y1 = torch.zeros_like(x1)
        m.multiplication_device(x1.data_ptr(), y1.data_ptr(), lsg.FP32)
        torch.cuda.synchronize()
        act = g.active > 0
        ys = y1.cpu().numpy()[act]
        assert np.abs(ys - yb[act]).max() <= 1e-6 * np.abs(ys).max()


@pytest.mark.parametrize("precision", [lsg.FP64, lsg.FP32])
def test_batch_cg_matches_single_solves(precision):
    grids, probs = generated_batch()
    b = lsg.Batch(grids, probs)
    rng = np.random.default_rng(1)
    fs = [rng.uniform(-1, 1, g.n) * g.active for g in grids]
    x = np.zeros(b.size)
    reps, tot = b.solve(1e-10, x, b.gather(fs), criterion=1, precision=precision)
    assert tot["converged"] == 1 and tot["rel_residual"] <= 1e-10
    for g, p, f, xb, r in zip(grids, probs, fs, b.split(x), reps):
        m = lsg.MatrixVectorHomogen(g, p)
        x1 = np.zeros(g.n)
        r1 = lsg.CG.solveHomogen(1e-10, x1, f, m, p, criterion=1, precision=lsg.FP64)
        assert r["converged"] == 1 and r["rel_residual"] <= 1e-10
        if precision == lsg.FP64:
            assert abs(r["iterations"] - r1["iterations"]) <= 1
        act = g.active > 0
        assert np.abs(xb[act] - x1[act]).max() / np.abs(x1).max() < 1e-8


def test_batch_reference_rule_and_zero_rhs():
    """Criterion 0 (the reference's delta rule): a grid with f = 0 is converged
    on entry (0 iterations, x stays 0) while the others iterate as on their own."""
    grids, probs = generated_batch()
    b = lsg.Batch(grids, probs)
    rng = np.random.default_rng(2)
    fs = [rng.uniform(-1, 1, g.n) * g.active for g in grids]
    fs[1] = np.zeros(grids[1].n)
    x = np.zeros(b.size)
    reps, _ = b.solve(1e-20, x, b.gather(fs), criterion=0, precision=lsg.FP64)
    assert reps[1]["iterations"] == 0
    assert not np.any(b.split(x)[1])
    for i in (0, 2, 3):
        m = lsg.MatrixVectorHomogen(grids[i], probs[i])
        x1 = np.zeros(grids[i].n)
        r1 = lsg.CG.solveHomogen(1e-20, x1, fs[i], m, probs[i], criterion=0, precision=lsg.FP64)
        assert abs(reps[i]["iterations"] - r1["iterations"]) <= 1


def test_batch_missing_coefficient_is_an_error():
    grids, probs = generated_batch()
    b = lsg.Batch(grids)
    b.set_problem(0, probs[0])
    x = np.zeros(b.size)
    with pytest.raises(lsg.LsgError):
        b.solve(1e-10, x, np.ones(b.size))
