"""Learned diagonal preconditioner: CUDA MLP kernels against the FP64 numpy
restatement (oracle/mlp_ref.py), training, and the solver with the learned
diagonal against plain Jacobi-preconditioned CG."""
import numpy as np
import pytest

import loadsg_b200 as lsg
from loadsg_b200 import learned
from oracle import mlp_ref

pytestmark = pytest.mark.gpu


def test_forward_and_gradient_match_fp64_reference():
    import torch
    F, rows = learned.n_features(5), 300
    rng = np.random.default_rng(3)
    p = learned.init_params(F, seed=5)
    p[-1] = 0.3
    X = rng.normal(0, 1, (rows, F)).astype(np.float32)
    Y = rng.normal(0, 0.5, rows).astype(np.float32)
    net = learned.MLP(F, p)
    Xd = torch.tensor(X, device="cuda")
    Yd = torch.tensor(Y, device="cuda")
    o = net.forward(Xd).cpu().numpy()
    o_ref, _ = mlp_ref.forward(p, X)
    # The hidden layers multiply BF16 by BF16 on the tensor cores with FP32
    # accumulation; the reference rounds at the same points but accumulates in
    # FP64, so an activation whose FP32 and FP64 values straddle a BF16 rounding
    # boundary differs by one BF16 unit (2^-8 relative): BF16-level tolerances.
    assert np.abs(o - o_ref).max() <= 3e-3 * (1 + np.abs(o_ref).max())
    loss, g = net.gradient(Xd, Yd)
    loss_ref, g_ref = mlp_ref.loss_and_grad(p, X, Y)
    assert abs(loss - loss_ref) <= 3e-3 * abs(loss_ref)
    assert np.abs(g - g_ref).max() <= 1e-2 * np.abs(g_ref).max()
    # and far below what an FP32-activation forward would leave: the rounding
    # points are the reference's
    assert np.median(np.abs(o - o_ref)) <= 1e-3 * (1 + np.abs(o_ref).max())


def test_training_reduces_loss():
    import torch
    g, prob, m = learned.make_instance(4, 4, 1, 1)
    X, Y = learned.instance_data(m)
    net = learned.MLP(learned.n_features(4), seed=1)
    l0 = net.gradient(X, Y)[0]
    for _ in range(150):
        net.step(X, Y, 3e-3)
    assert net.gradient(X, Y)[0] < 0.3 * l0


def test_learned_diagonal_solves_and_falls_back():
    import torch
    g, prob, m = learned.make_instance(4, 4, 1, 2)
    X, Y = learned.instance_data(m)
    net = learned.MLP(learned.n_features(4), seed=2)
    for _ in range(200):
        net.step(X, Y, 3e-3)
    net.install(m)
    rep = learned.solve_iterations(m, prob, 2, 0)
    assert rep["rel_residual"] <= 1.01e-10 and not rep["fell_back"]
    # a broken network (a NaN output weight) makes the learned diagonal
    # unusable; both solvers fall back to Jacobi and still converge
    p = net.params()
    p[-2] = np.nan
    bad = learned.MLP(learned.n_features(4), p)
    bad.install(m)
    for precision in (lsg.FP64, lsg.FP32):
        rep_bad = learned.solve_iterations(m, prob, 2, 0, precision=precision)
        assert rep_bad["fell_back"] == 1
        assert rep_bad["rel_residual"] <= 1.01e-10


def test_committed_network_against_jacobi_held_out():
    """The committed d = 5 network on held-out lognormal instances (seeds the
    training never saw) of the d = 5 corner grid, FP32 matvec inside FP64
    refinement to relative residual 1e-10, against the method without it:
    CG without a preconditioner and with the exact Jacobi diagonal (the
    reference's Preconditioning, applications/cg_method.h:805).  The learned
    diagonal needs far fewer iterations than no preconditioner, stays within 5 %
    of Jacobi's iterations, and its setup (features, MLP on the tensor cores,
    constant-coefficient base) is cheaper than assembling the exact diagonal."""
    import time
    import torch
    net = learned.MLP.load(learned.DEFAULT_WEIGHTS)
    rows = []
    for seed in (10000, 10001, 10002, 10003):
        g, prob, _ = learned.make_instance(5, 4, 2, seed)
        its = {}
        for name, pc in (("none", 1), ("jacobi", 0), ("learned", 2)):
            m = lsg.MatrixVectorHomogen(g, prob)  # fresh operator: no cached diagonal
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            if pc == 2:
                net.install(m)
            elif pc == 0:
                m.diagonal(prob)
            torch.cuda.synchronize()
            setup = time.perf_counter() - t0
            rep = learned.solve_iterations(m, prob, pc, 7, precision=lsg.FP32)
            assert rep["rel_residual"] <= 1.01e-10 and not rep["fell_back"], (name, rep)
            its[name] = (rep["iterations"], setup)
        rows.append(its)
        print(seed, its)
    mean = {k: float(np.mean([r[k][0] for r in rows])) for k in ("none", "jacobi", "learned")}
    assert mean["learned"] <= 0.2 * mean["none"]
    assert mean["learned"] <= 1.05 * mean["jacobi"]
    # setup on a larger grid of the family (d = 5, 60,928 points)
    g, prob, _ = learned.make_instance(5, 6, 1, 10000)
    m1, m2 = lsg.MatrixVectorHomogen(g, prob), lsg.MatrixVectorHomogen(g, prob)
    net.install(m1)
    m2.diagonal(prob)  # warm-up of both paths
    m1, m2 = lsg.MatrixVectorHomogen(g, prob), lsg.MatrixVectorHomogen(g, prob)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    net.install(m1)
    torch.cuda.synchronize()
    t_learned = time.perf_counter() - t0
    t0 = time.perf_counter()
    m2.diagonal(prob)
    torch.cuda.synchronize()
    t_jacobi = time.perf_counter() - t0
    print(f"setup on {g.n} points: learned {t_learned * 1e3:.2f} ms, exact Jacobi {t_jacobi * 1e3:.2f} ms")
    assert t_learned < t_jacobi
