"""Learned diagonal preconditioner: data, training and use.

A point's features (depth multi-index, coordinates, next-to-boundary flags,
local log-coefficient samples, whether its same-depth neighbours exist;
computed on the GPU) go through a 3x64 MLP
whose softplus output scales a cheap constant-coefficient diagonal:
D = base * softplus(mlp(features)).  The network is trained on the GPU
(loadsg_b200/csrc/lsg_mlp.cu: forward, backward and Adam kernels) to match the
exact prewavelet diagonal a(psi_i, psi_i) that the solver computes
(lsg_diag), i.e. on targets log(diag / base); among the training checkpoints
the one with the fewest CG iterations on validation instances is kept.  D is
SPD by construction; solves that stall with it fall back to the exact Jacobi
diagonal inside the library.

    python -m loadsg_b200.learned train --out loadsg_b200/weights/diag_mlp_d5.npz
"""
import argparse
import json
import ctypes
import os
import time

import numpy as np

from . import (COEF_EXPSIN, COEF_LOGNORMAL, AdaptiveSparseGrid, CG, FP32, FP64, LsgError, MatrixVectorHomogen,
               MidpointDiffusion, _check, _ptr, lib)

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "diag_mlp_d5.npz")
H = 64


def n_features(d):
    return 7 * d + 5


def n_params(F):
    return H * F + H + 2 * (H * H + H) + H + 1


def init_params(F, seed=0):
    """He-normal weights, zero biases; output bias so that softplus(o) = 1."""
    rng = np.random.default_rng(seed)
    p = []
    for fan_in, fan_out in [(F, H), (H, H), (H, H)]:
        p.append(rng.normal(0, np.sqrt(2.0 / fan_in), fan_out * fan_in))
        p.append(np.zeros(fan_out))
    p.append(rng.normal(0, np.sqrt(1.0 / H) * 0.1, H))
    p.append(np.array([np.log(np.e - 1.0)]))
    return np.concatenate(p).astype(np.float32)


def _mlp_lib():
    L = lib()
    if not hasattr(L, "_mlp_sigs"):
        P, I32, I64, F32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float
        for name, res, args in [
            ("lsg_mlp_create", ctypes.c_int, [I32, P, P]),
            ("lsg_mlp_destroy", None, [P]),
            ("lsg_mlp_get_params", ctypes.c_int, [P, P]),
            ("lsg_mlp_forward", ctypes.c_int, [P, P, I64, P, P]),
            ("lsg_mlp_gradient", ctypes.c_int, [P, P, P, I64, P, P]),
            ("lsg_mlp_train_step", ctypes.c_int, [P, P, P, I64, F32, P]),
            ("lsg_mlp_last_error", ctypes.c_char_p, []),
            ("lsg_mlp_num_params", I64, [I32]),
            ("lsg_operator_features", ctypes.c_int, [P, P, P]),
            ("lsg_operator_base_diag", ctypes.c_int, [P, P, P]),
            ("lsg_operator_install_learned", ctypes.c_int, [P, P, P]),
        ]:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        L._mlp_sigs = True
    return L


def _mcheck(rc):
    if rc != 0:
        L = _mlp_lib()
        raise LsgError(f"MLP error {rc}: {L.lsg_mlp_last_error().decode()} {L.lsg_last_error().decode()}")


class MLP:
    """The diagonal network on the current GPU (CUDA kernels in lsg_mlp.cu)."""

    def __init__(self, F, params=None, seed=0):
        self.F = F
        p = init_params(F, seed) if params is None else np.ascontiguousarray(params, np.float32)
        assert len(p) == n_params(F) == _mlp_lib().lsg_mlp_num_params(F)
        h = ctypes.c_void_p()
        _mcheck(_mlp_lib().lsg_mlp_create(F, _ptr(p), ctypes.byref(h)))
        self._h = h
        self._destroy = _mlp_lib().lsg_mlp_destroy  # kept: module globals are gone at interpreter exit

    def __del__(self):
        if getattr(self, "_h", None):
            self._destroy(self._h)
            self._h = None

    def params(self):
        out = np.zeros(n_params(self.F), np.float32)
        _mcheck(_mlp_lib().lsg_mlp_get_params(self._h, _ptr(out)))
        return out

    def forward(self, X):
        """X: torch float32 CUDA tensor rows x F -> outputs (torch)."""
        import torch
        out = torch.empty(X.shape[0], dtype=torch.float32, device=X.device)
        _mcheck(_mlp_lib().lsg_mlp_forward(self._h, ctypes.c_void_p(X.data_ptr()), X.shape[0],
                                            ctypes.c_void_p(out.data_ptr()), None))
        return out

    def gradient(self, X, Y):
        g = np.zeros(n_params(self.F), np.float32)
        loss = ctypes.c_float(0)
        _mcheck(_mlp_lib().lsg_mlp_gradient(self._h, ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(Y.data_ptr()),
                                             X.shape[0], _ptr(g), ctypes.byref(loss)))
        return float(loss.value), g

    def step(self, X, Y, lr):
        loss = ctypes.c_float(0)
        _mcheck(_mlp_lib().lsg_mlp_train_step(self._h, ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(Y.data_ptr()),
                                               X.shape[0], lr, ctypes.byref(loss)))
        return float(loss.value)

    def install(self, matrix):
        """Computes D = base * softplus(mlp(features)) for the operator and
        installs it as its learned diagonal (precond = 2)."""
        _mcheck(_mlp_lib().lsg_operator_install_learned(matrix._h, self._h, None))

    def save(self, path):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez(path, params=self.params(), F=self.F)

    @classmethod
    def load(cls, path=DEFAULT_WEIGHTS):
        z = np.load(path)
        return cls(int(z["F"]), z["params"])


def instance_data(matrix):
    """(features, targets, active mask) of one operator, as torch CUDA tensors:
    targets log(exact diagonal / base) at active points."""
    import torch
    g = matrix.grid
    L = _mlp_lib()
    F = n_features(g.d)
    feat = torch.empty((g.n, F), dtype=torch.float32, device="cuda")
    base = torch.empty(g.n, dtype=torch.float64, device="cuda")
    diag = torch.empty(g.n, dtype=torch.float64, device="cuda")
    _mcheck(L.lsg_operator_features(matrix._h, ctypes.c_void_p(feat.data_ptr()), None))
    _mcheck(L.lsg_operator_base_diag(matrix._h, ctypes.c_void_p(base.data_ptr()), None))
    _check(lib().lsg_diag_device(matrix._h, ctypes.c_void_p(diag.data_ptr()), None))
    act = torch.tensor(g.active, dtype=torch.bool, device="cuda")
    y = torch.log(diag[act] / base[act]).float()
    return feat[act].contiguous(), y.contiguous()


def lognormal_problem(d, seed, J=10, sigma=0.5):
    """a(x) = exp(sum_{j<J} xi_j prod_i sin(pi m_ji x_i)), xi_j ~ N(0, sigma^2),
    m_ji ~ U{1,2,3} (tensor-sine modes)."""
    rng = np.random.default_rng(seed)
    xi = rng.normal(0.0, sigma, J)
    m = rng.integers(1, 4, (J, d)).astype(np.float64)
    return MidpointDiffusion(COEF_LOGNORMAL, np.concatenate([[J], xi, m.ravel()]))


def expsin_problem(d, seed, sigma=0.3):
    """a(x) = exp(sum_{k=1..d} c_k sin(k pi x_k)), c_k ~ N(0, sigma^2)."""
    rng = np.random.default_rng(seed)
    return MidpointDiffusion(COEF_EXPSIN, rng.normal(0.0, sigma, d))


_GRIDS = {}


def corner_grid(d, level, refine):
    """The corner-refined grid of an instance; instances differ only in their
    coefficient, so one grid per (d, level, refine) serves them all."""
    key = (d, level, refine)
    if key not in _GRIDS:
        _GRIDS[key] = AdaptiveSparseGrid.adaptive(d, level, refine, 0.6, "corner")
    return _GRIDS[key]


def make_instance(d, level, refine, seed, family="lognormal"):
    g = corner_grid(d, level, refine)
    prob = lognormal_problem(d, seed) if family == "lognormal" else expsin_problem(d, seed)
    return g, prob, MatrixVectorHomogen(g, prob)


def solve_iterations(matrix, prob, precond, seed, tol=1e-10, precision=FP64):
    rng = np.random.default_rng(seed)
    f = rng.uniform(-1, 1, matrix.grid.n) * matrix.grid.active
    x = np.zeros(matrix.grid.n)
    rep = CG.solveHomogen(tol, x, f, matrix, prob, criterion=1, precond=precond, precision=precision, max_iter=5000)
    return rep


def train(out=DEFAULT_WEIGHTS, d=5, level=4, refine=2, n_train=64, n_val=8, epochs=60, batch=8192, lr=2e-3, seed=0,
          family="lognormal", log=print):
    import torch
    F = n_features(d)
    t0 = time.time()
    levels = list(level) if isinstance(level, (list, tuple)) else [level]
    feats, targets = [], []
    for s in range(n_train):
        _, _, m = make_instance(d, levels[s % len(levels)], refine, s, family)
        X, y = instance_data(m)
        feats.append(X)
        targets.append(y)
    X = torch.cat(feats)
    Y = torch.cat(targets)
    log(f"training rows {X.shape[0]} from {n_train} instances ({time.time() - t0:.1f}s)")
    val = [make_instance(d, levels[-1], refine, 10000 + s, family) for s in range(n_val)]  # deepest grids
    net = MLP(F, seed=seed)
    gen = torch.Generator(device="cuda").manual_seed(seed)
    best = (None, float("inf"), None)
    hist = []
    for ep in range(epochs):
        perm = torch.randperm(X.shape[0], device="cuda", generator=gen)
        lr_ep = lr * (0.5 * (1 + np.cos(np.pi * ep / epochs)))
        tot = 0.0
        nb = 0
        for b0 in range(0, X.shape[0], batch):
            idx = perm[b0:b0 + batch]
            tot += net.step(X[idx].contiguous(), Y[idx].contiguous(), lr_ep)
            nb += 1
        if ep % 10 == 9 or ep == epochs - 1:
            its = []
            for (g, prob, m) in val:
                net.install(m)
                its.append(solve_iterations(m, prob, 2, 7)["iterations"])
            mit = float(np.mean(its))
            hist.append((ep, tot / nb, mit))
            log(f"epoch {ep + 1}: loss {tot / nb:.5f}  validation CG iterations {mit:.1f}")
            if mit < best[1]:
                best = (net.params(), mit, ep)
    net = MLP(F, best[0])
    net.save(out)
    log(f"kept epoch {best[2] + 1} (validation iterations {best[1]:.1f}); saved {out}")
    return net, hist


def report(weights, d, level, refine, family, seeds, log=print):
    """Held-out comparison: CG iterations and device time (setup included) with
    no preconditioner, the exact Jacobi diagonal and the learned diagonal."""
    import torch
    net = MLP.load(weights)
    rows = []
    for s in seeds:
        g, prob, m = make_instance(d, level, refine, s, family)
        res = {"seed": s, "n": g.n}
        for name, pc in (("none", 1), ("jacobi", 0), ("learned", 2)):
            m2 = MatrixVectorHomogen(g, prob)  # fresh operator: no cached diagonal
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            if pc == 2:
                net.install(m2)
            rep = solve_iterations(m2, prob, pc, 7, precision=FP32)
            torch.cuda.synchronize()
            res[name] = (rep["iterations"], time.perf_counter() - t0, rep["rel_residual"], rep["fell_back"])
        rows.append(res)
        log(res)
    if rows:  # summary over the held-out instances
        summ = {"instances": len(rows), "n": rows[0]["n"], "d": d, "level": level, "refine": refine, "family": family}
        for name in ("none", "jacobi", "learned"):
            its = np.array([r[name][0] for r in rows], dtype=float)
            secs = np.array([r[name][1] for r in rows], dtype=float)
            summ[name] = {"iterations_mean": float(its.mean()), "iterations_min": int(its.min()),
                          "iterations_max": int(its.max()), "seconds_mean": float(secs.mean()),
                          "fell_back": int(sum(r[name][3] for r in rows))}
        lj = np.array([r["learned"][0] - r["jacobi"][0] for r in rows])
        summ["learned_minus_jacobi_iterations"] = {"mean": float(lj.mean()), "min": int(lj.min()), "max": int(lj.max())}
        log(json.dumps({"summary": summ}))
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "report"])
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--d", type=int, default=5)
    ap.add_argument("--level", default="4", help="level, or comma list cycled over the training instances")
    ap.add_argument("--refine", type=int, default=2)
    ap.add_argument("--family", default="lognormal")
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--n-train", type=int, default=64)
    ap.add_argument("--n-val", type=int, default=8)
    ap.add_argument("--seeds", default="10000,10001,10002,10003")
    a = ap.parse_args()
    if a.cmd == "train":
        levels = [int(v) for v in a.level.split(",")]
        train(out=a.out, d=a.d, level=levels, refine=a.refine, epochs=a.epochs, n_train=a.n_train, n_val=a.n_val,
              family=a.family)
    else:
        seeds = []
        for part in a.seeds.split(","):  # "10000,10001" or a range "10000-10199"
            lo, _, hi = part.partition("-")
            seeds += list(range(int(lo), int(hi) + 1)) if hi else [int(lo)]
        report(a.out, a.d, int(a.level.split(",")[-1]), a.refine, a.family, seeds)


if __name__ == "__main__":
    main()
