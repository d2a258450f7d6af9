"""Runs matrix-vector products of one benchmark operator, for profilers.

    python -m loadsg_b200.profile_matvec [WORKLOAD] [--precision fp32|fp64] [--reps N] [--profile]

Builds the operator of a seeded benchmark instance (workloads.py; default
d6_corner_L8, 1,494,847 points), then runs N products y = A x of a random
vector on the current stream and synchronises.  Operator set-up launches
k_cell_coef / k_sf_collapse once; every product launches the same kernel
sequence, so a profiler can select products by kernel name and launch count.
With --profile it also prints the per-phase CUDA event times of
lsg_matvec_profile (not for use under a profiler).
"""
import argparse
import sys

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", nargs="?", default="d6_corner_L8")
    ap.add_argument("--precision", choices=["fp32", "fp64"], default="fp32")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--profile", action="store_true")
    a = ap.parse_args(argv)
    import torch
    import loadsg_b200 as lsg
    from loadsg_b200.workloads import workload
    g, fam, params, _, desc = workload(a.workload, 0)
    prob = lsg.MidpointDiffusion(fam, params)
    m = lsg.MatrixVectorHomogen(g, prob)
    prec = lsg.FP32 if a.precision == "fp32" else lsg.FP64
    dt = torch.float32 if prec == lsg.FP32 else torch.float64
    x = torch.tensor(np.random.default_rng(5).uniform(-1, 1, g.n) * g.active, dtype=dt, device="cuda")
    y = torch.zeros_like(x)
    torch.cuda.synchronize()
    for _ in range(a.reps):
        m.multiplication_device(x.data_ptr(), y.data_ptr(), prec)
    torch.cuda.synchronize()
    info = m.info()
    print(f"{a.workload}: {g.n} points, {a.reps} {a.precision} products, device bytes {int(info['device_bytes'])}")
    if a.profile:
        ms, by, fl = m.profile(x.data_ptr(), y.data_ptr(), prec, 10)
        names = ["nodal", "P init", "prolongation", "cell operator", "restriction wavefronts + gather", "total"]
        for k, nm in enumerate(names):
            print(f"  {nm:32s} {ms[k]:8.3f} ms  {by[k] / 1e6:10.1f} MB  {by[k] / (ms[k] * 1e-3) / 1e9:8.1f} GB/s")
    return 0


if __name__ == "__main__":
    sys.exit(main())
