"""Seeded synthetic instances of the benchmark (grid, coefficient, right-hand
side), shared by bench.py and the profiling runner (profile_matvec.py).

The CPU-runnable instance is the reference arm's: a d = 3 regular grid of
level 7 (7,423 points) with a(x) = 1 + 0.5 prod sin(pi x_i) and f ~ U[-1,1]
from seed 0 in storage order, the same on every rank.  The other instances
draw their coefficient and right-hand side from seed 1000 + rank (one
independent instance per GPU).  Importing this module loads no native code.
"""
import numpy as np

CONFIG1 = {"workload": "d3_regular_L7", "d": 3, "level": 7, "n_points": 7423, "coef": "1+0.5 prod sin(pi x_i)",
           "rhs": "f ~ U[-1,1], seed 0, storage order", "tolerance": 1e-10}


def config1_rhs(n):
    """Right-hand side of the CPU-runnable instance (n = 7,423 nodal values)."""
    return np.random.default_rng(0).uniform(-1.0, 1.0, n)


def workload(name, rank=0):
    """(grid, coefficient family, params, f, description) of a named instance."""
    import loadsg_b200 as lsg
    rng = np.random.default_rng(1000 + rank)
    if name == "d6_corner_L8":
        # d=6 grid refined toward the corner (0,...,0): regular level 8, one round
        # adding the sons of every active point with max_k x_k < 0.6, then the
        # reference's completion (hanging nodes included): 1,494,847 points
        g = lsg.AdaptiveSparseGrid.adaptive(6, 8, 1, 0.6, "corner")
        c = rng.normal(0.0, 0.3, 6)
        fam, params = lsg.COEF_EXPSIN, list(c)
        desc = ("d=6 adaptive grid: regular level 8 refined 1 round toward the corner (max_k x_k < 0.6) "
                "+ completeDirichletGrid; a=exp(sum_k c_k sin(k pi x_k)), c_k~N(0,0.3^2); f~U[-1,1] on active points")
    elif name == "d6_adaptive_corner":
        # d=6 grid refined toward the corner (0,...,0): regular level 7, then 3
        # rounds adding the sons of every active point with max_k x_k < 0.6*2^(1-r),
        # then the reference's completion (hanging nodes included): 499,107 points
        g = lsg.AdaptiveSparseGrid.adaptive(6, 7, 3, 0.6, "corner")
        c = rng.normal(0.0, 0.3, 6)
        fam, params = lsg.COEF_EXPSIN, list(c)
        desc = ("d=6 adaptive grid: regular level 7 refined 3 rounds toward the corner (max_k x_k < 0.6*2^(1-r)) "
                "+ completeDirichletGrid; a=exp(sum_k c_k sin(k pi x_k)), c_k~N(0,0.3^2); f~U[-1,1] on active points")
    elif name.startswith("d6_regular_L"):
        level = int(name.split("L")[1])
        g = lsg.AdaptiveSparseGrid.regular(6, level)
        c = rng.normal(0.0, 0.3, 6)
        fam, params = lsg.COEF_EXPSIN, list(c)
        desc = f"d=6 regular sparse grid level {level}, a=exp(sum_k c_k sin(k pi x_k)), c_k~N(0,0.3^2)"
    elif name == "d3_regular_L7":
        g = lsg.AdaptiveSparseGrid.regular(3, 7)
        fam, params = lsg.COEF_SINPROD, [1.0, 0.5, 1.0, 1.0, 1.0]
        desc = "d=3 regular sparse grid level 7, a=1+0.5 prod sin(pi x_i)"
        return g, fam, params, config1_rhs(g.n), desc
    else:
        raise ValueError(f"unknown workload {name}")
    f = rng.uniform(-1.0, 1.0, g.n) * g.active
    return g, fam, params, f, desc
