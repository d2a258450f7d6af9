"""Generate the golden fixtures in tests/golden/ from the compiled reference.

Run in a container that has the reference sources (the path is given by
--refsrc or the environment variable LOADSG_REFERENCE).  For every case below it builds oracle/_ref/d<d>/ref_harness (the
unmodified LoAdSG sources compiled in place plus oracle/ref_harness.cpp), runs
it, and packs the arrays into tests/golden/<name>.npz.  The fixtures are small
(a few hundred KB in total) and committed; the GPU box never needs the
reference.

    python tests/golden/make_golden.py [--refsrc DIR] [--only NAME]   # DIR: the reference's library/source
    python tests/golden/make_golden.py --cmds prew2nodal,nodal2prew   # add commands to existing fixtures

    python tests/golden/make_golden.py --bd        # boundary-data right-hand sides -> bd_<name>.npz
    python tests/golden/make_golden.py --pde       # PDE_*::SetUp right-hand sides -> pde_<name>.npz
    python tests/golden/make_golden.py --complete  # completion of given point sets -> cmp_<name>.npz
    python tests/golden/make_golden.py --example   # poisson_regular.cpp's convergence table -> ex_poisson_d3.npz

prew2nodal / nodal2prew run calcNodalByPrew / calcPrewByNodal on the fixture's
x (BasisTransformations/BasisTransformations.cpp:486-545,670-706); mass /
massdiag use the midpoint plugin with the Q1 mass matrix, helmholtz the
reference's own HelmHoltz stencil (stencils/Stencil.h:873-919); h1norm /
l2norm are H1::getValue / L2::getValue (applications/H1_Norm.cpp) of x.
The bd_ fixtures hold a second grid with boundary points (the same build,
then completeNeumannGrid), boundary values g of a coefficient family, g after
CalcHierarchicalBasisForRHS, and InHomoBoundaryRHSHierarchical's multiply /
multiply_mass / multiply_mass_coeff onto the first grid
(MatrixVectorMultiplication/RHS.cpp:6-41,697-1008).  The pde_ fixtures
hold f on every point and g on the boundary points of that second grid, the
right-hand sides of PDE_Poisson_InHomRHS::SetUp and
PDE_Helmholtz_VariableCoeff::SetUp (applications/PDE.cpp, PDE.h), and the
transforms they use: CalcHierarchicalBasis of f on the second grid and
CalcNodalBasis of x on the first (BasisTransformations.cpp:174-198,390-409).
"""
import argparse
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle")

# Coefficient families (oracle/coefficient.h): params as passed to the plugin.
SINPROD = (1, [1.0, 0.5] + [1.0] * 8)           # a = 1 + 0.5 prod sin(pi x_i)
EXPSIN6 = (2, [0.3, -0.2, 0.25, 0.1, -0.15, 0.2, 0, 0])  # a = exp(sum c_k sin(k pi x_k))
SINPROD_M = (1, [1.0, 0.9, 2.0, 1.0, 3.0, 2.0, 1.0, 3.0, 1.0, 2.0])
CONST1 = (0, [1.0])
SIN2PI = (4, [1.0, 0.5])

# name, d, grid args, coefficient, commands
CASES = [
    ("d3_L3", 3, "level=3", SINPROD, ["tables", "matvec", "poisson", "diag", "cg"]),
    ("d3_L5", 3, "level=5", SINPROD, ["tables", "matvec", "poisson", "diag", "cg"]),
    ("d3_adapt", 3, "level=2 refine=3 theta=0.6 target=corner", SINPROD, ["tables", "matvec", "diag", "cg"]),
    ("d3_plane", 3, "level=3 refine=2 theta=0.3 target=plane", SIN2PI, ["tables", "matvec", "diag"]),
    ("d2_L6", 2, "level=6", SINPROD_M, ["tables", "matvec", "poisson", "diag", "cg"]),
    ("d2_adapt", 2, "level=3 refine=3 theta=0.45 target=corner", SINPROD, ["tables", "matvec", "diag", "cg"]),
    ("d4_L3", 4, "level=3", EXPSIN6, ["tables", "matvec", "diag", "cg"]),
    ("d4_plane", 4, "level=2 refine=2 theta=0.3 target=plane", SINPROD_M, ["tables", "matvec", "diag"]),
    ("d5_L2", 5, "level=2", EXPSIN6, ["tables", "matvec", "diag"]),
    ("d6_L2", 6, "level=2", EXPSIN6, ["tables", "matvec", "poisson", "diag", "cg"]),
    ("d6_L3", 6, "level=3", SINPROD_M, ["matvec", "diag"]),
    ("d7_L2", 7, "level=2", SINPROD_M, ["tables", "matvec", "poisson", "diag", "mass", "helmholtz", "massdiag"]),
    ("d8_L2", 8, "level=2", EXPSIN6, ["tables", "matvec", "poisson", "prew2nodal", "nodal2prew"]),
    # the CPU-runnable configuration: d = 3, level 7 (7,423 points), a = 1 + 0.5 prod sin(pi x_i)
    ("d3_L7", 3, "level=7", SINPROD, ["matvec", "poisson", "diag", "cg"]),
    # the benchmark's grid family (regular grid refined toward the corner, completed;
    # hanging nodes) at sizes the compiled reference solves in minutes
    ("d5_corner", 5, "level=3 refine=2 theta=0.6 target=corner", EXPSIN6, ["tables", "matvec", "diag", "cg"]),
    ("d6_corner", 6, "level=3 refine=2 theta=0.6 target=corner", EXPSIN6, ["tables", "matvec", "diag", "cg"]),
]
# per-cell corner dumps grow as 2^(2d) per cell; fixtures named here keep the counts only
NO_CELL_DUMP = {"d5_corner", "d6_corner"}


# boundary-data right-hand sides: name, d, grid args, boundary-value family (g)
BD_CASES = [
    ("bd_d2_L5", 2, "level=5", SIN2PI),
    ("bd_d2_adapt", 2, "level=3 refine=2 theta=0.6 target=corner", EXPSIN6),
    ("bd_d3_L4", 3, "level=4", SIN2PI),
    ("bd_d3_adapt", 3, "level=2 refine=3 theta=0.6 target=corner", EXPSIN6),
    ("bd_d4_L3", 4, "level=3", EXPSIN6),
    ("bd_d5_L2", 5, "level=2", SIN2PI),
    ("bd_d6_L2", 6, "level=2", EXPSIN6),
]


# right-hand sides of problems with boundary data (PDE_Poisson_InHomRHS,
# PDE_Helmholtz_VariableCoeff): name, d, grid args, f family, g family
PDE_CASES = [
    ("pde_d2_L4", 2, "level=4", SIN2PI, EXPSIN6),
    ("pde_d2_adapt", 2, "level=2 refine=2 theta=0.6 target=corner", EXPSIN6, SIN2PI),
    ("pde_d3_L3", 3, "level=3", EXPSIN6, SIN2PI),
    ("pde_d4_L2", 4, "level=2", SIN2PI, EXPSIN6),
]


# a caller's point set completed by the reference (completeDirichletGrid /
# completeNeumannGrid): name, d, seed, points, max steps from the centre
# (seed None: the two points of examples_doxygen/gridgeneration_adaptive.cpp)
COMPLETE_CASES = [
    ("cmp_d2_example", 2, None, 0, 0),
    ("cmp_d2_random", 2, 11, 6, 7),
    ("cmp_d3_random", 3, 12, 5, 6),
    ("cmp_d4_random", 4, 13, 4, 5),
]


def complete_input(d, seed, npts, steps):
    """Points reached from the centre by random son steps (deduplicated)."""
    if seed is None:
        c = [2] * d
        bl = [2 * (2 * v) for v in c]  # leftSon(0).leftSon(1).leftSon(0).leftSon(1) in d = 2: (8, 8)
        tr = [2 * (2 * v + 1) + 1 for v in c]  # the same with rightSon: (11, 11)
        return np.array([bl, tr], np.int32)
    rng = np.random.default_rng(seed)
    pts = []
    while len(pts) < npts:
        I = [2] * d
        for _ in range(int(rng.integers(2, steps + 1))):
            k = int(rng.integers(0, d))
            I[k] = 2 * I[k] + int(rng.integers(0, 2))
        if I not in pts:
            pts.append(I)
    return np.array(pts, np.int32)


def run(cmd, **kw):
    r = subprocess.run(cmd, capture_output=True, text=True, **kw)
    if r.returncode != 0:
        raise RuntimeError(f"{cmd} failed:\n{r.stdout}\n{r.stderr}")
    return r.stdout


def read_meta(path):
    meta, arrays = {}, []
    for line in open(path):
        parts = line.split()
        if not parts:
            continue
        if parts[0] == "array":
            arrays.append(parts[1])
        else:
            meta[parts[0]] = parts[1]
    return meta, arrays


DTYPES = {"i32": np.int32, "u8": np.uint8, "f64": np.float64}


def load_arrays(outdir, names, prefix):
    res = {}
    for n in names:
        stem, ext = n.rsplit(".", 1)
        res[prefix + stem] = np.fromfile(os.path.join(outdir, n), dtype=DTYPES[ext])
    return res


def make_case(name, d, gridargs, coef, cmds, refsrc):
    run(["make", "-s", "-C", ORACLE, "ref", f"D={d}", f"REFSRC={refsrc}", "-j8"])
    exe = os.path.join(ORACLE, "_ref", f"d{d}", "ref_harness")
    fam, params = coef
    cp = "cp=" + ",".join(repr(float(p)) for p in params)
    args = gridargs.split() + [f"coef={fam}", cp]
    out = {"d": np.int32(d), "coef_family": np.int32(fam), "coef_params": np.array(params, np.float64)}
    with tempfile.TemporaryDirectory() as tmp:
        run([exe, "grid", tmp] + args)
        meta, arrs = read_meta(os.path.join(tmp, "meta_grid.txt"))
        out.update(load_arrays(tmp, arrs, ""))
        n = int(meta["N"])
        rng = np.random.default_rng(sum(map(ord, name)))
        x = rng.uniform(-1.0, 1.0, n)
        f = rng.uniform(-1.0, 1.0, n) * (out["active"] > 0)
        x.tofile(os.path.join(tmp, "x_in.f64"))
        f.tofile(os.path.join(tmp, "f_in.f64"))
        out["x"] = x
        out["f"] = f
        for c in cmds:
            extra = []
            if c in ("matvec", "poisson", "prew2nodal", "nodal2prew", "mass", "helmholtz", "h1norm", "l2norm"):
                extra = [f"x={tmp}/x_in.f64"]
            if c == "cg":
                extra = [f"f={tmp}/f_in.f64", "eps=1e-20"]
            run([exe, c, tmp] + args + extra)
            meta, arrs = read_meta(os.path.join(tmp, f"meta_{c}.txt"))
            got = load_arrays(tmp, arrs, c + "_")
            out.update(got)
            for k, v in meta.items():
                if k not in ("ok",):
                    try:
                        out[f"{c}_meta_{k}"] = np.float64(float(v))
                    except ValueError:
                        pass
    out["gridargs"] = np.array(gridargs)
    if d >= 7 or name in NO_CELL_DUMP:  # per-cell corner dumps grow as 2^(2d) per cell; keep the counts only
        out.pop("tables_cells", None)
        out.pop("tables_cell_corners", None)
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{name}: N={n} -> {os.path.getsize(path)} bytes")


def add_commands(name, d, gridargs, coef, cmds, refsrc):
    """Runs further commands on an existing fixture's grid and x and stores their outputs."""
    path = os.path.join(HERE, f"{name}.npz")
    z = dict(np.load(path))
    run(["make", "-s", "-C", ORACLE, "ref", f"D={d}", f"REFSRC={refsrc}", "-j8"])
    exe = os.path.join(ORACLE, "_ref", f"d{d}", "ref_harness")
    fam, params = coef
    args = gridargs.split() + [f"coef={fam}", "cp=" + ",".join(repr(float(p)) for p in params)]
    with tempfile.TemporaryDirectory() as tmp:
        z["x"].tofile(os.path.join(tmp, "x_in.f64"))
        for c in cmds:
            run([exe, c, tmp] + args + [f"x={tmp}/x_in.f64"])
            meta, arrs = read_meta(os.path.join(tmp, f"meta_{c}.txt"))
            z.update(load_arrays(tmp, [a for a in arrs if a.startswith("y.") or a.startswith("diag.")], c + "_"))
            for k, v in meta.items():
                if k != "ok":
                    try:
                        z[f"{c}_meta_{k}"] = np.float64(float(v))
                    except ValueError:
                        pass
    np.savez_compressed(path, **z)
    print(f"{name}: added {cmds}")


def make_bd_case(name, d, gridargs, gcoef, refsrc):
    run(["make", "-s", "-C", ORACLE, "ref", f"D={d}", f"REFSRC={refsrc}", "-j8"])
    exe = os.path.join(ORACLE, "_ref", f"d{d}", "ref_harness")
    fam, params = gcoef
    args = gridargs.split() + [f"gfam={fam}", "gp=" + ",".join(repr(float(p)) for p in params)]
    out = {"d": np.int32(d), "g_family": np.int32(fam), "g_params": np.array(params, np.float64),
           "gridargs": np.array(gridargs)}
    with tempfile.TemporaryDirectory() as tmp:
        for c in ("grid", "bdrhs"):
            run([exe, c, tmp] + args)
            meta, arrs = read_meta(os.path.join(tmp, f"meta_{c}.txt"))
            out.update(load_arrays(tmp, arrs, ""))
            for k, v in meta.items():
                if k != "ok":
                    out[f"{c}_meta_{k}"] = np.float64(float(v))
    out["npoints"] = out["npoints"].reshape(-1, d)
    out["points"] = out["points"].reshape(-1, d)
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{name}: N={len(out['active'])} NN={len(out['nactive'])} -> {os.path.getsize(path)} bytes")


def make_pde_case(name, d, gridargs, fcoef, gcoef, refsrc):
    run(["make", "-s", "-C", ORACLE, "ref", f"D={d}", f"REFSRC={refsrc}", "-j8"])
    exe = os.path.join(ORACLE, "_ref", f"d{d}", "ref_harness")
    lst = lambda c: ",".join(repr(float(p)) for p in c[1])
    args = gridargs.split() + [f"ffam={fcoef[0]}", "fp=" + lst(fcoef), f"gfam={gcoef[0]}", "gp=" + lst(gcoef)]
    out = {"d": np.int32(d), "gridargs": np.array(gridargs)}
    with tempfile.TemporaryDirectory() as tmp:
        run([exe, "grid", tmp] + args)
        meta, arrs = read_meta(os.path.join(tmp, "meta_grid.txt"))
        out.update(load_arrays(tmp, arrs, ""))
        x = np.random.default_rng(sum(map(ord, name))).uniform(-1.0, 1.0, int(meta["N"]))
        x.tofile(os.path.join(tmp, "x_in.f64"))
        out["x"] = x
        run([exe, "pdesetup", tmp] + args + [f"x={tmp}/x_in.f64"])
        meta, arrs = read_meta(os.path.join(tmp, "meta_pdesetup.txt"))
        out.update(load_arrays(tmp, arrs, ""))
    out["npoints"] = out["npoints"].reshape(-1, d)
    out["points"] = out["points"].reshape(-1, d)
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{name}: N={len(out['active'])} NN={len(out['nactive'])} -> {os.path.getsize(path)} bytes")


def make_complete_case(name, d, seed, npts, steps, refsrc):
    run(["make", "-s", "-C", ORACLE, "ref", f"D={d}", f"REFSRC={refsrc}", "-j8"])
    exe = os.path.join(ORACLE, "_ref", f"d{d}", "ref_harness")
    pin = complete_input(d, seed, npts, steps)
    out = {"d": np.int32(d), "in_points": pin}
    with tempfile.TemporaryDirectory() as tmp:
        pin.tofile(os.path.join(tmp, "pts.i32"))
        for mode, prefix in (("dirichlet", ""), ("neumann", "n")):
            run([exe, "complete", tmp, f"np={len(pin)}", f"pts={tmp}/pts.i32", f"mode={mode}"])
            meta, arrs = read_meta(os.path.join(tmp, "meta_complete.txt"))
            got = load_arrays(tmp, arrs, prefix)
            out[prefix + "points"] = got[prefix + "points"].reshape(-1, d)
            out[prefix + "active"] = got[prefix + "active"]
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{name}: {len(pin)} points -> {len(out['active'])} (Dirichlet), {len(out['nactive'])} (Neumann)")


def make_poisson_example(refsrc, levels=5):
    """The convergence table of examples_doxygen/poisson_regular.cpp (d = 3,
    levels 1..5) from the reference's own API -> ex_poisson_d3.npz."""
    run(["make", "-s", "-C", ORACLE, "ref", "D=3", f"REFSRC={refsrc}", "-j8"])
    exe = os.path.join(ORACLE, "_ref", "d3", "ref_harness")
    with tempfile.TemporaryDirectory() as tmp:
        run([exe, "poissonex", tmp, f"levels={levels}"])
        meta, arrs = read_meta(os.path.join(tmp, "meta_poissonex.txt"))
        out = load_arrays(tmp, arrs, "")
    out["d"] = np.int32(3)
    path = os.path.join(HERE, "ex_poisson_d3.npz")
    np.savez_compressed(path, **out)
    print(f"ex_poisson_d3: dofs {out['dofs'].tolist()} iterations {out['iterations'].tolist()}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--refsrc", default=os.environ.get("LOADSG_REFERENCE"),
                    help="the reference's library/source directory (default: $LOADSG_REFERENCE)")
    ap.add_argument("--only", default=None)
    ap.add_argument("--cmds", default=None, help="comma list: add these commands to existing fixtures")
    ap.add_argument("--bd", action="store_true", help="the boundary-data right-hand-side fixtures")
    ap.add_argument("--pde", action="store_true", help="the PDE right-hand-side (SetUp) fixtures")
    ap.add_argument("--complete", action="store_true", help="completion of given point sets")
    ap.add_argument("--example", action="store_true", help="the Poisson example's convergence table")
    a = ap.parse_args()
    if not a.refsrc or not os.path.isdir(a.refsrc):
        raise SystemExit("give the reference's library/source directory with --refsrc or $LOADSG_REFERENCE")
    if a.example:
        make_poisson_example(a.refsrc)
        return
    if a.complete:
        for case in COMPLETE_CASES:
            if not a.only or case[0] == a.only:
                make_complete_case(*case, refsrc=a.refsrc)
        return
    if a.pde:
        for case in PDE_CASES:
            if not a.only or case[0] == a.only:
                make_pde_case(*case, refsrc=a.refsrc)
        return
    if a.bd:
        for case in BD_CASES:
            if not a.only or case[0] == a.only:
                make_bd_case(*case, refsrc=a.refsrc)
        return
    for case in CASES:
        if a.only and case[0] != a.only:
            continue
        if a.cmds:
            add_commands(case[0], case[1], case[2], case[3], a.cmds.split(","), refsrc=a.refsrc)
        else:
            make_case(*case, refsrc=a.refsrc)


if __name__ == "__main__":
    main()
