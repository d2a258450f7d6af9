"""Benchmark: time to relative residual 1e-10 of the prewavelet stiffness solve.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl native|reference] [--workload NAME]

One step = one solve of A x = f from x = 0 to ||f - A x|| / ||f|| <= 1e-10
(FP32 matvec inside FP64 iterative refinement, Jacobi or learned diagonal
preconditioner), inputs resident in HBM.  The default workload is the
mixed-precision configuration: a d=6 grid of 1,494,847 points (regular level
8 refined one round toward the corner, completed).  The JSON line also
carries the plain FP64 CG time on the same instance and the FP32+IR
solution's distance to it, the matvec times and GB/s, the roofline of the
cell-operator kernel (the dominant one), the end-to-end time through the C-ABI
with host buffers, and a same-instance leg: the CPU-runnable configuration
(d=3 level 7, 7,423 points) solved on the GPU with the right-hand side the
reference arm solves.

--impl reference runs the reference's own CG::solveHomogen (oracle/_ref, the
LoAdSG sources compiled in place; the -O3 timing build when present) on that
CPU-runnable instance on the host cores, measured, never scaled.  The
mixed-precision workload is out of the reference's reach (fixed hash
capacities, sgrid/sparseGrid.cc:46 and multilevelSparseGrid.h:21; O(N^2) grid
completion, GridGeneration.cpp:333-392).
Multi-GPU runs (torchrun) solve one independent instance per rank (weak
scaling, no collective on the data path).
"""
import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from loadsg_b200.workloads import CONFIG1, config1_rhs  # noqa: E402  (numpy only, no native code)

METRIC = "time-to-1e-10 residual: learned-precond FP32+IR vs plain FP64 CG; matvec GB/s"


def workload(name, rank):
    """Seeded synthetic instance: (grid, coefficient family, params, f, description)."""
    from loadsg_b200 import workloads
    try:
        return workloads.workload(name, rank)
    except ValueError as e:
        raise SystemExit(str(e))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def host_cores():
    """Cores this process may run on: the affinity mask, capped by a cgroup CPU
    quota when one is set (os.cpu_count() reports the whole host, and OpenMP
    with more threads than the quota allows slows to a crawl)."""
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    try:
        quota, period = open("/sys/fs/cgroup/cpu.max").read().split()[:2]
        if quota != "max":
            n = min(n, max(1, int(int(quota) // int(period))))
    except (OSError, ValueError):
        pass
    return max(1, n)


def reference_exe(d):
    """The reference harness: the -O3 timing build when it runs here, else the
    golden-vector build (-O2); (path, build name) or (None, reason)."""
    for sub, name in ((f"fast_d{d}", "-O3 -march=x86-64-v3"), (f"d{d}", "-O2 -march=x86-64-v2")):
        exe = os.path.join(ROOT, "oracle", "_ref", sub, "ref_harness")
        if os.path.exists(exe):
            try:
                with tempfile.TemporaryDirectory() as tmp:
                    subprocess.run([exe, "grid", tmp, "level=1"], check=True, capture_output=True, timeout=60)
                return exe, name
            except (subprocess.SubprocessError, OSError):
                continue
    return None, f"oracle/_ref/(fast_)d{d}/ref_harness missing or not runnable on this host"


def reference_config1(steps, warmup):
    """CG::solveHomogen of the reference (applications/cg_method.h:759-886) on the
    CPU-runnable instance, on the host cores, measured (never scaled).  Its stop
    rule is r^T D^-1 r <= eps; eps = 1e-20 f^T D^-1 f asks for a relative
    (preconditioned) residual of 1e-10, with D the reference's own Jacobi
    diagonal (Preconditioning, cg_method.h:81-754, command "diag").  The true
    relative residual is recomputed by the harness."""
    exe, build = reference_exe(3)
    if exe is None:
        return {"value": None, "unit": "s", "cores": 0, "kind": "reference", "sample": build}
    cores = host_cores()
    common = [f"level={CONFIG1['level']}", "coef=1", "cp=1,0.5,1,1,1"]
    times, reps = [], []
    with tempfile.TemporaryDirectory() as tmp:
        subprocess.run([exe, "grid", tmp] + common, check=True, capture_output=True,
                       env=dict(os.environ, OMP_NUM_THREADS="1"))
        n = int([l.split()[1] for l in open(os.path.join(tmp, "meta_grid.txt")) if l.startswith("N ")][0])
        f = config1_rhs(n)
        f.tofile(os.path.join(tmp, "f.f64"))
        # thread count: the reference's matvec is nearly serial and OpenMP can
        # oversubscribe a container's cores, so one timed matvec per candidate
        # picks the fastest setting
        probe = {}
        for t in sorted({1, 2, 4, cores}):
            if t > cores:
                continue
            env_t = dict(os.environ, OMP_NUM_THREADS=str(t), OMP_WAIT_POLICY="PASSIVE")
            try:
                subprocess.run([exe, "matvec", tmp, f"x={tmp}/f.f64"] + common, check=True, capture_output=True,
                               env=env_t, timeout=60)
                meta = dict(l.split()[:2] for l in open(os.path.join(tmp, "meta_matvec.txt")) if len(l.split()) >= 2)
                probe[t] = float(meta["matvec_seconds"])
            except (subprocess.SubprocessError, KeyError, OSError):
                continue
        threads = min(probe, key=probe.get) if probe else 1
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_WAIT_POLICY="PASSIVE")
        subprocess.run([exe, "diag", tmp] + common, check=True, capture_output=True, env=env, timeout=300)
        dg = np.fromfile(os.path.join(tmp, "diag.f64"))
        eps = 1e-20 * float(np.sum(f * f / dg))
        for k in range(max(0, min(warmup, 1)) + steps):
            try:
                subprocess.run([exe, "cg", tmp, f"f={tmp}/f.f64", f"eps={eps!r}"] + common, check=True,
                               capture_output=True, env=env, timeout=600)
            except subprocess.TimeoutExpired:
                return {"value": None, "unit": "s", "cores": cores, "kind": "reference",
                        "sample": f"reference CG on {CONFIG1['workload']} did not finish within 600 s"}
            meta = dict(l.split()[:2] for l in open(os.path.join(tmp, "meta_cg.txt")) if len(l.split()) >= 2)
            if k >= min(warmup, 1):
                times.append(float(meta["solve_seconds"]))
                reps.append(meta)
        x_ref = np.fromfile(os.path.join(tmp, "x.f64"))
    last = reps[-1]
    return {"value": float(np.mean(times)), "unit": "s", "cores": threads, "kind": "reference",
            "build": build, "threads": threads, "host_cores": cores, "matvec_seconds_by_threads": probe,
            "iterations": int(last["iterations"]),
            "rel_residual": float(last["relres"]), "precond_seconds": float(last["precond_seconds"]),
            "eps": eps, "times": times, "n_points": n, "x_norm": float(np.linalg.norm(x_ref)),
            "sample": (f"the reference's CG::solveHomogen (Jacobi) on {CONFIG1['workload']} ({n} points), "
                       f"eps = 1e-20 f^T D^-1 f, {threads} thread(s) (fastest of {sorted(probe)} by a timed matvec), "
                       f"{build}, measured over {len(times)} solve(s)")}


def boundary_rhs_leg(lsg, torch, stream, reference=True):
    """Boundary-data right-hand sides (InHomoBoundaryRHSHierarchical,
    MatrixVectorMultiplication/RHS.cpp:697-1008, and CalcHierarchicalBasisForRHS,
    RHS.cpp:6-41) on d = 3 regular grids of level 5 and 7 with their boundary
    grids (completeNeumannGrid), boundary data g = exp(0.3 sin(pi x0) - 0.2 x1 +
    x2^2).  Device times (CUDA events, mean of 3 after a call that builds the
    tables) per form, and the host-buffer call of all three forms; the
    reference's own forms (oracle/_ref) run on level 5, the largest level it
    finishes in seconds."""
    out = {}
    for L in (5, 7):
        g = lsg.AdaptiveSparseGrid.regular(3, L)
        ng = lsg.AdaptiveSparseGrid.neumann(3, L)
        x = ng.coordinates()
        b = ng.boundary_mask()
        gv = np.where(b, np.exp(0.3 * np.sin(np.pi * x[:, 0]) - 0.2 * x[:, 1] + x[:, 2] ** 2), 0.0)
        m = lsg.MatrixVectorHomogen(g)
        rhs = lsg.InHomoBoundaryRHSHierarchical(m, ng)
        t0 = time.perf_counter()
        lsg.CalcHierarchicalBasisForRHS(gv, ng)
        hier_ms = (time.perf_counter() - t0) * 1e3
        y = np.zeros(g.n)
        rhs.multiply(gv, y)  # builds the tables
        hd = torch.tensor(gv, device="cuda")
        yd = torch.zeros(g.n, dtype=torch.float64, device="cuda")
        ms = []
        for kind in (lsg.BDRHS_GRADIENT, lsg.BDRHS_MASS, lsg.BDRHS_MASS_COEFF):
            rhs.multiply_device(kind, hd.data_ptr(), yd.data_ptr(), stream)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(3):
                rhs.multiply_device(kind, hd.data_ptr(), yd.data_ptr(), stream)
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1) / 3)
        t0 = time.perf_counter()
        for meth in (rhs.multiply, rhs.multiply_mass, rhs.multiply_mass_coeff):
            meth(gv, y)
        e2e_ms = (time.perf_counter() - t0) * 1e3
        # the whole right-hand side of -lap u = f, u = g on the boundary (PDE_Poisson_InHomRHS::SetUp)
        fv = np.exp(-x[:, 0] * x[:, 1]) + x[:, 2]
        gb = np.where(b, np.exp(0.3 * np.sin(np.pi * x[:, 0]) - 0.2 * x[:, 1] + x[:, 2] ** 2), 0.0)
        pde = lsg.PDE_Poisson_InHomRHS(ng, g, m)
        t0 = time.perf_counter()
        pde.SetUp(fv, gb)
        setup_ms = (time.perf_counter() - t0) * 1e3
        out[f"d3_L{L}"] = {"points": g.n, "boundary_points": int(b.sum()), "hierarchize_host_call_ms": hier_ms,
                           "gradient_ms": ms[0], "mass_ms": ms[1], "mass_coeff_ms": ms[2],
                           "three_forms_host_call_ms": e2e_ms, "pde_poisson_setup_host_call_ms": setup_ms}
        log(f"boundary rhs d=3 L{L}: {g.n} points, {int(b.sum())} boundary points, device ms {ms}")
    exe = os.path.join(ROOT, "oracle", "_ref", "d3", "ref_harness")
    if reference and os.path.exists(exe):
        cores = host_cores()
        env = dict(os.environ, OMP_NUM_THREADS=str(cores), OMP_WAIT_POLICY="PASSIVE")
        with tempfile.TemporaryDirectory() as tmp:
            try:
                subprocess.run([exe, "bdrhs", tmp, "level=5", "gfam=4", "gp=1,0.5"], check=True, capture_output=True,
                               env=env, timeout=300)
                meta = dict(l.split()[:2] for l in open(os.path.join(tmp, "meta_bdrhs.txt")) if len(l.split()) >= 2)
                out["reference_d3_L5"] = {"threads": cores, "gradient_s": float(meta["stiff_seconds"]),
                                          "mass_s": float(meta["mass_seconds"]),
                                          "mass_coeff_s": float(meta["coeff_seconds"])}
            except (subprocess.SubprocessError, KeyError, OSError) as e:
                out["reference_d3_L5"] = {"unavailable": str(e)[:200]}
    return out


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the cell-operator
# launches (k_sf and k_cells) of one FP32 matvec, from one ncu capture of the
# same workload on a B200; copied here, not measured by the bench run itself
TRAFFIC = {"d6_corner_L8": 2.0743e9}
TRAFFIC_SOURCE = ("ncu capture (one pass: dram__bytes_read.sum + dram__bytes_write.sum) of the k_sf and k_cells "
                  "launches of one FP32 product of this workload; copied, not measured in this run")


def same_instance_leg(lsg, torch, dev, stream, steps, ref=True):
    """The CPU-runnable configuration solved on the GPU with the right-hand side
    the reference arm solves (same grid, storage order and coefficient): FP64
    CG with the Jacobi diagonal (the reference's method) and FP32+IR with it,
    both to ||f - A x|| / ||f|| <= 1e-10, device time (mean of `steps` after a
    warm-up) and through host buffers; then the reference itself on the host."""
    g, fam, params, f_host, desc = workload("d3_regular_L7", 0)
    prob = lsg.MidpointDiffusion(fam, params)
    m = lsg.MatrixVectorHomogen(g, prob)
    f = torch.tensor(f_host, dtype=torch.float64, device=dev)
    x = torch.zeros_like(f)
    out = {"config": dict(CONFIG1), "description": desc}
    xs = {}
    for name, prec in (("fp64_cg_jacobi", lsg.FP64), ("fp32_ir_jacobi", lsg.FP32)):
        o = lsg.SolverOpts(1e-10, 1, 3000, 0, prec, 1000, 1e-5, 1)
        x.zero_()
        lsg.CG.solve_device(m, f.data_ptr(), x.data_ptr(), o, stream)  # warm-up (diagonal, graphs)
        secs = []
        for _ in range(max(1, steps)):
            x.zero_()
            r = lsg.CG.solve_device(m, f.data_ptr(), x.data_ptr(), o, stream)
            secs.append(r["seconds"])
        xs[name] = x.clone()
        xh = np.zeros(g.n)
        t0 = time.perf_counter()
        rh = lsg.CG.solveHomogen(1e-10, xh, f_host, m, prob, criterion=1, precision=prec, max_iter=3000,
                                 precond=0, inner_iter=1000, inner_tol=1e-5)
        host_s = time.perf_counter() - t0
        out[name] = {"seconds": float(np.mean(secs)), "iterations": r["iterations"],
                     "rel_residual": r["rel_residual"], "host_buffer_seconds": host_s,
                     "host_buffer_iterations": rh["iterations"]}
    out["fp32_ir_vs_fp64_solution_rel_diff"] = float(
        torch.linalg.norm(xs["fp32_ir_jacobi"] - xs["fp64_cg_jacobi"]) / torch.linalg.norm(xs["fp64_cg_jacobi"]))
    if ref:
        res = reference_config1(steps, 1)
        out["reference"] = res
        log(f"same instance: reference {res.get('value')} s ({res.get('iterations')} iterations)")
    log(f"same instance: FP64 {out['fp64_cg_jacobi']['seconds']:.4f} s, FP32+IR {out['fp32_ir_jacobi']['seconds']:.4f} s")
    return out


def max_over_ranks(x, dist, device):
    """The slowest rank's value (replicas: the job takes as long as its slowest GPU)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


_T0 = time.perf_counter()


def log(msg):
    """Progress on stderr (the JSON line alone goes to stdout)."""
    print(f"[bench {time.perf_counter() - _T0:8.1f}s] {msg}", file=sys.stderr, flush=True)


# device bytes per grid point of a batch operator (FP64 and FP32 buffers of the
# per-case slabs and the tables), by dimension: sizes the groups of the batch leg
BATCH_BYTES_PER_POINT = {4: 2000, 5: 3200, 6: 5000}


def batch_leg(lsg, torch, dev, stream, count=48, seed=7, levels=(3, 6), mem_gb=100.0, compare_every=1):
    """Many uneven grids solved in batches against grids solved one after
    another: d ~ U{4,5,6}, regular level ~ U{levels}, a = 1 + 0.9 prod
    sin(pi m_i x_i) with m_i ~ U{1..3}, f ~ U[-1,1]; FP32+IR with Jacobi to
    relative residual 1e-10.  Grids go into consecutive groups of at most
    mem_gb estimated device memory; each group is one batch (one CUDA graph
    per batched iteration).  The one-at-a-time comparison takes every
    compare_every-th grid, solved alone and as one batch."""
    rng = np.random.default_rng(seed)
    grids, probs, fs = [], [], []
    t0 = time.perf_counter()
    for _ in range(count):
        d = int(rng.integers(4, 7))
        level = int(rng.integers(levels[0], levels[1] + 1))
        g = lsg.AdaptiveSparseGrid.regular(d, level)
        grids.append(g)
        probs.append(lsg.MidpointDiffusion(lsg.COEF_SINPROD, [1.0, 0.9] + list(rng.integers(1, 4, d).astype(float))))
        fs.append(rng.uniform(-1, 1, g.n) * g.active)
    log(f"batch: {count} grids, {sum(g.n for g in grids)} points generated in {time.perf_counter() - t0:.1f}s")
    o = lsg.SolverOpts(1e-10, 1, 3000, 0, lsg.FP32, 1000, 1e-5, 1)
    warm = lsg.SolverOpts(1e-10, 1, 4, 0, lsg.FP32, 4, 1e-5, 1)  # builds and captures the iteration graphs

    def solve_batch(idx):
        t0 = time.perf_counter()
        b = lsg.Batch([grids[i] for i in idx], [probs[i] for i in idx])
        setup = time.perf_counter() - t0
        b.autotune(lsg.FP32, reps=2)
        f = torch.tensor(b.gather([fs[i] for i in idx]), dtype=torch.float64, device=dev)
        x = torch.zeros_like(f)
        b.solve_device(f.data_ptr(), x.data_ptr(), warm, stream)
        x.zero_()
        reps, tot = b.solve_device(f.data_ptr(), x.data_ptr(), o, stream)
        out = {"grids": len(idx), "points": int(b.size), "seconds": tot["seconds"], "iterations": tot["iterations"],
               "max_rel_residual": tot["rel_residual"], "converged": bool(tot["converged"]),
               "kernel_launches": int(tot["kernel_launches"]), "setup_seconds": setup}
        del b
        return out

    groups, cur, cur_b = [], [], 0.0
    for i, g in enumerate(grids):
        est = BATCH_BYTES_PER_POINT[g.d] * g.n / 1e9
        if cur and cur_b + est > mem_gb:
            groups.append(cur)
            cur, cur_b = [], 0.0
        cur.append(i)
        cur_b += est
    groups.append(cur)
    parts = []
    for gi, idx in enumerate(groups):
        r = solve_batch(idx)
        parts.append(r)
        log(f"batch group {gi}: {r['grids']} grids, {r['points']} points, solved in {r['seconds']:.3f}s "
            f"({r['iterations']} batched iterations, converged {r['converged']})")
    total = sum(r["seconds"] for r in parts)
    sub = list(range(0, count, compare_every))
    sub_batched = total if compare_every == 1 else solve_batch(sub)["seconds"]
    seq = 0.0
    for i in sub:
        m = lsg.MatrixVectorHomogen(grids[i], probs[i])
        fd = torch.tensor(fs[i], dtype=torch.float64, device=dev)
        xd = torch.zeros_like(fd)
        lsg.CG.solve_device(m, fd.data_ptr(), xd.data_ptr(), warm, stream)
        xd.zero_()
        r = lsg.CG.solve_device(m, fd.data_ptr(), xd.data_ptr(), o, stream)
        seq += r["seconds"]
        del m
    log(f"batch: {len(sub)} grids one at a time {seq:.3f}s, as one batch {sub_batched:.3f}s")
    return {"grids": count, "points": int(sum(g.n for g in grids)), "levels": list(levels),
            "description": batch_leg.__doc__.split(":", 1)[1].strip(),
            "groups": len(parts), "group_mem_gb": mem_gb, "seconds": total,
            "batched_iterations": max(r["iterations"] for r in parts),
            "max_rel_residual": max(r["max_rel_residual"] for r in parts),
            "all_converged": all(r["converged"] for r in parts),
            "kernel_launches": sum(r["kernel_launches"] for r in parts),
            "setup_seconds": sum(r["setup_seconds"] for r in parts), "group_results": parts,
            "compare_grids": len(sub), "compare_batched_seconds": sub_batched, "one_at_a_time_seconds": seq,
            "speedup": seq / sub_batched if sub_batched > 0 else None}


def d8_sweep(lsg, torch, solve_up_to=40000):
    """FP32/FP64 matvec time, algorithmic GB/s and cell-operator GFLOP/s on d=8
    grids refined toward the hyperplane x_1 = 1/2 (regular level L, 2 rounds
    adding the sons of points with |x_1 - 1/2| < 0.3 * 2^(1-r), completed),
    a = 1 + 0.5 sin(2 pi x_1) cos(2 pi x_2); on the smaller grids also the
    FP32+IR and FP64 solves to relative residual 1e-10."""
    try:
        hbm = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except Exception:
        hbm = 6650.0
    for level in (2, 3, 4):
        t0 = time.perf_counter()
        g = lsg.AdaptiveSparseGrid.adaptive(8, level, 2, 0.3, "plane")
        prob = lsg.MidpointDiffusion(lsg.COEF_SIN2PI, [1.0, 0.5])
        m = lsg.MatrixVectorHomogen(g, prob)
        setup = time.perf_counter() - t0
        info = m.info()
        x32 = torch.randn(g.n, dtype=torch.float32, device="cuda")
        y32 = torch.zeros_like(x32)
        x64, y64 = x32.double(), torch.zeros(g.n, dtype=torch.float64, device="cuda")
        m.profile(x32.data_ptr(), y32.data_ptr(), lsg.FP32, 1)
        ms32, by32, flops = m.profile(x32.data_ptr(), y32.data_ptr(), lsg.FP32, 3)
        ms64, by64, _ = m.profile(x64.data_ptr(), y64.data_ptr(), lsg.FP64, 2)
        line = {"sweep": "d8_plane", "level": level, "refine": 2, "n_points": g.n, "n_active": g.getDOFS(),
                "case_cells": int(info["case_cells"]), "device_bytes": int(info["device_bytes"]),
                "setup_seconds": setup, "fp32_ms": ms32[5], "fp64_ms": ms64[5],
                "fp32_gbs": by32[5] / (ms32[5] * 1e-3) / 1e9, "fp64_gbs": by64[5] / (ms64[5] * 1e-3) / 1e9,
                "fp32_hbm_frac": by32[5] / (ms32[5] * 1e-3) / 1e9 / hbm,
                "cell_op_gflops_fp32": flops / (ms32[3] * 1e-3) / 1e9}
        if g.n <= solve_up_to:
            rng = np.random.default_rng(0)
            f = torch.tensor(rng.uniform(-1, 1, g.n) * g.active, device="cuda")
            x = torch.zeros_like(f)
            st = torch.cuda.current_stream().cuda_stream
            for name, prec in (("fp32_ir", lsg.FP32), ("fp64", lsg.FP64)):
                x.zero_()
                r = lsg.CG.solve_device(m, f.data_ptr(), x.data_ptr(),
                                        lsg.SolverOpts(1e-10, 1, 20000, 0, prec, 1000, 1e-5, 1), st)
                line[f"{name}_solve"] = {"seconds": r["seconds"], "iterations": r["iterations"],
                                         "rel_residual": r["rel_residual"]}
        print(json.dumps(line), flush=True)
        del m


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--workload", default="d6_corner_L8")
    ap.add_argument("--precond", type=int, default=2, help="0 Jacobi, 1 none, 2 learned diagonal")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-bdrhs", action="store_true", help="skip the boundary-data right-hand-side leg")
    ap.add_argument("--batch-grids", type=int, default=48, help="grids in the batch leg")
    ap.add_argument("--batch-levels", default="3,6", help="regular levels of the batch grids: lo,hi")
    ap.add_argument("--batch-mem-gb", type=float, default=100.0, help="estimated device memory per batch")
    ap.add_argument("--batch-compare-every", type=int, default=1,
                    help="one-at-a-time comparison on every k-th grid (solved alone and as one batch)")
    ap.add_argument("--batch-only", action="store_true", help="run only the batch leg (one JSON line)")
    ap.add_argument("--sweep", action="store_true",
                    help="matvec sweep over d=8 grids refined toward x_1 = 1/2 (one JSON line per grid) instead")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-same-instance", action="store_true", help="skip the CPU-runnable same-instance leg")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        # the reference's own CPU code only: no part of this repository's library is loaded
        if rank != 0:
            return
        res = reference_config1(args.steps, args.warmup)
        line = {"metric": METRIC, "value": res["value"], "unit": "s", "impl": "reference", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": min(args.warmup, 1), "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": dict(CONFIG1),
                "cpu_baseline": res,
                "e2e": {"value": res["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    import loadsg_b200 as lsg

    torch.cuda.set_device(local)
    if args.sweep:
        if rank == 0:
            d8_sweep(lsg, torch)
        return
    if args.batch_only:
        dev = torch.device("cuda", local)
        b = batch_leg(lsg, torch, dev, torch.cuda.current_stream().cuda_stream, count=args.batch_grids,
                      levels=tuple(int(v) for v in args.batch_levels.split(",")), mem_gb=args.batch_mem_gb,
                      compare_every=args.batch_compare_every)
        if rank == 0:
            print(json.dumps({"batch": b}))
        return
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    g, fam, params, f_host, desc = workload(args.workload, rank)
    prob = lsg.MidpointDiffusion(fam, params)
    t0 = time.perf_counter()
    m = lsg.MatrixVectorHomogen(g, prob)
    setup_s = time.perf_counter() - t0
    info = m.info()
    log(f"operator: {g.n} points in {setup_s:.1f}s")
    # launch parameters picked by the autotuner (setup, not timed)
    tune_setting, tune_ms, tune_default_ms = m.autotune(lsg.FP32, reps=3)
    log(f"autotune: {tune_default_ms:.2f} -> {tune_ms:.2f} ms per FP32 matvec")
    # preconditioner setup: exact Jacobi diagonal vs the learned diagonal
    precond = args.precond
    weights = os.path.join(ROOT, "loadsg_b200", "weights", f"diag_mlp_d{g.d}.npz")
    learned_ms = jacobi_ms = None
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    m.diagonal(prob)
    torch.cuda.synchronize()
    jacobi_ms = (time.perf_counter() - t0) * 1e3
    if precond == 2:
        if os.path.exists(weights):
            from loadsg_b200.learned import MLP
            net = MLP.load(weights)
            net.install(m)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            net.install(m)
            torch.cuda.synchronize()
            learned_ms = (time.perf_counter() - t0) * 1e3
        else:
            precond = 0
    dev = torch.device("cuda", local)
    f = torch.tensor(f_host, dtype=torch.float64, device=dev)
    x = torch.zeros(g.n, dtype=torch.float64, device=dev)

    def opts(precision, precond):
        return lsg.SolverOpts(1e-10, 1, 3000, precond, precision, 1000, 1e-5, 1)

    stream = torch.cuda.current_stream().cuda_stream

    failed = []  # solves that ended in a library error: logged and reported, the line still prints

    def guarded(fn, what):
        try:
            return fn()
        except lsg.LsgError as e:
            log(f"{what} failed: {e}")
            failed.append(f"{what}: {e}")
            return None

    def solve(precision, precond, what="solve"):
        x.zero_()
        return guarded(lambda: lsg.CG.solve_device(m, f.data_ptr(), x.data_ptr(), opts(precision, precond), stream),
                       what)

    log(f"preconditioner setup: jacobi {jacobi_ms} ms, learned {learned_ms} ms")
    for _ in range(args.warmup):
        rep = solve(lsg.FP32, precond, "warm-up solve")
        if rep:
            log(f"warm-up solve: {rep['seconds']:.2f}s, {rep['iterations']} iterations")
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(args.steps):
            rep = solve(lsg.FP32, precond, "timed solve")
            if rep:
                reps.append(rep)
                log(f"timed solve: {rep['iterations']} iterations, {rep['outer_iterations']} refinement steps")
        ev1.record()
        torch.cuda.synchronize()
    step_s = max_over_ranks(ev0.elapsed_time(ev1) / 1e3 / args.steps, dist, dev)
    x_ir = x.clone()

    # plain FP64 CG on the same instance (the comparison the metric names; the
    # reference's CG is always Jacobi-preconditioned), and FP32+IR with Jacobi
    log(f"timed: {step_s:.2f}s per solve")
    rep64 = solve(lsg.FP64, 0, "FP64 CG") or {}
    log(f"FP64 CG: {rep64.get('seconds')}s")
    # the FP32+IR solution's distance to the FP64 CG solution of the same system
    sol_err = float(torch.linalg.norm(x_ir - x) / torch.linalg.norm(x)) if rep64 else None
    log(f"FP32+IR vs FP64 solution: relative difference {sol_err}")
    rep_jac = (solve(lsg.FP32, 0, "FP32+IR Jacobi") or {}) if precond != 0 else reps[-1] if reps else {}
    log(f"FP32+IR Jacobi: {rep_jac.get('seconds')}s")
    # end to end through the C-ABI with host buffers
    xh = np.zeros(g.n)
    torch.cuda.synchronize()
    te = time.perf_counter()
    for _ in range(args.steps):
        xh[:] = 0.0
        rep_e2e = guarded(lambda: lsg.CG.solveHomogen(1e-10, xh, f_host, m, prob, criterion=1, precision=lsg.FP32,
                                                      max_iter=3000, precond=precond, inner_iter=1000,
                                                      inner_tol=1e-5), "e2e solve")
        if rep_e2e:
            log(f"e2e solve: {rep_e2e['iterations']} iterations, {rep_e2e['outer_iterations']} refinement steps")
    e2e_s = (time.perf_counter() - te) / args.steps
    log(f"e2e: {e2e_s:.2f}s per solve")

    same = None if args.no_same_instance else guarded(
        lambda: same_instance_leg(lsg, torch, dev, stream, args.steps,
                                  ref=(not args.no_cpu_baseline and world == 1 and rank == 0)), "same-instance leg")

    # matvec bandwidth and the cell-operator roofline (CUDA events inside the library)
    x32 = torch.randn(g.n, dtype=torch.float32, device=dev)
    y32 = torch.zeros(g.n, dtype=torch.float32, device=dev)
    x64 = x32.double()
    y64 = torch.zeros(g.n, dtype=torch.float64, device=dev)
    m.profile(x32.data_ptr(), y32.data_ptr(), lsg.FP32, 2)
    ms32, by32, flops = m.profile(x32.data_ptr(), y32.data_ptr(), lsg.FP32, 5)
    ms64, by64, _ = m.profile(x64.data_ptr(), y64.data_ptr(), lsg.FP64, 3)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        hbm, peak_src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        hbm, peak_src = 6650.0, "fallback"
    # the cell operator's launches (k_sf, and k_cells for sparse slabs) of one FP32
    # matvec: algorithmic bytes (slab read, slab written, collapsed coefficients)
    # over their CUDA-event time
    achieved = by32[3] / (ms32[3] * 1e-3) / 1e9
    traffic = TRAFFIC.get(args.workload)

    batch = None if args.no_batch else guarded(lambda: batch_leg(lsg, torch, dev, stream, count=args.batch_grids),
                                               "batch leg")
    bdrhs = None if args.no_bdrhs else guarded(
        lambda: boundary_rhs_leg(lsg, torch, stream, reference=not args.no_cpu_baseline and world == 1 and rank == 0),
        "boundary rhs leg")

    if rank != 0:
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    cpu = same.get("reference") if same else None
    last = reps[-1] if reps else {}
    line = {
        "metric": METRIC, "value": step_s, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": step_s * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 matvec / f64 refinement", "data": "synthetic",
        "config": {"workload": args.workload, "description": desc, "n_points": g.n, "n_active": g.getDOFS(),
                   "tolerance": 1e-10, "precond": ["jacobi", "none", "learned"][precond],
                   "parallelism": f"replicas x{world}", "l2": "working set larger than L2 (126 MB)"},
        "iterations": last.get("iterations"), "outer_iterations": last.get("outer_iterations"),
        "rel_residual": last.get("rel_residual"), "failed_solves": failed,
        "fp64_cg": {"seconds": rep64.get("seconds"), "iterations": rep64.get("iterations"),
                    "rel_residual": rep64.get("rel_residual"), "precond": "jacobi (the reference's method)"},
        "fp32_ir_vs_fp64_solution_rel_diff": sol_err,
        "speedup_vs_fp64_cg": rep64["seconds"] / step_s if rep64 and step_s > 0 else None,
        "fp32_ir_jacobi": {"seconds": rep_jac.get("seconds"), "iterations": rep_jac.get("iterations"),
                           "rel_residual": rep_jac.get("rel_residual")},
        "preconditioner_setup_ms": {"jacobi_exact_diag": jacobi_ms, "learned": learned_ms},
        "tuning": {"setting": tune_setting, "matvec_ms_fp32": tune_ms, "matvec_ms_fp32_default": tune_default_ms},
        "matvec": {"fp32_ms": ms32[5], "fp64_ms": ms64[5], "fp32_gbs": by32[5] / (ms32[5] * 1e-3) / 1e9,
                   "fp64_gbs": by64[5] / (ms64[5] * 1e-3) / 1e9,
                   "phases": ["nodal", "P init", "prolongation", "cell operator", "restriction wavefronts + gather"],
                   "phase_ms_fp32": list(ms32[:5]), "phase_ms_fp64": list(ms64[:5]),
                   "phase_bytes_fp32": list(by32[:5]),
                   "cell_op_gflops_fp32": flops / (ms32[3] * 1e-3) / 1e9,
                   # nominal FP32 rate: 148 SMs x 128 lanes x 2 flops x 1.965 GHz = 74.4 TFLOP/s
                   "cell_op_fp32_frac_of_nominal": flops / (ms32[3] * 1e-3) / 74.4e12},
        "roofline": {"bound": "hbm", "kernel": "cell operator (k_sf; k_cells for sparse slabs), FP32",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_source": peak_src, "traffic": traffic,
                     "traffic_source": TRAFFIC_SOURCE if traffic else None,
                     "bytes_per_matvec": by32[3], "ms_per_matvec": ms32[3]},
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 16 * g.n, "d2h_bytes_per_step": 8 * g.n},
        "setup_seconds": setup_s, "plan_seconds": info["plan_seconds"], "device_bytes": info["device_bytes"],
        "clocks": clk.summary(),
        "gpu_launches": int(sum(r["kernel_launches"] for r in reps)),
    }
    if same is not None:
        line["same_instance"] = same
    if batch is not None:
        line["batch"] = batch
    if bdrhs is not None:
        line["boundary_rhs"] = bdrhs
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
