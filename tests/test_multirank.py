"""Host-side logic of bench.py for N > 1 GPUs, on CPU: replicas only (one
independent instance per rank, no collective on the data path), timing is the
maximum over ranks, and the reference arm runs on rank 0 alone.  Ranks are
processes on a gloo process group over 127.0.0.1."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = bench.max_over_ranks(1.5 + rank, dist, "cpu")
    finally:
        dist.destroy_process_group()


def test_time_is_max_over_ranks():
    world = 2
    with mp.get_context("spawn").Manager() as mgr:  # no fork of a multi-threaded parent
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        assert dict(out) == {0: 2.5, 1: 2.5}


def test_single_process_value_passes_through():
    assert bench.max_over_ranks(3.25, None, "cpu") == 3.25


def test_each_rank_solves_its_own_instance():
    # the seeded synthetic workloads (the d = 3 level-7 case is the reference's
    # fixed instance, the same on every rank, and is not one of them)
    g0, fam0, p0, f0, _ = bench.workload("d6_regular_L3", 0)
    g1, fam1, p1, f1, _ = bench.workload("d6_regular_L3", 1)
    assert g0.n == g1.n and fam0 == fam1  # same size per GPU: weak scaling
    assert not np.array_equal(f0, f1)     # independent right-hand sides
    assert not np.any(f0[g0.active == 0])
    ga, _, _, fa, _ = bench.workload("d3_regular_L7", 0)
    gb, _, _, fb, _ = bench.workload("d3_regular_L7", 1)
    assert ga.n == 7423 and np.array_equal(fa, fb)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_line():
    """Rank 0 of the reference arm: the reference's own CG::solveHomogen on the
    CPU-runnable instance (7,423 points), one JSON line with the native arm's
    metric and unit, a measured (never scaled) value, and no part of this
    repository's library loaded."""
    import json
    exe = os.path.join(ROOT, "oracle", "_ref", "fast_d3", "ref_harness")
    if not os.path.exists(exe):
        pytest.skip("the reference harness (oracle/_ref) is not built")
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '1']; "
            "runpy.run_path('bench.py', run_name='__main__'); "
            "import loadsg_b200; assert loadsg_b200._LIB is None, 'liblsg.so was loaded'")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == "s"
    assert line["higher_is_better"] is False and line["config"]["n_points"] == 7423
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["n_points"] == 7423 and cb["iterations"] > 0
    assert cb["rel_residual"] <= 1.01e-10 and line["value"] == cb["value"] > 0
    assert line["e2e"] == {"value": line["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
