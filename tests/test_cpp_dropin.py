"""The header-only C++ drop-in (include/loadsg/loadsg.hpp) compiles against
liblsg.so on the CPU; on a GPU it solves a d=3 problem through the C-ABI."""
import os
import subprocess

import pytest

import loadsg_b200 as lsg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_example(tmp_path):
    exe = str(tmp_path / "dropin_example")
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "dropin_example.cpp"), lsg.LIB_PATH,
           "-Wl,-rpath," + os.path.dirname(lsg.LIB_PATH), "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_header_neumann_completion_matches_generator(tmp_path):
    """completeNeumannGrid of the C++ drop-in equals the library's generator
    (itself pinned to the reference's storage order), point for point."""
    import numpy as np
    exe = str(tmp_path / "neumann_grid")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "neumann_grid.cpp"), lsg.LIB_PATH,
                    "-Wl,-rpath," + os.path.dirname(lsg.LIB_PATH), "-o", exe], check=True, capture_output=True)
    for level in (3, 5):
        out = subprocess.run([exe, str(level)], check=True, capture_output=True, text=True).stdout
        rows = np.array([list(map(int, line.split())) for line in out.splitlines()], np.int64)
        g = lsg.AdaptiveSparseGrid.neumann(3, level)
        assert np.array_equal(rows[:, 1:], g.points) and np.array_equal(rows[:, 0], g.active)


def test_header_adaptive_example_matches_reference(tmp_path):
    """The reference's adaptive-grid example (two points, completeDirichletGrid)
    through the C++ drop-in: the grid the compiled reference builds from the
    same two points (tests/golden/cmp_d2_example.npz), 23 DOFs and 18 hanging
    nodes."""
    import numpy as np
    exe = str(tmp_path / "gridgeneration_adaptive")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "gridgeneration_adaptive.cpp"), lsg.LIB_PATH,
                    "-Wl,-rpath," + os.path.dirname(lsg.LIB_PATH), "-o", exe], check=True, capture_output=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.splitlines()
    rows = np.array([list(map(int, line.split())) for line in out if not line.startswith("#")], np.int64)
    z = np.load(os.path.join(ROOT, "tests", "golden", "cmp_d2_example.npz"))
    assert np.array_equal(rows[:, 1:], z["points"]) and np.array_equal(rows[:, 0], z["active"])
    assert out[-1] == "# 23 18"


def test_poisson_example_port_compiles(tmp_path):
    """The reference's Poisson example written against the drop-in
    (tests/cpp/poisson_regular_port.cpp) compiles and links; its table is
    checked on the GPU through the same library calls in tests/test_poisson_example.py."""
    exe = str(tmp_path / "poisson_regular_port")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "poisson_regular_port.cpp"), lsg.LIB_PATH,
                    "-Wl,-rpath," + os.path.dirname(lsg.LIB_PATH), "-o", exe], check=True, capture_output=True)
    assert os.path.exists(exe)


def test_dropin_header_compiles_and_links(tmp_path):
    assert os.path.exists(build_example(tmp_path))


@pytest.mark.gpu
def test_dropin_solves_on_gpu(tmp_path):
    exe = build_example(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "relres" in r.stdout
