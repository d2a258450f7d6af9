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


def test_dropin_header_compiles_and_links(tmp_path):
    assert os.path.exists(build_example(tmp_path))


@pytest.mark.gpu
def test_dropin_solves_on_gpu(tmp_path):
    exe = build_example(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "relres" in r.stdout
