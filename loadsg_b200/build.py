"""Builds loadsg_b200/liblsg.so for sm_100a (in-tree, no JIT cache).

    python -m loadsg_b200.build

nvcc compiles the CUDA translation unit and the host planner (OpenMP) and
links them into one shared library with the static CUDA runtime.
"""
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "liblsg.so")
BUILD = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["lsg_device.cu", "lsg_batch.cu", "lsg_basis.cu", "lsg_bdrhs.cu", "lsg_mlp.cu", "lsg_plan.cpp", "lsg_sf.cpp", "lsg_grid.cpp", "lsg_gridgen.cpp"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "lsg.h"))
    deps.append(__file__)
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force=False, verbose=False):
    if not force and not _stale():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    host = ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []
    common = host + ["-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp", "-lineinfo"]
    def compile_one(s):
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        cmd = [cc] + common + ARCH + ["-c", src, "-o", obj]
        if s.endswith(".cu") and verbose:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose:
            sys.stderr.write(r.stderr)
        return obj

    with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    tmp = OUT + ".tmp"
    cmd = [cc] + host + ARCH + ["-shared", "-o", tmp] + objs + ["-Xcompiler", "-fopenmp", "-lgomp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
