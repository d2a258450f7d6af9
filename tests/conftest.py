import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

_ALL = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))
# operator fixtures (matvec, diagonal, CG, transforms) and boundary-data
# right-hand-side fixtures (bd_*: a grid with boundary points beside the grid)
GOLDEN = [p for p in _ALL if not os.path.basename(p).startswith(("bd_", "pde_", "cmp_", "ex_"))]
GOLDEN_BD = [p for p in _ALL if os.path.basename(p).startswith("bd_")]
# right-hand sides of boundary-data problems (PDE_*::SetUp) and their transforms
GOLDEN_PDE = [p for p in _ALL if os.path.basename(p).startswith("pde_")]
# a caller's point set completed by the reference (completeDirichletGrid / completeNeumannGrid)
GOLDEN_COMPLETE = [p for p in _ALL if os.path.basename(p).startswith("cmp_")]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def load_golden(path):
    z = np.load(path)
    d = int(z["d"])
    out = {k: z[k] for k in z.files}
    out["points"] = z["points"].reshape(-1, d)
    out["name"] = os.path.basename(path)[:-4]
    return out


@pytest.fixture(params=GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def golden(request):
    return load_golden(request.param)
