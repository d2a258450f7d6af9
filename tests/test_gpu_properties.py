"""Size-independent properties of the operator at the benchmark's full size
(d = 6, 499,107 points, the bench workload) and on a d = 8 grid, where no
reference output exists: the prewavelet stiffness matrix is symmetric and
positive definite on the active points, the product is linear, and FP32
agrees with FP64 to single-precision rounding."""
import numpy as np
import pytest

import bench
import loadsg_b200 as lsg

pytestmark = pytest.mark.gpu


def grids():
    g6, fam, params, _, _ = bench.workload("d6_adaptive_corner", 0)
    g8 = lsg.AdaptiveSparseGrid.adaptive(8, 3, 2, 0.3, "plane")
    return [("d6_corner_499k", g6, lsg.MidpointDiffusion(fam, params)),
            ("d8_plane_31k", g8, lsg.MidpointDiffusion(lsg.COEF_SIN2PI, [1.0, 0.5]))]


@pytest.fixture(scope="module", params=[0, 1], ids=["d6_corner_499k", "d8_plane_31k"])
def case(request):
    import torch
    name, g, prob = grids()[request.param]
    m = lsg.MatrixVectorHomogen(g, prob)
    act = torch.tensor(g.active, device="cuda", dtype=torch.float64)

    def apply(x, precision=lsg.FP64):
        dt = torch.float64 if precision == lsg.FP64 else torch.float32
        xin = x.to(dt).contiguous()
        y = torch.zeros_like(xin)
        m.multiplication_device(xin.data_ptr(), y.data_ptr(), precision)
        torch.cuda.synchronize()
        return y.double() * act

    gen = torch.Generator(device="cuda").manual_seed(7)
    x = torch.rand(g.n, device="cuda", dtype=torch.float64, generator=gen) * 2 - 1
    y = torch.rand(g.n, device="cuda", dtype=torch.float64, generator=gen) * 2 - 1
    return name, apply, x * act, y * act


def test_symmetric(case):
    _, apply, x, y = case
    Ax, Ay = apply(x), apply(y)
    a, b = float(x @ Ay), float(y @ Ax)
    assert abs(a - b) <= 1e-12 * float(x.norm() * Ay.norm())


def test_positive_definite(case):
    _, apply, x, y = case
    for v in (x, y, x - 0.5 * y):
        assert float(v @ apply(v)) > 0.0


def test_linear(case):
    _, apply, x, y = case
    lhs = apply(1.5 * x - 0.25 * y)
    rhs = 1.5 * apply(x) - 0.25 * apply(y)
    assert float((lhs - rhs).abs().max()) <= 1e-12 * float(rhs.abs().max())


def test_fp32_matches_fp64(case):
    _, apply, x, _ = case
    y64, y32 = apply(x), apply(x, lsg.FP32)
    assert float((y32 - y64).abs().max()) <= 2e-5 * float(y64.abs().max())
