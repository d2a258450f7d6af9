"""The allocation-free matvec entry point (lsg_matvec_device_noalloc).

It exists for callers that cannot allocate device memory when they need a
product: host applications whose own allocator owns the whole device, and
loops that cannot pay for the synchronisation of cudaMalloc/cudaFree.  Its
work space is a fixed array in the library.  This file is collected last so
that a failure here leaves every other test already run; it passes alone in a
fresh process as well."""
import ctypes

import numpy as np
import pytest

import loadsg_b200 as lsg

pytestmark = pytest.mark.gpu


def _call(m, x, y, precision):
    rc = lsg.lib().lsg_matvec_device_noalloc(m._h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                              precision, None)
    return rc


@pytest.mark.parametrize("precision", [lsg.FP64, lsg.FP32])
def test_noalloc_matches_allocating_entry_point(precision):
    """On a fresh operator the no-alloc call comes first: it must not grow the
    operator's device memory nor take memory from the device; two calls in a
    row, and then the allocating entry point, give the same bits."""
    import torch
    dt = torch.float64 if precision == lsg.FP64 else torch.float32
    g = lsg.AdaptiveSparseGrid.regular(3, 6)
    prob = lsg.MidpointDiffusion(lsg.COEF_SINPROD, [1.0, 0.5, 1, 1, 1])
    x = torch.tensor(np.random.default_rng(7).uniform(-1, 1, g.n), dtype=dt, device="cuda")
    # load the matvec kernels once through another operator, so that the check
    # below sees only what the call itself would take
    warm = lsg.MatrixVectorHomogen(g, prob)
    y = torch.zeros(g.n, dtype=dt, device="cuda")
    assert _call(warm, x, y, precision) == 0, lsg.lib().lsg_last_error()
    torch.cuda.synchronize()
    m = lsg.MatrixVectorHomogen(g, prob)
    bytes0, free0 = m.info()["device_bytes"], torch.cuda.mem_get_info()[0]
    outs = []
    for _ in range(2):  # two calls in a row share (and reuse) the fixed array
        y = torch.full((g.n,), 3.0, dtype=dt, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        assert _call(m, x, y, precision) == 0, lsg.lib().lsg_last_error()
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free_before
        outs.append(y.clone())
    assert m.info()["device_bytes"] == bytes0
    assert torch.cuda.mem_get_info()[0] >= free0 - 2 * g.n * x.element_size()  # only the test's own y tensors
    y_ref = torch.zeros(g.n, dtype=dt, device="cuda")
    m.multiplication_device(x.data_ptr(), y_ref.data_ptr(), precision)
    torch.cuda.synchronize()
    assert torch.equal(outs[0], outs[1])
    assert torch.equal(outs[0], y_ref)


def test_noalloc_rejects_oversized_grid():
    import torch
    g = lsg.AdaptiveSparseGrid.regular(6, 6)  # needs more than the fixed 32 MiB
    prob = lsg.MidpointDiffusion(lsg.COEF_CONST, [1.0])
    m = lsg.MatrixVectorHomogen(g, prob)
    x = torch.zeros(g.n, dtype=torch.float64, device="cuda")
    y = torch.zeros(g.n, dtype=torch.float64, device="cuda")
    rc = _call(m, x, y, lsg.FP64)
    assert rc == -1
    assert b"fixed array holds" in lsg.lib().lsg_last_error()
