"""The factorised dense-slab cell operator (lsg_sf.h) on the CPU.

The GPU applies the level-T cell operator of a dense slab as
z = E^T diag(a~ Lambda) E u over per-dimension reduced modes, with dimensions
of one interior node collapsed into summed coefficients, the outermost
dimensions chunked to fit shared memory and the two innermost fused in
registers.  lsg_plan_check_slab_operator runs the host emulation of exactly
that plan next to the cell-by-cell apply of the reference's
LocalStiffnessMatrices::applyLocalMatrix
(localStiffnessMatrices/LocalStiffnessMatrices.cpp:555-582) on random
coefficients and inputs; the two must agree to rounding for every slab shape,
both forms, and work-space limits small enough to force every chunking path.
"""
import ctypes

import numpy as np
import pytest

import loadsg_b200 as lsg

P = ctypes.c_void_p


def _lib():
    L = lsg.lib()
    f = L.lsg_plan_check_slab_operator
    f.restype = ctypes.c_int
    f.argtypes = [P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32] + [P] * 5
    return L


def _check_grid(g, wcaps, nas=(7, 3), maxslabs=25, seed=0):
    L = _lib()
    plan = P()
    lsg._check(L.lsg_plan_create(g.d, lsg._ptr(g.points), lsg._ptr(g.active), g.n, ctypes.byref(plan)))
    try:
        info = lsg._Info()
        L.lsg_plan_info(plan, ctypes.byref(info))
        nD = info.n_depths
        cells = np.zeros(nD, np.int64)
        L.lsg_plan_export_cell_counts(plan, lsg._ptr(cells))
        rng = np.random.default_rng(seed)
        worst, paths = 0.0, set()
        for t in rng.permutation(nD)[:maxslabs]:
            cnt = ctypes.c_int64(0)
            L.lsg_plan_export_slab(plan, int(t), None, ctypes.byref(cnt))
            a = rng.uniform(0.5, 2.0, cells[t])
            u = rng.uniform(-1.0, 1.0, cnt.value)
            for form in (lsg.FORM_STIFFNESS, lsg.FORM_MASS):
                for w in wcaps:
                    for na in nas:
                        z1, z2, inf = np.zeros(cnt.value), np.zeros(cnt.value), np.zeros(6, np.int32)
                        rc = L.lsg_plan_check_slab_operator(plan, int(t), form, w, na, lsg._ptr(a), lsg._ptr(u),
                                                            lsg._ptr(z1), lsg._ptr(z2), lsg._ptr(inf))
                        if rc != 0:
                            msg = L.lsg_last_error().decode()
                            assert "do not fit" in msg, msg  # a x b alone above a tiny work space
                            continue
                        worst = max(worst, np.abs(z1 - z2).max() / np.abs(z1).max())
                        paths.add((int(inf[0]), int(inf[1]), inf[3] > 0, inf[4] > 0, inf[5] > 0))
        return worst, paths
    finally:
        L.lsg_plan_destroy(plan)


@pytest.mark.parametrize("d,level", [(1, 6), (2, 5), (3, 4), (4, 3), (5, 3), (6, 3), (7, 2), (8, 2)])
def test_factorised_equals_cell_loop_regular(d, level):
    worst, paths = _check_grid(lsg.AdaptiveSparseGrid.regular(d, level), wcaps=(1 << 30, 4096, 600))
    assert worst < 1e-13, worst
    assert paths


def test_factorised_equals_cell_loop_adaptive_corner():
    # the benchmark's grid family (dense slabs of a corner-refined d = 6 grid)
    worst, paths = _check_grid(lsg.AdaptiveSparseGrid.adaptive(6, 4, 1, 0.6, "corner"), wcaps=(1 << 30, 4096, 600),
                               maxslabs=12)
    assert worst < 1e-13, worst
    assert any(p[1] > 0 for p in paths)  # a chunked plan was exercised


@pytest.mark.parametrize("d,level,wcaps", [(4, 5, (200, 90, 30)), (6, 4, (300, 100, 40)), (3, 7, (500, 120, 40))])
def test_factorised_every_chunking_path(d, level, wcaps):
    worst, paths = _check_grid(lsg.AdaptiveSparseGrid.regular(d, level), wcaps=wcaps, maxslabs=25)
    assert worst < 1e-13, worst
    assert max(p[1] for p in paths) >= 2      # two chunked dimensions
    assert any(not p[2] for p in paths)       # no register dimension (a virtual)
    assert any(p[0] >= 1 for p in paths)      # shared-memory sweeps


def test_fast_division():
    """The kernels divide by plan constants with a multiply-high: check it."""
    L = _lib()
    # exercised through the plan: any failure would show above; here the rule itself
    rng = np.random.default_rng(3)
    for dv in list(range(1, 300)) + [int(v) for v in rng.integers(1, 1 << 24, 200)]:
        s = int(np.ceil(np.log2(dv))) if dv > 1 else 0
        m = ((1 << 32) * ((1 << s) - dv)) // dv + 1
        q = np.concatenate([np.arange(0, 4096), rng.integers(0, 1 << 31, 4096)]).astype(np.uint64)
        got = (((q * np.uint64(m)) >> np.uint64(32)) + q) >> np.uint64(s)
        assert np.array_equal(got, q // np.uint64(dv)), dv
    assert L is not None
