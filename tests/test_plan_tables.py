"""Host planner (liblsg.so, no GPU): integer tables bit-exact against the
reference's own lookups dumped in tests/golden, and the C-ABI symbol set."""
import ctypes
import os
import re

import numpy as np
import pytest

import loadsg_b200 as lsg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def make_plan(golden):
    return lsg.Plan(lsg.AdaptiveSparseGrid(golden["points"], golden["active"]))


def test_all_header_symbols_exported():
    hdr = open(os.path.join(ROOT, "include", "lsg.h")).read()
    names = set(re.findall(r"\b(lsg_[a-z0-9_]+)\s*\(", hdr))
    names.discard("lsg_operator")
    L = ctypes.CDLL(lsg.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    assert len(names) >= 20


def test_depth_list_and_case_order(golden):
    if "tables_depthlist" not in golden:
        pytest.skip("no tables in this fixture")
    d = int(golden["d"])
    p = make_plan(golden)
    D = p.depths()
    assert np.array_equal(D.ravel(), golden["tables_depthlist"])
    off = golden["tables_sorted_off"]
    srt = golden["tables_sorted"].reshape(-1, d)
    for c in range(1 << d):
        ids = p.sorted_depths(c)
        assert np.array_equal(D[ids], srt[off[c]:off[c + 1]])


def test_exact_depth_points_and_slabs(golden):
    if "tables_exact" not in golden:
        pytest.skip("no tables in this fixture")
    d = int(golden["d"])
    p = make_plan(golden)
    D = p.depths()
    ex, exo = golden["tables_exact"], golden["tables_exact_off"]
    dep = np.floor(np.log2(golden["points"])).astype(np.int64)
    total = 0
    for t in range(len(D)):
        slab = p.slab(t)
        want = np.nonzero((dep <= D[t]).all(axis=1))[0]
        assert np.array_equal(np.sort(slab), want)
        total += len(slab)
        exact = set(ex[exo[t]:exo[t + 1]].tolist())
        assert exact == set(np.nonzero((dep == D[t]).all(axis=1))[0].tolist())
    assert total == int(golden["tables_meta_mgrid_size"])


def test_cells_match_reference(golden):
    if "tables_cells" not in golden:
        pytest.skip("no tables in this fixture")
    d = int(golden["d"])
    nc = 1 << d
    p = make_plan(golden)
    ref = golden["tables_cells"].reshape(-1, nc)
    corners_idx = golden["tables_cell_corners"].reshape(-1, nc, d)
    off = golden["tables_cells_off"]
    counts = p.cell_counts()
    for t in range(len(counts)):
        assert counts[t] == off[t + 1] - off[t]
        mine = p.cells(t)
        # reference corner order (CellIndexIterator) -> bit k = right in dim k
        rc = ref[off[t]:off[t + 1]]
        ci = corners_idx[off[t]:off[t + 1]]
        if len(rc) == 0:
            continue
        # right side in dim k <=> larger coordinate than the corner with bit k clear
        coord = np.where(ci == 0, 0.0, np.where(ci == 1, 1.0, 0.0))
        inner = ci >= 2
        lv = np.floor(np.log2(np.maximum(ci, 1)))
        coord = np.where(inner, (2 * (ci - 2 ** lv) + 1) / 2 ** lv, coord)
        lo = coord.min(axis=1, keepdims=True)
        bits = ((coord > lo).astype(np.int64) << np.arange(d)).sum(axis=2)
        reord = np.full_like(rc, -2)
        for c in range(len(rc)):
            reord[c, bits[c]] = rc[c]
        a = sorted(map(tuple, reord.tolist()))
        b = sorted(map(tuple, mine.tolist()))
        assert a == b


def test_neighbors_and_stencils(golden):
    if "tables_nbr1d" not in golden:
        pytest.skip("no tables in this fixture")
    d = int(golden["d"])
    p = make_plan(golden)
    nb = p.neighbors()
    assert np.array_equal(nb.ravel(), golden["tables_nbr1d"].astype(np.int64))
    sj, sw, so = golden["tables_stencil_j"], golden["tables_stencil_w"], golden["tables_stencil_off"]
    for k in range(len(golden["active"])):
        if not golden["active"][k]:
            continue
        idx, w = p.stencil(k)
        assert np.array_equal(idx, sj[so[k]:so[k + 1]])
        assert np.array_equal(w, sw[so[k]:so[k + 1]])  # bit-exact weights


def test_regular_generator_reproduces_storage_order(golden):
    args = str(golden["gridargs"])
    if "refine" in args:
        pytest.skip("adaptive grid")
    level = int(args.split("=")[1])
    g = lsg.AdaptiveSparseGrid.regular(int(golden["d"]), level)
    assert np.array_equal(g.points, golden["points"])


@pytest.mark.parametrize("d,level,n", [(3, 7, 7423), (4, 6, 7937), (6, 5, 10625), (6, 9, 1496065)])
def test_regular_sizes(d, level, n):
    assert lsg.AdaptiveSparseGrid.regular(d, level).n == n


@pytest.mark.parametrize("d,level,refine,n,hanging", [(5, 4, 2, 5768, 5), (6, 5, 2, 40811, 6),
                                                     (6, 7, 3, 499107, 6)])
def test_corner_family_sizes(d, level, refine, n, hanging):
    """The benchmark's grid family, completed with every stage of
    completeDirichletGrid (addPoints2 included at every size)."""
    g = lsg.AdaptiveSparseGrid.adaptive(d, level, refine, 0.6, "corner")
    assert g.n == n and int((g.active == 0).sum()) == hanging


def test_invalid_grids_rejected():
    with pytest.raises(lsg.LsgError):
        lsg.Plan(lsg.AdaptiveSparseGrid(np.array([[0, 2]], np.int32)))  # boundary point
    with pytest.raises(lsg.LsgError):
        lsg.Plan(lsg.AdaptiveSparseGrid(np.array([[2, 2], [2, 2]], np.int32)))  # duplicate


def test_adaptive_generator_reproduces_reference(golden):
    """Refinement + completeDirichletGrid restated in lsg_gridgen.cpp gives the
    reference's grid: same points, same storage order, same hanging nodes."""
    args = str(golden["gridargs"])
    if "refine" not in args:
        pytest.skip("regular grid")
    kv = dict(a.split("=") for a in args.split())
    g = lsg.AdaptiveSparseGrid.adaptive(int(golden["d"]), int(kv["level"]), int(kv["refine"]), float(kv["theta"]),
                                        kv.get("target", "corner"))
    assert np.array_equal(g.points, golden["points"])
    assert np.array_equal(g.active, golden["active"])


@pytest.mark.parametrize("path", __import__("conftest").GOLDEN_BD,
                         ids=lambda p: os.path.basename(p)[:-4])
def test_neumann_generator_reproduces_reference(path):
    """completeNeumannGrid (sgrid/sparseGrid.cc:654-740) restated in
    lsg_gridgen.cpp: the boundary grid of every boundary-data fixture, points
    and storage order equal to the reference's."""
    z = np.load(path)
    kv = dict(a.split("=") for a in str(z["gridargs"]).split())
    g = lsg.AdaptiveSparseGrid.neumann(int(z["d"]), int(kv["level"]), int(kv.get("refine", 0)),
                                       float(kv.get("theta", 0.5)), kv.get("target", "corner"))
    assert np.array_equal(g.points, z["npoints"])
    assert np.array_equal(g.active, z["nactive"])
    assert g.boundary_mask().any() and np.all(g.coordinates()[g.points == 0] == 0.0)
    assert np.all(g.coordinates()[g.points == 1] == 1.0)


@pytest.mark.parametrize("path", __import__("conftest").GOLDEN_COMPLETE,
                         ids=lambda p: os.path.basename(p)[:-4])
def test_completion_of_given_points_matches_reference(path):
    """completeDirichletGrid / completeNeumannGrid of a caller's point set
    (lsg_grid_complete): the reference's points, order and hanging flags.
    cmp_d2_example is the two points of the reference's adaptive-grid example."""
    z = np.load(path)
    g = lsg.AdaptiveSparseGrid(z["in_points"])
    g.completeDirichletGrid()
    assert np.array_equal(g.points, z["points"]) and np.array_equal(g.active, z["active"])
    h = lsg.AdaptiveSparseGrid(z["in_points"])
    h.completeNeumannGrid()
    assert np.array_equal(h.points, z["npoints"]) and np.array_equal(h.active, z["nactive"])


def test_completion_pipeline_equals_generator():
    """Refinement without completion, then lsg_grid_complete, equals the
    generator's refinement with completion (pinned to the reference above)."""
    for d, lv, r, th, tg in [(2, 3, 3, 0.45, "corner"), (3, 2, 3, 0.6, "corner"), (4, 2, 2, 0.3, "plane")]:
        raw = lsg.AdaptiveSparseGrid.adaptive(d, lv, r, th, tg, complete=False)
        raw.completeDirichletGrid()
        ref = lsg.AdaptiveSparseGrid.adaptive(d, lv, r, th, tg)
        assert np.array_equal(raw.points, ref.points) and np.array_equal(raw.active, ref.active)


def test_completion_rejects_bad_input():
    with pytest.raises(lsg.LsgError):
        lsg.AdaptiveSparseGrid(np.array([[2, 4], [2, 4]], np.int32)).completeDirichletGrid()  # duplicate
