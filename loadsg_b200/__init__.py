"""loadsg_b200 -- B200-native prewavelet matvec and CG for LoAdSG grids.

Python mirror of the reference's interface for this path (LoAdSG,
library/source/):

  AdaptiveSparseGrid            sgrid/sparseGrid.h:86-387 (points in storage order)
  MidpointDiffusion             the StencilTemplate::integration plugin
                                (stencils/Stencil.h:740) with the coefficient
                                sampled at cell midpoints
  MatrixVectorHomogen           MatrixVectorMultiplication/MatrixVectorHomogen.h:32-652
    .multiplication(x, Ax, p)   MatrixVectorHomogen.h:91-92
  CG.solveHomogen(...)          applications/cg_method.h:27-33,759-886
  Preconditioning.diagonal      applications/cg_method.h:81-754

All compute runs in liblsg.so (hand-written sm_100a CUDA behind the C-ABI of
include/lsg.h).  There is no CPU fallback: if the library is missing or no GPU
is present, the calls raise.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblsg.so")
_LIB = None

FP64, FP32 = 0, 1
COEF_CONST, COEF_SINPROD, COEF_EXPSIN, COEF_LOGNORMAL, COEF_SIN2PI = range(5)


class LsgError(RuntimeError):
    pass


class _Info(ctypes.Structure):
    _fields_ = [
        ("d", ctypes.c_int32),
        ("n_points", ctypes.c_int64),
        ("n_active", ctypes.c_int64),
        ("n_depths", ctypes.c_int32),
        ("n_slab_entries", ctypes.c_int64),
        ("n_cells", ctypes.c_int64),
        ("case_slab_entries", ctypes.c_int64),
        ("case_cells", ctypes.c_int64),
        ("device_bytes", ctypes.c_int64),
        ("plan_seconds", ctypes.c_double),
        ("matvec_bytes_fp64", ctypes.c_double),
        ("matvec_flops", ctypes.c_double),
    ]


class SolverOpts(ctypes.Structure):
    _fields_ = [
        ("eps", ctypes.c_double),
        ("criterion", ctypes.c_int32),
        ("max_iter", ctypes.c_int32),
        ("precond", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("inner_iter", ctypes.c_int32),
        ("inner_tol", ctypes.c_double),
        ("use_graph", ctypes.c_int32),
    ]


class SolveReport(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int32),
        ("outer_iterations", ctypes.c_int32),
        ("rel_residual", ctypes.c_double),
        ("seconds", ctypes.c_double),
        ("converged", ctypes.c_int32),
        ("fell_back", ctypes.c_int32),
        ("kernel_launches", ctypes.c_int64),
    ]


class Tuning(ctypes.Structure):
    """Launch parameters of the matvec (lsg_tuning in include/lsg.h)."""
    _fields_ = [
        ("cell_threads", ctypes.c_int32),
        ("cell_space_kb", ctypes.c_int32),
        ("class_ratio", ctypes.c_int32),
        ("level_threads", ctypes.c_int32),
        ("level_cap", ctypes.c_int32),
        ("prolong_threads", ctypes.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def lib():
    """Loads liblsg.so (built in-tree by `python -m loadsg_b200.build`)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise LsgError(f"{LIB_PATH} is missing; build it with `python -m loadsg_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        P, I32, I64, D = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
        sig = {
            "lsg_operator_create": (ctypes.c_int, [I32, P, P, I64, P]),
            "lsg_operator_destroy": (None, [P]),
            "lsg_operator_info": (ctypes.c_int, [P, P]),
            "lsg_operator_set_coefficient": (ctypes.c_int, [P, I32, P, I32]),
            "lsg_matvec": (ctypes.c_int, [P, P, P]),
            "lsg_matvec_device": (ctypes.c_int, [P, P, P, I32, P]),
            "lsg_diag": (ctypes.c_int, [P, P]),
            "lsg_matvec_profile": (ctypes.c_int, [P, P, P, I32, I32, P, P, P]),
            "lsg_matvec_device_noalloc": (ctypes.c_int, [P, P, P, I32, P]),
            "lsg_diag_device": (ctypes.c_int, [P, P, P]),
            "lsg_cg_solve": (ctypes.c_int, [P, P, P, P, P]),
            "lsg_cg_solve_device": (ctypes.c_int, [P, P, P, P, P, P]),
            "lsg_set_learned_diag": (ctypes.c_int, [P, P]),
            "lsg_plan_create": (ctypes.c_int, [I32, P, P, I64, P]),
            "lsg_plan_destroy": (None, [P]),
            "lsg_plan_info": (ctypes.c_int, [P, P]),
            "lsg_plan_export_depths": (ctypes.c_int, [P, P]),
            "lsg_plan_export_sorted_depths": (ctypes.c_int, [P, I32, P, P]),
            "lsg_plan_export_cell_counts": (ctypes.c_int, [P, P]),
            "lsg_plan_export_cells": (ctypes.c_int, [P, I32, P, P]),
            "lsg_plan_export_slab": (ctypes.c_int, [P, I32, P, P]),
            "lsg_plan_export_neighbors": (ctypes.c_int, [P, P]),
            "lsg_plan_export_stencil": (ctypes.c_int, [P, I64, P, P, P]),
            "lsg_grid_regular": (ctypes.c_int, [I32, I32, P, I64, P]),
            "lsg_grid_adaptive": (ctypes.c_int, [I32, I32, I32, D, I32, I32, P, P, I64, P]),
            "lsg_operator_set_form": (ctypes.c_int, [P, I32]),
            "lsg_hierarchize_boundary": (ctypes.c_int, [I32, I64, P, P]),
            "lsg_boundary_rhs": (ctypes.c_int, [P, I32, I64, P, P, P]),
            "lsg_boundary_rhs_device": (ctypes.c_int, [P, I32, I64, P, P, P, P]),
            "lsg_grid_complete": (ctypes.c_int, [I32, I64, P, P, I32, P, P, I64, P]),
            "lsg_hierarchize": (ctypes.c_int, [I32, I64, P, P, P]),
            "lsg_dehierarchize": (ctypes.c_int, [I32, I64, P, P, P]),
            "lsg_pde_boundary_rhs": (ctypes.c_int, [P, I32, I64, P, P, P, P, P]),
            "lsg_h1_norm": (ctypes.c_int, [P, P, P]),
            "lsg_l2_norm": (ctypes.c_int, [P, P, P]),
            "lsg_calc_nodal_by_prew": (ctypes.c_int, [P, P, P]),
            "lsg_calc_prew_by_nodal": (ctypes.c_int, [P, P, P]),
            "lsg_calc_nodal_by_prew_device": (ctypes.c_int, [P, P, P, P]),
            "lsg_calc_prew_by_nodal_device": (ctypes.c_int, [P, P, P, P]),
            "lsg_operator_get_tuning": (ctypes.c_int, [P, P]),
            "lsg_operator_set_tuning": (ctypes.c_int, [P, P]),
            "lsg_operator_autotune": (ctypes.c_int, [P, I32, I32, P, P, P]),
            "lsg_batch_autotune": (ctypes.c_int, [P, I32, I32]),
            "lsg_batch_create": (ctypes.c_int, [I32, P, P, P, P, P]),
            "lsg_batch_destroy": (None, [P]),
            "lsg_batch_size": (I64, [P]),
            "lsg_batch_offsets": (ctypes.c_int, [P, P]),
            "lsg_batch_set_coefficient": (ctypes.c_int, [P, I32, I32, P, I32]),
            "lsg_batch_matvec_device": (ctypes.c_int, [P, P, P, I32, P]),
            "lsg_batch_cg_solve_device": (ctypes.c_int, [P, P, P, P, P, P, P]),
            "lsg_batch_cg_solve": (ctypes.c_int, [P, P, P, P, P, P]),
            "lsg_last_error": (ctypes.c_char_p, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if isinstance(a, np.ndarray) else ctypes.c_void_p(a)


def _check(rc):
    if rc != 0:
        raise LsgError(f"liblsg error {rc}: {lib().lsg_last_error().decode()}")


# --------------------------------------------------------------------------- grids
class AdaptiveSparseGrid:
    """Grid points (1D indices, storage order) and active flags.

    Mirrors the parts of the reference's AdaptiveSparseGrid this path reads:
    getIndexOfTable(k) (sgrid/sparseGrid.h:566-572), getActiveTable() and
    getMaximalOccupiedSecondTable()."""

    def __init__(self, points, active=None):
        self.points = np.ascontiguousarray(points, dtype=np.int32)
        if self.points.ndim != 2:
            raise ValueError("points must be N x d")
        self.n, self.d = self.points.shape
        if active is None:
            active = np.ones(self.n, np.uint8)
        self.active = np.ascontiguousarray(active, dtype=np.uint8)

    @classmethod
    def regular(cls, d, level):
        """AddRecursiveSonsOfPoint(center, level) (sgrid/sparseGrid.cc:557-566)."""
        n = ctypes.c_int64(0)
        _check(lib().lsg_grid_regular(d, level, None, 0, ctypes.byref(n)))
        pts = np.zeros((n.value, d), np.int32)
        _check(lib().lsg_grid_regular(d, level, _ptr(pts), n.value, ctypes.byref(n)))
        return cls(pts)

    @classmethod
    def adaptive(cls, d, level, refine, theta, target="corner", complete=True):
        """Regular grid of `level`, `refine` refinement rounds toward the corner
        (max_k x_k < theta 2^(1-r)) or the plane x_0 = 1/2, then the reference's
        completeDirichletGrid (sgrid/sparseGrid.cc:771-787)."""
        t = {"corner": 0, "plane": 1}[target]
        n = ctypes.c_int64(0)
        _check(lib().lsg_grid_adaptive(d, level, refine, theta, t, int(complete), None, None, 0, ctypes.byref(n)))
        pts = np.zeros((n.value, d), np.int32)
        act = np.zeros(n.value, np.uint8)
        _check(lib().lsg_grid_adaptive(d, level, refine, theta, t, int(complete), _ptr(pts), _ptr(act), n.value,
                                       ctypes.byref(n)))
        return cls(pts, act)

    @classmethod
    def neumann(cls, d, level, refine=0, theta=0.5, target="corner"):
        """The grid of `regular` (refine = 0) or `adaptive` with the same
        arguments, then completeNeumannGrid (sgrid/sparseGrid.cc:654-740): its
        boundary points, all active, in the reference's storage order.  This is
        the second grid that boundary data g live on."""
        t = {"corner": 0, "plane": 1}[target]
        mask = (0x3E if refine > 0 else 0) | 64
        n = ctypes.c_int64(0)
        _check(lib().lsg_grid_adaptive(d, level, refine, theta, t, mask, None, None, 0, ctypes.byref(n)))
        pts = np.zeros((n.value, d), np.int32)
        act = np.zeros(n.value, np.uint8)
        _check(lib().lsg_grid_adaptive(d, level, refine, theta, t, mask, _ptr(pts), _ptr(act), n.value,
                                       ctypes.byref(n)))
        return cls(pts, act)

    def _complete(self, mask):
        n = ctypes.c_int64(0)
        _check(lib().lsg_grid_complete(self.d, self.n, _ptr(self.points), _ptr(self.active), mask, None, None, 0,
                                       ctypes.byref(n)))
        pts = np.zeros((n.value, self.d), np.int32)
        act = np.zeros(n.value, np.uint8)
        _check(lib().lsg_grid_complete(self.d, self.n, _ptr(self.points), _ptr(self.active), mask, _ptr(pts),
                                       _ptr(act), n.value, ctypes.byref(n)))
        self.points, self.active, self.n = pts, act, n.value

    def completeDirichletGrid(self):
        """AdaptiveSparseGrid::completeDirichletGrid (sgrid/sparseGrid.cc:771-787),
        in place: the missing interior points and the hanging nodes of this
        point set, added in the reference's order."""
        self._complete(1)

    def completeNeumannGrid(self):
        """AdaptiveSparseGrid::completeNeumannGrid (sgrid/sparseGrid.cc:654-740),
        in place: neighbours and boundary points of the active points."""
        self._complete(64)

    def boundary_mask(self):
        """Points with a 1D index 0 or 1 (coordinate 0 or 1) in some dimension."""
        return (self.points < 2).any(axis=1)

    def getMaximalOccupiedSecondTable(self):
        return self.n

    def getDOFS(self):
        return int(self.active.sum())

    def coordinates(self):
        """Coordinates of all points (IndexOneD::coordinate, indices/index.h:718-730)."""
        idx = self.points.astype(np.int64)
        t = np.floor(np.log2(np.maximum(idx, 2))).astype(np.int64)
        x = (2 * (idx - (1 << t)) + 1) / (2.0 ** t)
        return np.where(idx < 2, idx.astype(np.float64), x)  # boundary indices 0, 1 sit at 0, 1


FORM_STIFFNESS, FORM_MASS = 0, 1


class MidpointDiffusion:
    """-div(a grad u) with a sampled at cell midpoints: the local stiffness
    entry of a cell is a(x_c) times the exact Q1 entry (the value a
    StencilTemplate::integration plugin returns, stencils/Stencil.h:740)."""

    form = FORM_STIFFNESS

    def __init__(self, family, params):
        self.family = int(family)
        self.params = np.zeros(256, np.float64)
        p = np.asarray(params, np.float64).ravel()
        self.params[: len(p)] = p
        self.nparams = len(p)


class MidpointMass(MidpointDiffusion):
    """a(x) u v with a sampled at cell midpoints: a(x_c) times the exact Q1 mass
    entry.  For a = 1 this is the reference's HelmHoltz operator
    (stencils/Stencil.h:873-919): right-hand sides <f, psi_i> from nodal values
    of f, and L2 norms u^T M u of prewavelet expansions."""

    form = FORM_MASS


class Plan:
    """Host-only flattened tables (no GPU needed); for parity tests."""

    def __init__(self, grid):
        self.grid = grid
        h = ctypes.c_void_p()
        _check(lib().lsg_plan_create(grid.d, _ptr(grid.points), _ptr(grid.active), grid.n, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.lsg_plan_destroy(self._h)
            self._h = None

    def info(self):
        i = _Info()
        _check(lib().lsg_plan_info(self._h, ctypes.byref(i)))
        return {k: getattr(i, k) for k, _ in _Info._fields_}

    def depths(self):
        nd = self.info()["n_depths"]
        out = np.zeros((nd, self.grid.d), np.int32)
        _check(lib().lsg_plan_export_depths(self._h, _ptr(out)))
        return out

    def sorted_depths(self, case):
        nd = self.info()["n_depths"]
        out = np.zeros(nd, np.int32)
        cnt = ctypes.c_int32(0)
        _check(lib().lsg_plan_export_sorted_depths(self._h, case, _ptr(out), ctypes.byref(cnt)))
        return out[: cnt.value]

    def cell_counts(self):
        out = np.zeros(self.info()["n_depths"], np.int64)
        _check(lib().lsg_plan_export_cell_counts(self._h, _ptr(out)))
        return out

    def cells(self, t):
        cnt = ctypes.c_int64(0)
        _check(lib().lsg_plan_export_cells(self._h, t, None, ctypes.byref(cnt)))
        out = np.zeros((cnt.value, 1 << self.grid.d), np.int64)
        _check(lib().lsg_plan_export_cells(self._h, t, _ptr(out), ctypes.byref(cnt)))
        return out

    def slab(self, t):
        cnt = ctypes.c_int64(0)
        _check(lib().lsg_plan_export_slab(self._h, t, None, ctypes.byref(cnt)))
        out = np.zeros(cnt.value, np.int64)
        _check(lib().lsg_plan_export_slab(self._h, t, _ptr(out), ctypes.byref(cnt)))
        return out

    def neighbors(self):
        out = np.zeros((self.grid.n, self.grid.d, 2), np.int64)
        _check(lib().lsg_plan_export_neighbors(self._h, _ptr(out)))
        return out

    def stencil(self, k):
        m = 5 ** self.grid.d
        idx = np.zeros(m, np.int64)
        w = np.zeros(m, np.float64)
        cnt = ctypes.c_int32(0)
        _check(lib().lsg_plan_export_stencil(self._h, k, _ptr(idx), _ptr(w), ctypes.byref(cnt)))
        return idx[: cnt.value], w[: cnt.value]


# --------------------------------------------------------------------------- operator
class MatrixVectorHomogen:
    """Prewavelet stiffness operator on one grid, resident on the current GPU
    (MatrixVectorHomogen(grid, mgrid, symmetry, mpi_on), MatrixVectorHomogen.h:72-77)."""

    def __init__(self, grid, problem=None):
        self.grid = grid
        h = ctypes.c_void_p()
        _check(lib().lsg_operator_create(grid.d, _ptr(grid.points), _ptr(grid.active), grid.n, ctypes.byref(h)))
        self._h = h
        self._problem = None
        if problem is not None:
            self.set_problem(problem)

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.lsg_operator_destroy(self._h)
            self._h = None

    def set_problem(self, problem):
        if problem is not self._problem:
            _check(lib().lsg_operator_set_coefficient(self._h, problem.family, _ptr(problem.params), problem.nparams))
            _check(lib().lsg_operator_set_form(self._h, problem.form))
            self._problem = problem

    def info(self):
        i = _Info()
        _check(lib().lsg_operator_info(self._h, ctypes.byref(i)))
        return {k: getattr(i, k) for k, _ in _Info._fields_}

    def multiplication(self, prew, Ax, problem):
        """Ax[active] = A_prew prew (host arrays of length N, storage order)."""
        self.set_problem(problem)
        x = np.ascontiguousarray(prew, np.float64)
        if Ax.dtype != np.float64 or not Ax.flags.c_contiguous:
            raise ValueError("Ax must be a contiguous float64 array")
        _check(lib().lsg_matvec(self._h, _ptr(x), _ptr(Ax)))
        return Ax

    def multiplication_device(self, x_ptr, y_ptr, precision=FP64, stream=0):
        """Device-pointer variant (torch tensors: pass t.data_ptr())."""
        _check(lib().lsg_matvec_device(self._h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr), precision,
                                       ctypes.c_void_p(stream)))

    def tuning(self):
        t = Tuning()
        _check(lib().lsg_operator_get_tuning(self._h, ctypes.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        t = Tuning()
        _check(lib().lsg_operator_get_tuning(self._h, ctypes.byref(t)))
        for k, v in kw.items():
            setattr(t, k, int(v))
        _check(lib().lsg_operator_set_tuning(self._h, ctypes.byref(t)))

    def autotune(self, precision=FP32, reps=3, cache=None):
        """Picks the matvec launch parameters by timing (lsg_operator_autotune).
        With cache (a JSON path, or True for $LSG_TUNING_CACHE or
        ~/.cache/loadsg_b200/tuning.json) settings are reused for operators of
        the same dimension, size class and precision.  Returns (setting,
        best ms, ms with the previous setting); ms are None on a cache hit."""
        from . import tuning as _tuning
        return _tuning.autotune(self, precision, reps, cache)

    def profile(self, x_ptr, y_ptr, precision=FP32, iters=5):
        """Mean ms per matvec phase (nodal, P init, prolongation, cell operator,
        restriction wavefronts with the final gather, total) plus algorithmic
        bytes per phase and cell-operator flops."""
        ms = np.zeros(6)
        by = np.zeros(6)
        fl = np.zeros(1)
        _check(lib().lsg_matvec_profile(self._h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr), precision, iters,
                                        _ptr(ms), _ptr(by), _ptr(fl)))
        return ms, by, float(fl[0])

    def diagonal(self, problem):
        """Exact Jacobi diagonal (Preconditioning::precondLocalStiffnessMatrix)."""
        self.set_problem(problem)
        out = np.zeros(self.grid.n)
        _check(lib().lsg_diag(self._h, _ptr(out)))
        return out

    def set_learned_diagonal(self, diag):
        diag = np.ascontiguousarray(diag, np.float64)
        _check(lib().lsg_set_learned_diag(self._h, _ptr(diag)))


class CG:
    @staticmethod
    def solveHomogen(eps, x, f, matrix, problem, criterion=0, max_iter=500, precond=0, precision=FP64,
                     inner_iter=1000, inner_tol=1e-5, use_graph=True):
        """CG::solveHomogen (applications/cg_method.h:759-886).  x (in/out) and f
        are host float64 arrays.  criterion 0 is the reference's stopping rule on
        r^T D^-1 r; criterion 1 stops at ||f - A x|| / ||f|| <= eps.  Returns the
        report (iterations, rel_residual, seconds, ...)."""
        matrix.set_problem(problem)
        o = SolverOpts(eps, criterion, max_iter, precond, precision, inner_iter, inner_tol, int(use_graph))
        rep = SolveReport()
        if x.dtype != np.float64 or not x.flags.c_contiguous:
            raise ValueError("x must be a contiguous float64 array")
        f = np.ascontiguousarray(f, np.float64)
        _check(lib().lsg_cg_solve(matrix._h, _ptr(f), _ptr(x), ctypes.byref(o), ctypes.byref(rep)))
        return {k: getattr(rep, k) for k, _ in SolveReport._fields_}

    @staticmethod
    def solve_device(matrix, f_ptr, x_ptr, opts, stream=0):
        rep = SolveReport()
        _check(lib().lsg_cg_solve_device(matrix._h, ctypes.c_void_p(f_ptr), ctypes.c_void_p(x_ptr),
                                         ctypes.byref(opts), ctypes.byref(rep), ctypes.c_void_p(stream)))
        return {k: getattr(rep, k) for k, _ in SolveReport._fields_}


# --------------------------------------------------------------------------- basis transforms
def calcNodalByPrew(prew, u, matrix):
    """calcNodalByPrew(prew, u) (BasisTransformations/BasisTransformations.cpp:670-706):
    u = values at every grid point of the prewavelet expansion prew (0 at
    hanging points).  Host float64 arrays of length N; the grid comes from the
    MatrixVectorHomogen (no coefficient needed)."""
    prew = np.ascontiguousarray(prew, np.float64)
    if u.dtype != np.float64 or not u.flags.c_contiguous:
        raise ValueError("u must be a contiguous float64 array")
    _check(lib().lsg_calc_nodal_by_prew(matrix._h, _ptr(prew), _ptr(u)))


def calcPrewByNodal(prew, u, matrix):
    """calcPrewByNodal(prew, u) (BasisTransformations.cpp:486-545): prew = the
    prewavelet coefficients whose expansion takes the values u at the active
    points (0 at hanging points); u is not modified."""
    u = np.ascontiguousarray(u, np.float64)
    if prew.dtype != np.float64 or not prew.flags.c_contiguous:
        raise ValueError("prew must be a contiguous float64 array")
    _check(lib().lsg_calc_prew_by_nodal(matrix._h, _ptr(prew), _ptr(u)))


def calcNodalByPrew_device(prew_ptr, u_ptr, matrix, stream=0):
    _check(lib().lsg_calc_nodal_by_prew_device(matrix._h, ctypes.c_void_p(prew_ptr), ctypes.c_void_p(u_ptr),
                                               ctypes.c_void_p(stream)))


def calcPrewByNodal_device(prew_ptr, u_ptr, matrix, stream=0):
    _check(lib().lsg_calc_prew_by_nodal_device(matrix._h, ctypes.c_void_p(prew_ptr), ctypes.c_void_p(u_ptr),
                                               ctypes.c_void_p(stream)))


# --------------------------------------------------------------------------- boundary data
BDRHS_GRADIENT, BDRHS_MASS, BDRHS_MASS_COEFF = 0, 1, 2


def CalcHierarchicalBasisForRHS(u, grid):
    """CalcHierarchicalBasisForRHS(u) (MatrixVectorMultiplication/RHS.cpp:6-41),
    in place on the host array u of the grid with boundary points `grid`: the
    boundary values become hierarchical coefficients (interior entries are left
    alone).  The reference's vector carries its grid; here it is passed."""
    if u.dtype != np.float64 or not u.flags.c_contiguous or u.shape != (grid.n,):
        raise ValueError("u must be a contiguous float64 array of the grid's length")
    _check(lib().lsg_hierarchize_boundary(grid.d, grid.n, _ptr(grid.points), _ptr(u)))


class InHomoBoundaryRHSHierarchical:
    """InHomoBoundaryRHSHierarchical (MatrixVectorMultiplication/RHS.h:278-427):
    products of the prewavelets of `matrix`'s grid with boundary data given by
    hierarchical coefficients on `boundary_grid` (a grid with boundary points,
    e.g. AdaptiveSparseGrid.neumann).  The reference constructs it from the
    interior grid and reads the boundary grid from the coefficient vector."""

    def __init__(self, matrix, boundary_grid):
        self.matrix = matrix
        self.boundary_grid = boundary_grid

    def _run(self, kind, hierarchical, dirichlet):
        bg = self.boundary_grid
        h = np.ascontiguousarray(hierarchical, np.float64)
        if h.shape != (bg.n,):
            raise ValueError("hierarchical must have one value per boundary-grid point")
        if dirichlet.dtype != np.float64 or not dirichlet.flags.c_contiguous or dirichlet.shape != (self.matrix.grid.n,):
            raise ValueError("dirichlet must be a contiguous float64 array of the grid's length")
        _check(lib().lsg_boundary_rhs(self.matrix._h, kind, bg.n, _ptr(bg.points), _ptr(h), _ptr(dirichlet)))

    def multiply(self, hierarchical, dirichlet):
        """RHS.cpp:697-774: dirichlet[active] = integral grad psi_i . grad g."""
        self._run(BDRHS_GRADIENT, hierarchical, dirichlet)

    def multiply_mass(self, hierarchical, dirichlet):
        """RHS.cpp:776-852: dirichlet[active] = integral psi_i g."""
        self._run(BDRHS_MASS, hierarchical, dirichlet)

    def multiply_mass_coeff(self, hierarchical, dirichlet):
        """RHS.cpp:854-1008: dirichlet[active] = integral psi_i g prod_k (1 - x_k^2)."""
        self._run(BDRHS_MASS_COEFF, hierarchical, dirichlet)

    def multiply_device(self, kind, hier_ptr, dirichlet_ptr, stream=0):
        """Device form: hier (boundary-grid length) and dirichlet in device memory."""
        bg = self.boundary_grid
        _check(lib().lsg_boundary_rhs_device(self.matrix._h, kind, bg.n, _ptr(bg.points), ctypes.c_void_p(hier_ptr),
                                             ctypes.c_void_p(dirichlet_ptr), ctypes.c_void_p(stream)))


def _grid_vector(u, grid):
    if u.dtype != np.float64 or not u.flags.c_contiguous or u.shape != (grid.n,):
        raise ValueError("u must be a contiguous float64 array of the grid's length")


def CalcHierarchicalBasis(u, grid):
    """CalcHierarchicalBasis(u) (BasisTransformations/BasisTransformations.cpp:390-409)
    in place on the host array u of `grid` (boundary points allowed): nodal
    values to hierarchical coefficients at the active points."""
    _grid_vector(u, grid)
    _check(lib().lsg_hierarchize(grid.d, grid.n, _ptr(grid.points), _ptr(grid.active), _ptr(u)))


def CalcNodalBasis(u, grid):
    """CalcNodalBasis(u) (BasisTransformations.cpp:174-198): the inverse of
    CalcHierarchicalBasis, in place."""
    _grid_vector(u, grid)
    _check(lib().lsg_dehierarchize(grid.d, grid.n, _ptr(grid.points), _ptr(grid.active), _ptr(u)))


PDE_POISSON, PDE_HELMHOLTZ = 0, 1


class PDE_Poisson_InHomRHS:
    """PDE_Poisson_InHomRHS (applications/PDE.h:16-31, PDE.cpp:9-52): the
    right-hand side on the interior grid of -lap u = f with u = g on the
    boundary, reduced to zero boundary values.  neumann_grid holds boundary
    points (AdaptiveSparseGrid.neumann), dirichlet_grid is the grid of
    `matrix`.  SetUp(f_neumann, g_neumann) takes f at every point and g at the
    boundary points of neumann_grid (host arrays, transformed in place as in
    the reference); getRHS() returns the right-hand side (0 at hanging points)."""

    kind = PDE_POISSON

    def __init__(self, neumann_grid, dirichlet_grid, matrix):
        if dirichlet_grid.n != matrix.grid.n or dirichlet_grid.d != neumann_grid.d:
            raise ValueError("dirichlet_grid must be the grid of matrix, of the same dimension as neumann_grid")
        self.neumann_grid, self.dirichlet_grid, self.matrix = neumann_grid, dirichlet_grid, matrix
        self.f_dirichlet = np.zeros(dirichlet_grid.n)

    def SetUp(self, f_neumann, g_neumann):
        ng = self.neumann_grid
        _grid_vector(f_neumann, ng)
        _grid_vector(g_neumann, ng)
        _check(lib().lsg_pde_boundary_rhs(self.matrix._h, self.kind, ng.n, _ptr(ng.points), _ptr(ng.active),
                                          _ptr(f_neumann), _ptr(g_neumann), _ptr(self.f_dirichlet)))

    def getRHS(self):
        return self.f_dirichlet


class PDE_Helmholtz_VariableCoeff(PDE_Poisson_InHomRHS):
    """PDE_Helmholtz_VariableCoeff (applications/PDE.h:47-120): -lap u + c u = f
    with c(x) = prod_k (1 - x_k^2) and u = g on the boundary."""

    kind = PDE_HELMHOLTZ


class H1:
    """H1::getValue (applications/H1_Norm.cpp): the H1 seminorm of the function
    with nodal values u.  The reference takes (grid, mgrid); here the
    MatrixVectorHomogen of the grid (any coefficient: the norm uses a = 1)."""

    def __init__(self, matrix):
        self.matrix = matrix

    def getValue(self, u):
        u = np.ascontiguousarray(u, np.float64)
        out = np.zeros(1)
        _check(lib().lsg_h1_norm(self.matrix._h, _ptr(u), _ptr(out)))
        return float(out[0])


class L2(H1):
    """L2::getValue (applications/H1_Norm.cpp): the L2 norm of the function with
    nodal values u (mass form, the reference's HelmHoltz with a = 1)."""

    def getValue(self, u):
        u = np.ascontiguousarray(u, np.float64)
        out = np.zeros(1)
        _check(lib().lsg_l2_norm(self.matrix._h, _ptr(u), _ptr(out)))
        return float(out[0])


# --------------------------------------------------------------------------- batches
def _report(rep):
    return {k: getattr(rep, k) for k, _ in SolveReport._fields_}


class Batch:
    """Many grids (any mix of dimensions and sizes), each with its own
    coefficient, applied and solved together (lsg_batch_* in include/lsg.h).
    Batch vectors hold the grids' vectors side by side: grid i is
    ``v[offsets[i]:offsets[i+1]]`` in its own storage order."""

    def __init__(self, grids, problems=None):
        self.grids = list(grids)
        k = len(self.grids)
        dims = np.array([g.d for g in self.grids], np.int32)
        pts = (ctypes.c_void_p * k)(*[g.points.ctypes.data for g in self.grids])
        act = (ctypes.c_void_p * k)(*[g.active.ctypes.data for g in self.grids])
        ns = np.array([g.n for g in self.grids], np.int64)
        h = ctypes.c_void_p()
        _check(lib().lsg_batch_create(k, _ptr(dims), pts, act, _ptr(ns), ctypes.byref(h)))
        self._h = h
        self._destroy = lib().lsg_batch_destroy
        off = np.zeros(k + 1, np.int64)
        _check(lib().lsg_batch_offsets(self._h, _ptr(off)))
        self.offsets = off[:-1]
        self.size = int(off[-1])
        if problems is not None:
            for i, p in enumerate(problems):
                self.set_problem(i, p)

    def __del__(self):
        if getattr(self, "_h", None):
            self._destroy(self._h)
            self._h = None

    def autotune(self, precision=FP32, reps=3):
        _check(lib().lsg_batch_autotune(self._h, precision, reps))

    def set_problem(self, i, problem):
        _check(lib().lsg_batch_set_coefficient(self._h, i, problem.family, _ptr(problem.params), problem.nparams))

    def gather(self, parts):
        """Batch vector from per-grid host arrays."""
        v = np.zeros(self.size)
        for i, a in enumerate(parts):
            v[self.offsets[i]:self.offsets[i] + self.grids[i].n] = a
        return v

    def split(self, v):
        return [v[self.offsets[i]:self.offsets[i] + self.grids[i].n] for i in range(len(self.grids))]

    def matvec_device(self, x_ptr, y_ptr, precision=FP64, stream=0):
        _check(lib().lsg_batch_matvec_device(self._h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr), precision,
                                             ctypes.c_void_p(stream)))

    def solve(self, eps, x, f, criterion=1, max_iter=500, precond=0, precision=FP64, inner_iter=1000,
              inner_tol=1e-5, use_graph=True):
        """CG of every grid; x (in/out) and f are host batch vectors.  Returns
        (per-grid reports, batch report)."""
        if x.dtype != np.float64 or not x.flags.c_contiguous:
            raise ValueError("x must be a contiguous float64 array")
        f = np.ascontiguousarray(f, np.float64)
        o = SolverOpts(eps, criterion, max_iter, precond, precision, inner_iter, inner_tol, int(use_graph))
        reps = (SolveReport * len(self.grids))()
        tot = SolveReport()
        _check(lib().lsg_batch_cg_solve(self._h, _ptr(f), _ptr(x), ctypes.byref(o), reps, ctypes.byref(tot)))
        return [_report(r) for r in reps], _report(tot)

    def solve_device(self, f_ptr, x_ptr, opts, stream=0):
        reps = (SolveReport * len(self.grids))()
        tot = SolveReport()
        _check(lib().lsg_batch_cg_solve_device(self._h, ctypes.c_void_p(f_ptr), ctypes.c_void_p(x_ptr),
                                               ctypes.byref(opts), reps, ctypes.byref(tot), ctypes.c_void_p(stream)))
        return [_report(r) for r in reps], _report(tot)
