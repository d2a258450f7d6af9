"""CPU oracle (test infrastructure only).

Python binding of oracle/liblsg_oracle.so, the C restatement of LoAdSG's
prewavelet matvec, Jacobi diagonal and CG.  Only tests/, the smoke check in
__graft_entry__.py and bench.py's CPU-baseline legs import this package; the
product path (loadsg_b200) never does.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE, "oracle"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liblsg_oracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        L.lsgo_grid_create.restype = P
        L.lsgo_grid_create.argtypes = [ctypes.c_int, P, P, ctypes.c_int64]
        L.lsgo_grid_free.argtypes = [P]
        L.lsgo_num_depths.argtypes = [P]
        L.lsgo_depths.argtypes = [P, P]
        L.lsgo_sorted_depths.argtypes = [P, ctypes.c_int, P]
        L.lsgo_num_cells.restype = ctypes.c_int64
        L.lsgo_num_cells.argtypes = [P, P]
        L.lsgo_lookup.restype = ctypes.c_int64
        L.lsgo_lookup.argtypes = [P, P]
        L.lsgo_matvec.argtypes = [P, ctypes.c_int, P, P, P]
        L.lsgo_diag.argtypes = [P, ctypes.c_int, P, P]
        L.lsgo_cg.argtypes = [P, ctypes.c_int, P, P, P, ctypes.c_double, ctypes.c_int, P]
        L.lsgo_nodal_by_prew.argtypes = [P, P, P]
        L.lsgo_set_form.argtypes = [P, ctypes.c_int]
        L.lsgo_hierarchize_boundary.argtypes = [P, P]
        L.lsgo_boundary_rhs.argtypes = [P, P, ctypes.c_int, P, P]
        L.lsgo_hierarchize.argtypes = [P, P, ctypes.c_int]
        _LIB = L
    return _LIB


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class OracleGrid:
    """A grid given by its points (N x d 1D indices, storage order) and active flags."""

    def __init__(self, points, active):
        self.points = np.ascontiguousarray(points, dtype=np.int32)
        self.active = np.ascontiguousarray(active, dtype=np.uint8)
        self.n, self.d = self.points.shape
        self._h = lib().lsgo_grid_create(self.d, _ptr(self.points), _ptr(self.active), self.n)
        if not self._h:
            raise ValueError("invalid grid")

    def __del__(self):
        if getattr(self, "_h", None):
            lib().lsgo_grid_free(self._h)
            self._h = None

    def depths(self):
        nd = lib().lsgo_num_depths(self._h)
        out = np.zeros((nd, self.d), np.int32)
        lib().lsgo_depths(self._h, _ptr(out))
        return out

    def sorted_depths(self, case):
        nd = lib().lsgo_num_depths(self._h)
        out = np.zeros((nd, self.d), np.int32)
        k = lib().lsgo_sorted_depths(self._h, case, _ptr(out))
        return out[:k]

    def num_cells(self, T):
        T = np.ascontiguousarray(T, np.int32)
        return lib().lsgo_num_cells(self._h, _ptr(T))

    def lookup(self, idx):
        idx = np.ascontiguousarray(idx, np.int32)
        return lib().lsgo_lookup(self._h, _ptr(idx))

    @staticmethod
    def _params(params):
        p = np.zeros(256, np.float64)
        params = np.asarray(params, np.float64)
        p[: len(params)] = params
        return p

    def matvec(self, family, params, x, y=None, form=0):
        """form 0: diffusion (stiffness), 1: mass (the reference's HelmHoltz local matrix)."""
        lib().lsgo_set_form(self._h, form)
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.n) if y is None else np.array(y, np.float64)
        p = self._params(params)
        if lib().lsgo_matvec(self._h, family, _ptr(p), _ptr(x), _ptr(y)) != 0:
            raise MemoryError("oracle matvec failed")
        return y

    def diag(self, family, params, form=0):
        lib().lsgo_set_form(self._h, form)
        out = np.zeros(self.n)
        p = self._params(params)
        lib().lsgo_diag(self._h, family, _ptr(p), _ptr(out))
        return out

    def nodal_by_prew(self, prew):
        """calcNodalByPrew (BasisTransformations.cpp:670-706), restated in C."""
        prew = np.ascontiguousarray(prew, np.float64)
        u = np.zeros(self.n)
        if lib().lsgo_nodal_by_prew(self._h, _ptr(prew), _ptr(u)) != 0:
            raise MemoryError("oracle transform failed")
        return u

    def prew_by_nodal(self, u):
        """calcPrewByNodal (BasisTransformations.cpp:486-545) as the exact inverse
        of nodal_by_prew on the active points: p_A = A_AA^-1 u_A, 0 at hanging
        points, with A assembled column by column (small grids only).  The
        compiled reference agrees with this to ~1e-15 on the golden grids."""
        act = np.nonzero(self.active)[0]
        A = np.zeros((self.n, len(act)))
        e = np.zeros(self.n)
        for c, j in enumerate(act):
            e[j] = 1.0
            A[:, c] = self.nodal_by_prew(e)
            e[j] = 0.0
        p = np.zeros(self.n)
        p[act] = np.linalg.solve(A[act], np.asarray(u, np.float64)[act])
        return p

    def norm(self, u, h1=True):
        """H1::getValue / L2::getValue (applications/H1_Norm.cpp): v = the exact
        inverse of calcNodalByPrew applied to u, sqrt(v . A v) over active points
        with the coefficient-1 stiffness (H1) or mass (L2) matrix; small grids."""
        v = self.prew_by_nodal(u)
        Av = self.matvec(0, [1.0], v, form=0 if h1 else 1)
        act = np.asarray(self.active) > 0
        return float(np.sqrt(np.sum(v[act] * Av[act])))

    def hierarchize_boundary(self, u):
        """CalcHierarchicalBasisForRHS (MatrixVectorMultiplication/RHS.cpp:6-41)
        on a grid with boundary points: returns the transformed copy of u."""
        u = np.array(u, np.float64)
        if lib().lsgo_hierarchize_boundary(self._h, _ptr(u)) != 0:
            raise ValueError("a boundary point lacks a 1D parent")
        return u

    def boundary_rhs(self, ngrid, kind, hier, y=None):
        """InHomoBoundaryRHSHierarchical (RHS.cpp:697-1008) onto this grid from
        the hierarchical boundary coefficients hier of ngrid (a grid with
        boundary points): kind 0 multiply (gradients), 1 multiply_mass, 2
        multiply_mass_coeff (weight prod (1 - x_k^2)).  Active entries of y are
        written, the others keep their values (0 for a fresh y)."""
        hier = np.ascontiguousarray(hier, np.float64)
        y = np.zeros(self.n) if y is None else np.array(y, np.float64)
        if lib().lsgo_boundary_rhs(self._h, ngrid._h, kind, _ptr(hier), _ptr(y)) != 0:
            raise ValueError("oracle boundary right-hand side failed")
        return y

    def hierarchize(self, u):
        """CalcHierarchicalBasis(u) (BasisTransformations.cpp:390-409): a copy."""
        u = np.array(u, np.float64)
        lib().lsgo_hierarchize(self._h, _ptr(u), -1)
        return u

    def dehierarchize(self, u):
        """CalcNodalBasis(u) (BasisTransformations.cpp:174-198): a copy."""
        u = np.array(u, np.float64)
        lib().lsgo_hierarchize(self._h, _ptr(u), +1)
        return u

    def pde_rhs(self, ngrid, f, g, helmholtz=False):
        """PDE_Poisson_InHomRHS::SetUp (applications/PDE.cpp:9-52), or with
        helmholtz PDE_Helmholtz_VariableCoeff::SetUp (PDE.h:62-114): the
        right-hand side on this grid of -lap u (+ c u) = f, u = g on the
        boundary, for f on every point of ngrid (a grid with boundary points)
        and g on its boundary points.  Composed from the restated pieces;
        the inverse transform is the dense one of prew_by_nodal (small grids)."""
        fh = ngrid.hierarchize(f)
        interior = (ngrid.points >= 2).all(axis=1) & (ngrid.active > 0)
        fd = np.zeros(self.n)
        for k in np.nonzero(interior)[0]:
            j = self.lookup(ngrid.points[k])
            if j >= 0:
                fd[j] = fh[k]
        fh[interior] = 0.0
        fd = self.dehierarchize(fd)
        prew = self.prew_by_nodal(fd)
        rhs = self.matvec(0, [1.0], prew, form=1)  # HelmHoltz (Stencil.h:873-919)
        act = self.active > 0
        rhs[act] = rhs[act] + self.boundary_rhs(ngrid, 1, fh)[act]
        gh = ngrid.hierarchize_boundary(g)
        rhs[act] = rhs[act] - self.boundary_rhs(ngrid, 0, gh)[act]
        if helmholtz:
            rhs[act] = rhs[act] - self.boundary_rhs(ngrid, 2, gh)[act]
        return rhs

    def cg(self, family, params, f, eps, maxit=500, x0=None):
        lib().lsgo_set_form(self._h, 0)
        f = np.ascontiguousarray(f, np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, np.float64)
        p = self._params(params)
        it = np.zeros(1, np.int32)
        lib().lsgo_cg(self._h, family, _ptr(p), _ptr(f), _ptr(x), eps, maxit, _ptr(it))
        return x, int(it[0])
