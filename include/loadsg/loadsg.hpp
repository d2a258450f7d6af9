// loadsg.hpp -- header-only C++ drop-in for LoAdSG's prewavelet matvec / CG path,
// built on the C-ABI of lsg.h (liblsg.so).  Class and method names follow the
// reference (paths relative to LoAdSG's library/source/):
//
//   AdaptiveSparseGrid            sgrid/sparseGrid.h:86-387
//     AddRecursiveSonsOfPoint     sgrid/sparseGrid.cc:557-566 (center point, level)
//     AddPoint / getIndexOfTable / getActiveTable / getMaximalOccupiedSecondTable
//   VectorSparseG                 extemp/vector.h:247-441 (double per storage index)
//   StencilTemplate plugin        stencils/Stencil.h:740 -> MidpointDiffusion (family + params)
//   MatrixVectorHomogen           MatrixVectorMultiplication/MatrixVectorHomogen.h:32-652
//     multiplication(prew, Ax, problem)   MatrixVectorHomogen.h:91-92
//   CG::solveHomogen              applications/cg_method.h:27-33
//
//   MultiLevelAdaptiveSparseGrid  sgrid/multilevelSparseGrid.h:13-143 (a handle: the
//                                 multilevel store lives in the operator's slabs)
//   calcPrewByNodal / calcNodalByPrew (prew, u)   BasisTransformations/BasisTransformations.h:117,123
//
// The reference's own signatures are all here: MatrixVectorHomogen(grid,
// mgrid, symmetry, mpi_on) (MatrixVectorHomogen.h:72-77), CG::solveHomogen(eps,
// x, f, &iterations, usol, matrix, stencil, &time) (cg_method.h:27-33), the
// two-argument transforms (the operator is found through the vector's grid),
// and L2 / H1 built from (grid, mgrid).  include/loadsg/compat/source/
// sparseEXPDE.h maps the reference's non-template names (dimension from the
// DimensionSparseGrid macro, IndexDimension, vector expressions) onto these, so
// a reference main compiles with the compat directory on the include path.
//
// Differences a caller must know: the grid is frozen when the first operator
// is built from it (the tables are flattened once); errors throw lsg::Error
// instead of exit(1); the MPI flag of MatrixVectorHomogen must be false (one
// GPU, no MPI) and the symmetry flag is accepted as given (the operator is
// symmetric either way).
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../lsg.h"

namespace lsg {

struct Error : std::runtime_error {
    explicit Error(const std::string& m) : std::runtime_error(m) {}
};

inline void check(int rc) {
    if (rc != LSG_OK) throw Error(std::string("liblsg: ") + lsg_last_error());
}

template <int D>
class MatrixVectorHomogen;

template <int D>
class AdaptiveSparseGrid {
public:
    using Index = std::array<int32_t, D>;
    // the reference's switch between all and only active points in its vector
    // loops (sgrid/sparseGrid.h:186); vector operations here always cover all
    // entries, as the reference's expression templates do with the switch off
    bool WorkOnHangingNodes = false;
    // AddRecursiveSonsOfPoint(center, level) with the center point given as
    // indices (the reference's IndexDimension()): every index must be 2.
    void AddRecursiveSonsOfPoint(const Index& center, int level) {
        for (int d = 0; d < D; ++d)
            if (center[d] != 2) throw Error("AddRecursiveSonsOfPoint: only the center point is supported");
        AddRecursiveSonsOfPoint(level);
    }
    // The operator the two-argument transforms and the (grid, mgrid) norms use:
    // the last MatrixVectorHomogen built on this grid, else one made on first use.
    MatrixVectorHomogen<D>& op() const;
    void attach(MatrixVectorHomogen<D>* m) const { attached_ = m; }
    void detach(MatrixVectorHomogen<D>* m) const {
        if (attached_ == m) attached_ = nullptr;
    }
    // AddPoint (sgrid/sparseGrid.cc:482-516): appends in storage order, returns
    // false if the point is already present (it is then marked active).
    bool AddPoint(const Index& I, bool active = true) {
        auto it = where_.find(I);
        if (it != where_.end()) {
            if (active) active_[it->second] = 1;
            return false;
        }
        where_[I] = (int64_t)active_.size();
        points_.insert(points_.end(), I.begin(), I.end());
        active_.push_back(active ? 1 : 0);
        return true;
    }
    // AddRecursiveSonsOfPoint(center, level) for a regular sparse grid, in the
    // reference's storage order.
    void AddRecursiveSonsOfPoint(int level) {
        int64_t n = 0;
        check(lsg_grid_regular(D, level, nullptr, 0, &n));
        std::vector<int32_t> pts(n * D);
        check(lsg_grid_regular(D, level, pts.data(), n, &n));
        for (int64_t k = 0; k < n; ++k) {
            Index I;
            for (int d = 0; d < D; ++d) I[d] = pts[k * D + d];
            AddPoint(I);
        }
    }
    // completeDirichletGrid (sgrid/sparseGrid.cc:771-787): the missing interior
    // points and the hanging nodes of this point set, added in the
    // reference's order (lsg_grid_complete).
    void completeDirichletGrid() {
        const int64_t n = getMaximalOccupiedSecondTable();
        int64_t m = 0;
        check(lsg_grid_complete(D, n, points_.data(), active_.data(), 1, nullptr, nullptr, 0, &m));
        std::vector<int32_t> pts(m * D);
        std::vector<uint8_t> act(m);
        check(lsg_grid_complete(D, n, points_.data(), active_.data(), 1, pts.data(), act.data(), m, &m));
        points_.swap(pts);
        active_.swap(act);
        where_.clear();
        for (int64_t k = 0; k < m; ++k) where_[getIndexOfTable(k)] = k;
    }
    // completeNeumannGrid (sgrid/sparseGrid.cc:654-740): passes in which every
    // active point adds (or activates) its same-level neighbours where its
    // depth is > 0 and the opposite boundary point where it is 0; only a newly
    // added point asks for another pass.  Adds the grid's boundary points.
    void completeNeumannGrid() {
        for (bool changed = true; changed;) {
            changed = false;
            int64_t end = getMaximalOccupiedSecondTable();
            for (int64_t i = 0; i < end; ++i) {
                if (!active_[i]) continue;
                const Index I = getIndexOfTable(i);
                for (int k = 0; k < D; ++k) {
                    Index J = I;
                    if (I[k] > 1) {
                        J[k] = I[k] >> (__builtin_ctz((unsigned)I[k]) + 1);
                        changed |= AddPoint(J);
                        J[k] = I[k] >> (__builtin_ctz(~(unsigned)I[k]) + 1);
                        changed |= AddPoint(J);
                    } else {
                        J[k] = 1;
                        changed |= AddPoint(J);
                        J[k] = 0;
                        changed |= AddPoint(J);
                    }
                }
            }
        }
    }
    int64_t getMaximalOccupiedSecondTable() const { return (int64_t)active_.size(); }
    Index getIndexOfTable(int64_t k) const {
        Index I;
        for (int d = 0; d < D; ++d) I[d] = points_[k * D + d];
        return I;
    }
    const uint8_t* getActiveTable() const { return active_.data(); }
    const int32_t* points() const { return points_.data(); }
    int64_t getDOFS() const {
        int64_t c = 0;
        for (auto a : active_) c += a;
        return c;
    }

private:
    std::vector<int32_t> points_;
    std::vector<uint8_t> active_;
    std::map<Index, int64_t> where_;
    mutable MatrixVectorHomogen<D>* attached_ = nullptr;
    mutable std::shared_ptr<MatrixVectorHomogen<D>> own_;
};

// MultiLevelAdaptiveSparseGrid (sgrid/multilevelSparseGrid.h:13-143): the
// reference's (I, T) store.  The flattened slabs of the operator hold it here,
// so this is a handle on the grid that keeps the reference's constructor.
template <int D>
class MultiLevelAdaptiveSparseGrid {
public:
    explicit MultiLevelAdaptiveSparseGrid(AdaptiveSparseGrid<D>* grid) : grid_(grid) {}
    AdaptiveSparseGrid<D>* getSparseGrid() const { return grid_; }

private:
    AdaptiveSparseGrid<D>* grid_;
};

template <int D>
class VectorSparseG {
public:
    explicit VectorSparseG(const AdaptiveSparseGrid<D>& g) : grid_(&g), data_(g.getMaximalOccupiedSecondTable(), 0.0) {}
    const AdaptiveSparseGrid<D>* getSparseGrid() const { return grid_; }
    double getValue(int64_t k) const { return data_[k]; }
    void setValue(int64_t k, double v) { data_[k] = v; }
    double* getDatatableVector() { return data_.data(); }
    const double* getDatatableVector() const { return data_.data(); }
    int64_t size() const { return (int64_t)data_.size(); }
    void operator=(double v) { std::fill(data_.begin(), data_.end(), v); }
    VectorSparseG& operator=(const VectorSparseG& o) {
        if (this != &o) {
            if (o.size() != size()) throw Error("VectorSparseG: vectors of different grids");
            data_ = o.data_;
        }
        return *this;
    }
    VectorSparseG(const VectorSparseG&) = default;
    // element-wise over all entries, like the reference's expression templates (extemp/extempAlg.h)
    friend VectorSparseG operator+(const VectorSparseG& a, const VectorSparseG& b) { return combine(a, b, 1.0); }
    friend VectorSparseG operator-(const VectorSparseG& a, const VectorSparseG& b) { return combine(a, b, -1.0); }
    friend VectorSparseG operator*(double s, const VectorSparseG& a) {
        VectorSparseG r(*a.grid_);
        for (int64_t k = 0; k < a.size(); ++k) r.data_[k] = s * a.data_[k];
        return r;
    }

private:
    static VectorSparseG combine(const VectorSparseG& a, const VectorSparseG& b, double sb) {
        if (a.size() != b.size()) throw Error("VectorSparseG: vectors of different grids");
        VectorSparseG r(*a.grid_);
        for (int64_t k = 0; k < a.size(); ++k) r.data_[k] = a.data_[k] + sb * b.data_[k];
        return r;
    }
    const AdaptiveSparseGrid<D>* grid_;
    std::vector<double> data_;
};

// The variable-coefficient plugin: a(x) sampled at cell midpoints times the
// exact Q1 stiffness entry (what StencilTemplate::integration returns).
struct MidpointDiffusion {
    int32_t family;
    std::vector<double> params;
    int32_t form = LSG_FORM_STIFFNESS;  // LSG_FORM_MASS: a(x) u v (HelmHoltz for a = 1)
};

// The reference's constant-coefficient operators (stencils/Stencil.h):
// Poisson is a = 1 with the stiffness form, HelmHoltz a = 1 with the mass
// form (Stencil.h:873-919).  The grid argument mirrors their constructors.
struct Poisson : MidpointDiffusion {
    template <class Grid>
    explicit Poisson(const Grid&) : MidpointDiffusion{LSG_COEF_CONST, {1.0}, LSG_FORM_STIFFNESS} {}
};
struct HelmHoltz : MidpointDiffusion {
    template <class Grid>
    explicit HelmHoltz(const Grid&) : MidpointDiffusion{LSG_COEF_CONST, {1.0}, LSG_FORM_MASS} {}
};

// L_infty(v) of the reference (applications/norms.h): the largest magnitude
template <int D>
inline double L_infty(const VectorSparseG<D>& v) {
    double m = 0.0;
    for (int64_t k = 0; k < v.size(); ++k) m = std::max(m, std::fabs(v.getValue(k)));
    return m;
}

template <int D>
class MatrixVectorHomogen {
public:
    explicit MatrixVectorHomogen(const AdaptiveSparseGrid<D>& g) : grid_(&g) {
        check(lsg_operator_create(D, g.points(), g.getActiveTable(), g.getMaximalOccupiedSecondTable(), &op_));
        g.attach(this);
    }
    // The reference's constructor (MatrixVectorHomogen.h:72-77).
    MatrixVectorHomogen(AdaptiveSparseGrid<D>& g, MultiLevelAdaptiveSparseGrid<D>& mgrid, bool symmetry, bool mpi_on)
        : MatrixVectorHomogen(g) {
        (void)symmetry;
        if (mgrid.getSparseGrid() != &g) throw Error("MatrixVectorHomogen: mgrid was built on another grid");
        if (mpi_on) throw Error("MatrixVectorHomogen: no MPI distribution (one GPU)");
    }
    ~MatrixVectorHomogen() {
        grid_->detach(this);
        lsg_operator_destroy(op_);
    }
    MatrixVectorHomogen(const MatrixVectorHomogen&) = delete;
    MatrixVectorHomogen& operator=(const MatrixVectorHomogen&) = delete;

    void setProblem(const MidpointDiffusion& p) {
        if (have_ && p.family == fam_ && p.params == par_ && p.form == form_) return;
        check(lsg_operator_set_coefficient(op_, p.family, p.params.data(), (int32_t)p.params.size()));
        check(lsg_operator_set_form(op_, p.form));
        form_ = p.form;
        fam_ = p.family;
        par_ = p.params;
        have_ = true;
    }
    // Ax = A_prew prew at active points (hanging entries of Ax untouched).
    void multiplication(const VectorSparseG<D>& prew, VectorSparseG<D>& Ax, const MidpointDiffusion& problem) {
        setProblem(problem);
        check(lsg_matvec(op_, prew.getDatatableVector(), Ax.getDatatableVector()));
    }
    lsg_operator* handle() { return op_; }
    // picks the matvec launch parameters by timing (lsg_operator_autotune); needs a problem set
    void autotune(const MidpointDiffusion& problem, int32_t precision = LSG_FP32, int reps = 3) {
        setProblem(problem);
        check(lsg_operator_autotune(op_, precision, reps, nullptr, nullptr, nullptr));
    }

private:
    const AdaptiveSparseGrid<D>* grid_;
    lsg_operator* op_ = nullptr;
    bool have_ = false;
    int32_t fam_ = -1, form_ = LSG_FORM_STIFFNESS;
    std::vector<double> par_;
};

template <int D>
MatrixVectorHomogen<D>& AdaptiveSparseGrid<D>::op() const {
    if (attached_) return *attached_;
    if (!own_) {
        own_ = std::make_shared<MatrixVectorHomogen<D>>(*this);
        attached_ = own_.get();
    }
    return *own_;
}

struct CG {
    // CG::solveHomogen(eps, x, f, &iterations, usol, matrix, stencil, &time)
    // (applications/cg_method.h:27-33): Jacobi-preconditioned CG with the
    // reference's stopping rule on r^T D^-1 r.  usol is accepted as the
    // reference takes it (its error history output is not written); *time
    // receives the solve's seconds.
    template <int D>
    static bool solveHomogen(double eps, VectorSparseG<D>& x, const VectorSparseG<D>& f, int* iterations,
                             const VectorSparseG<D>& usol, MatrixVectorHomogen<D>& matrix,
                             const MidpointDiffusion& problem, double* time) {
        (void)usol;
        return solveHomogen<D>(eps, x, f, iterations, matrix, problem, time);
    }
    template <int D>
    static bool solveHomogen(double eps, VectorSparseG<D>& x, const VectorSparseG<D>& f, int* iterations,
                             MatrixVectorHomogen<D>& matrix, const MidpointDiffusion& problem, double* seconds,
                             lsg_solver_opts* opts = nullptr) {
        matrix.setProblem(problem);
        lsg_solver_opts o{};
        if (opts) o = *opts;
        else {
            o.eps = eps;
            o.criterion = 0;
            o.use_graph = 1;
        }
        lsg_solve_report rep{};
        check(lsg_cg_solve(matrix.handle(), f.getDatatableVector(), x.getDatatableVector(), &o, &rep));
        if (iterations) *iterations = rep.iterations;
        if (seconds) *seconds = rep.seconds;
        return true;
    }
};

// calcNodalByPrew(prew, u) / calcPrewByNodal(prew, u)
// (BasisTransformations/BasisTransformations.h:119-125): the grid's flattened
// tables live in the operator, so the operator is passed as well.
template <int D>
inline void calcNodalByPrew(const VectorSparseG<D>& prew, VectorSparseG<D>& u, MatrixVectorHomogen<D>& matrix) {
    check(lsg_calc_nodal_by_prew(matrix.handle(), prew.getDatatableVector(), u.getDatatableVector()));
}
template <int D>
inline void calcPrewByNodal(VectorSparseG<D>& prew, const VectorSparseG<D>& u, MatrixVectorHomogen<D>& matrix) {
    check(lsg_calc_prew_by_nodal(matrix.handle(), prew.getDatatableVector(), u.getDatatableVector()));
}
// The reference's two-argument forms: the operator of the vectors' grid.
template <int D>
inline void calcNodalByPrew(const VectorSparseG<D>& prew, VectorSparseG<D>& u) {
    calcNodalByPrew<D>(prew, u, prew.getSparseGrid()->op());
}
template <int D>
inline void calcPrewByNodal(VectorSparseG<D>& prew, const VectorSparseG<D>& u) {
    calcPrewByNodal<D>(prew, u, prew.getSparseGrid()->op());
}

// H1::getValue / L2::getValue (applications/H1_Norm.cpp): the H1 seminorm and
// the L2 norm of the function with nodal values u.  The reference constructs
// them from (grid, mgrid); here from the grid's operator (any coefficient:
// the norms use a = 1 and leave the operator's own coefficient in place).
template <int D>
class H1 {
public:
    explicit H1(MatrixVectorHomogen<D>& matrix) : m_(matrix) {}
    H1(AdaptiveSparseGrid<D>& grid, MultiLevelAdaptiveSparseGrid<D>&) : m_(grid.op()) {}
    double getValue(const VectorSparseG<D>& u) {
        double v = 0.0;
        check(lsg_h1_norm(m_.handle(), u.getDatatableVector(), &v));
        return v;
    }

private:
    MatrixVectorHomogen<D>& m_;
};
template <int D>
class L2 {
public:
    explicit L2(MatrixVectorHomogen<D>& matrix) : m_(matrix) {}
    L2(AdaptiveSparseGrid<D>& grid, MultiLevelAdaptiveSparseGrid<D>&) : m_(grid.op()) {}
    double getValue(const VectorSparseG<D>& u) {
        double v = 0.0;
        check(lsg_l2_norm(m_.handle(), u.getDatatableVector(), &v));
        return v;
    }

private:
    MatrixVectorHomogen<D>& m_;
};

// CalcHierarchicalBasisForRHS(u) (MatrixVectorMultiplication/RHS.cpp:6-41):
// u lives on a grid with boundary points; its boundary values become
// hierarchical coefficients.
template <int D>
inline void CalcHierarchicalBasisForRHS(VectorSparseG<D>& u) {
    const AdaptiveSparseGrid<D>& g = *u.getSparseGrid();
    check(lsg_hierarchize_boundary(D, g.getMaximalOccupiedSecondTable(), g.points(), u.getDatatableVector()));
}

// InHomoBoundaryRHSHierarchical (MatrixVectorMultiplication/RHS.h:278-427):
// the reference is constructed from the interior grid; here from its operator.
// The boundary grid comes with the coefficient vector, as in the reference.
template <int D>
class InHomoBoundaryRHSHierarchical {
public:
    explicit InHomoBoundaryRHSHierarchical(MatrixVectorHomogen<D>& matrix) : m_(matrix) {}
    void multiply(const VectorSparseG<D>& hierarchical, VectorSparseG<D>& dirichlet) {
        run(LSG_BDRHS_GRADIENT, hierarchical, dirichlet);
    }
    void multiply_mass(const VectorSparseG<D>& hierarchical, VectorSparseG<D>& dirichlet) {
        run(LSG_BDRHS_MASS, hierarchical, dirichlet);
    }
    void multiply_mass_coeff(const VectorSparseG<D>& hierarchical, VectorSparseG<D>& dirichlet) {
        run(LSG_BDRHS_MASS_COEFF, hierarchical, dirichlet);
    }

private:
    void run(int32_t kind, const VectorSparseG<D>& h, VectorSparseG<D>& y) {
        const AdaptiveSparseGrid<D>& bg = *h.getSparseGrid();
        check(lsg_boundary_rhs(m_.handle(), kind, bg.getMaximalOccupiedSecondTable(), bg.points(),
                               h.getDatatableVector(), y.getDatatableVector()));
    }
    MatrixVectorHomogen<D>& m_;
};

// CalcHierarchicalBasis(u) / CalcNodalBasis(u)
// (BasisTransformations/BasisTransformations.cpp:390-409, :174-198) on the
// vector's own grid, boundary points allowed.
template <int D>
inline void CalcHierarchicalBasis(VectorSparseG<D>& u) {
    const AdaptiveSparseGrid<D>& g = *u.getSparseGrid();
    check(lsg_hierarchize(D, g.getMaximalOccupiedSecondTable(), g.points(), g.getActiveTable(), u.getDatatableVector()));
}
template <int D>
inline void CalcNodalBasis(VectorSparseG<D>& u) {
    const AdaptiveSparseGrid<D>& g = *u.getSparseGrid();
    check(lsg_dehierarchize(D, g.getMaximalOccupiedSecondTable(), g.points(), g.getActiveTable(), u.getDatatableVector()));
}

// PDE_Poisson_InHomRHS / PDE_Helmholtz_VariableCoeff (applications/PDE.h,
// PDE.cpp): the right-hand side on the interior grid of a problem with
// boundary data; SetUp transforms f and g in place as the reference does.
template <int D, int32_t KIND>
class PDE_InHomRHS {
public:
    PDE_InHomRHS(AdaptiveSparseGrid<D>& n_grid, AdaptiveSparseGrid<D>& d_grid, MatrixVectorHomogen<D>& matrix)
        : ngrid_(n_grid), f_dirichlet_(d_grid), matrix_(matrix) {}
    void SetUp(VectorSparseG<D>& f_neumann, VectorSparseG<D>& g_neumann) {
        check(lsg_pde_boundary_rhs(matrix_.handle(), KIND, ngrid_.getMaximalOccupiedSecondTable(), ngrid_.points(),
                                   ngrid_.getActiveTable(), f_neumann.getDatatableVector(),
                                   g_neumann.getDatatableVector(), f_dirichlet_.getDatatableVector()));
    }
    VectorSparseG<D>& getRHS() { return f_dirichlet_; }

private:
    AdaptiveSparseGrid<D>& ngrid_;
    VectorSparseG<D> f_dirichlet_;
    MatrixVectorHomogen<D>& matrix_;
};
template <int D>
using PDE_Poisson_InHomRHS = PDE_InHomRHS<D, LSG_PDE_POISSON>;
template <int D>
using PDE_Helmholtz_VariableCoeff = PDE_InHomRHS<D, LSG_PDE_HELMHOLTZ>;

}  // namespace lsg
