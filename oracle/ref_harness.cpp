// Reference harness: TEST INFRASTRUCTURE ONLY.
//
// A driver of our own that is compiled against the unmodified LoAdSG sources
// (oracle/Makefile builds them in place) and calls only the reference's public
// API.  It generates the golden vectors that pin the oracle and the CUDA path:
//   * grids built by AdaptiveSparseGrid::AddRecursiveSonsOfPoint
//     (library/source/sgrid/sparseGrid.cc:557-566), optional refinement by
//     AddPoint of sons, then completeDirichletGrid (sparseGrid.cc:771-787);
//   * integer tables read back through the reference's own lookups
//     (DepthList, sortDepths, MultiDepthHashGrid, CellData, nextFiveP);
//   * the variable-coefficient matvec through the reference plugin point
//     StencilTemplate::integration (library/source/stencils/Stencil.h:740)
//     consumed by LocalStiffnessMatricesMemoryDistribution and
//     MatrixVectorHomogen::multiplication (MatrixVectorHomogen.h:659-759);
//   * the Jacobi diagonal (Preconditioning, applications/cg_method.h:81-754)
//     and CG::solveHomogen (cg_method.h:759-886);
//   * the basis transforms calcNodalByPrew / calcPrewByNodal
//     (BasisTransformations/BasisTransformations.cpp:486-545,670-706).
// Outputs are raw little-endian arrays in an output directory plus meta.txt;
// tests/golden/make_golden.py packs them into .npz fixtures.
#include "sparseEXPDE.h"
#include "coefficient.h"

#include <chrono>
#include <cstdio>
#include <fstream>
#include <map>
#include <string>
#include <vector>

static const int D = DimensionSparseGrid;

// ---------------------------------------------------------------- options
static std::map<std::string, std::string> g_opt;
static std::string opt(const char *k, const char *def) {
    auto it = g_opt.find(k);
    return it == g_opt.end() ? std::string(def) : it->second;
}
static std::vector<double> parse_list(const std::string &s) {
    std::vector<double> v;
    size_t i = 0;
    while (i < s.size()) {
        size_t j = s.find(',', i);
        if (j == std::string::npos) j = s.size();
        if (j > i) v.push_back(atof(s.substr(i, j - i).c_str()));
        i = j + 1;
    }
    return v;
}

// ---------------------------------------------------------------- I/O
static std::string g_out;
static std::ofstream g_meta;
template <class T>
static void dump(const char *name, const std::vector<T> &v) {
    std::string p = g_out + "/" + name;
    FILE *f = fopen(p.c_str(), "wb");
    if (!f) { perror(p.c_str()); exit(2); }
    if (!v.empty()) fwrite(v.data(), sizeof(T), v.size(), f);
    fclose(f);
    g_meta << "array " << name << " " << v.size() << "\n";
}
static std::vector<double> read_f64(const std::string &p, size_t n) {
    std::vector<double> v(n, 0.0);
    FILE *f = fopen(p.c_str(), "rb");
    if (!f) { perror(p.c_str()); exit(2); }
    size_t got = fread(v.data(), sizeof(double), n, f);
    fclose(f);
    if (got != n) { fprintf(stderr, "short read %s\n", p.c_str()); exit(2); }
    return v;
}

// ---------------------------------------------------------------- plugin
// Midpoint-coefficient diffusion: a(x_c) times the exact Q1 stiffness entry.
class MidpointDiffusion : public StencilTemplate {
public:
    int family;
    std::vector<double> p;
    int form = 0;  // 0: a(x_c) * Q1 stiffness, 1: a(x_c) * Q1 mass
    MidpointDiffusion(AdaptiveSparseGrid &g, int fam, std::vector<double> par)
        : StencilTemplate(g), family(fam), p(par) { p.resize(LSG_COEF_MAXPARAM, 0.0); }
    double integration(CellDimension &cell, CellIndexDirection &dp, CellIndexDirection &dq) override {
        double h[D], xc[D];
        unsigned mp = 0, mq = 0;
        for (int d = 0; d < D; ++d) {
            double lo = cell.getLeftBoundary(d), hi = cell.getRightBoundary(d);
            h[d] = hi - lo;
            xc[d] = 0.5 * (lo + hi);
            if (dp.getDirection(d) == Right) mp |= 1u << d;
            if (dq.getDirection(d) == Right) mq |= 1u << d;
        }
        return lsg_coef_eval(family, p.data(), D, xc) * lsg_q1_entry(form, D, h, mp, mq);
    }
};

// ---------------------------------------------------------------- grid
static bool refine_point(const IndexDimension &I, int round, const std::string &target, double theta) {
    double thr = theta / double(1 << (round - 1));
    if (target == "corner") {
        for (int d = 0; d < D; ++d)
            if (!(I.coordinate(d) < thr)) return false;
        return true;
    }
    if (target == "plane") return fabs(I.coordinate(0) - 0.5) < thr;
    return false;
}

static void build_grid(AdaptiveSparseGrid &grid) {
    int level = atoi(opt("level", "3").c_str());
    int refine = atoi(opt("refine", "0").c_str());
    double theta = atof(opt("theta", "0.5").c_str());
    std::string target = opt("target", "corner");
    IndexDimension center;
    grid.AddRecursiveSonsOfPoint(center, level);
    for (int r = 1; r <= refine; ++r) {
        std::vector<IndexDimension> todo;
        for (unsigned long k = 0; k < grid.getMaximalOccupiedSecondTable(); ++k) {
            if (!grid.getActiveTable()[k]) continue;
            IndexDimension I = grid.getIndexOfTable(k);
            if (refine_point(I, r, target, theta)) todo.push_back(I);
        }
        for (auto &I : todo)
            for (int d = 0; d < D; ++d) {
                grid.AddPoint(I.leftSon(d));
                grid.AddPoint(I.rightSon(d));
            }
    }
    if (refine > 0 || opt("complete", "0") == "1") grid.completeDirichletGrid();
}

static void dump_grid(AdaptiveSparseGrid &grid) {
    unsigned long N = grid.getMaximalOccupiedSecondTable();
    std::vector<int32_t> idx(N * D);
    std::vector<uint8_t> act(N);
    for (unsigned long k = 0; k < N; ++k) {
        IndexDimension I = grid.getIndexOfTable(k);
        for (int d = 0; d < D; ++d) idx[k * D + d] = I.getIndex(d);
        act[k] = grid.getActiveTable()[k] ? 1 : 0;
    }
    dump("points.i32", idx);
    dump("active.u8", act);
    g_meta << "N " << N << "\nd " << D << "\ndofs " << grid.getDOFS() << "\n";
}

// ---------------------------------------------------------------- tables
static long lookup(AdaptiveSparseGrid &grid, IndexDimension I) {
    unsigned long k;
    if (grid.occupied(k, I)) return (long)k;
    return -1;
}

static void dump_tables(AdaptiveSparseGrid &grid) {
    unsigned long N = grid.getMaximalOccupiedSecondTable();
    DepthList dl(grid);
    std::vector<int32_t> depths;
    std::vector<Depth> dv;
    for (auto it = dl.begin_all(); it != dl.end_all(); ++it) {
        dv.push_back(*it);
        for (int d = 0; d < D; ++d) depths.push_back(it->at(d));
    }
    dump("depthlist.i32", depths);
    // per-case sorted depth order (CasesIterator bit i = restriction in dim i)
    std::vector<int32_t> sorted, sorted_off;
    for (CasesIterator ci; ci.goon(); ++ci) {
        bool *r = ci.getcase();
        dl.sortDepths(r);
        sorted_off.push_back((int32_t)sorted.size() / D);
        for (Depth T : *dl.getSortierteTiefen())
            for (int d = 0; d < D; ++d) sorted.push_back(T.at(d));
    }
    sorted_off.push_back((int32_t)sorted.size() / D);
    dump("sorted.i32", sorted);
    dump("sorted_off.i32", sorted_off);
    // points of exact depth (MultiDepthHashGrid insertion order)
    std::vector<int32_t> exact, exact_off;
    for (Depth T : dv) {
        exact_off.push_back((int32_t)exact.size());
        SingleDepthHashGrid &g = grid.getMultiDepthHashGrid()->getGridForDepth(T);
        for (auto k : g._mapPosToGridPos) exact.push_back((int32_t)k);
    }
    exact_off.push_back((int32_t)exact.size());
    dump("exact.i32", exact);
    dump("exact_off.i32", exact_off);
    // multilevel store size
    MultiLevelAdaptiveSparseGrid mgrid(&grid);
    g_meta << "mgrid_size " << mgrid.getMaximalOccupiedSecondTable() << "\n";
    // same-level 1D neighbours (IndexDimension::nextLeft/nextRight) per dim
    std::vector<int32_t> nb(N * D * 2);
    for (unsigned long k = 0; k < N; ++k) {
        IndexDimension I = grid.getIndexOfTable(k);
        for (int d = 0; d < D; ++d) {
            nb[(k * D + d) * 2 + 0] = (int32_t)lookup(grid, I.nextLeft(d));
            nb[(k * D + d) * 2 + 1] = (int32_t)lookup(grid, I.nextRight(d));
        }
    }
    dump("nbr1d.i32", nb);
    // prewavelet 5^d stencil of every active point at its own depth (nextFiveP,
    // indices/index.cc:252-327) as used by calcNodal (MatrixVectorHomogen.cpp:43-74)
    std::vector<int32_t> st_j, st_off;
    std::vector<double> st_w;
    for (unsigned long k = 0; k < N; ++k) {
        st_off.push_back((int32_t)st_j.size());
        if (!grid.getActiveTable()[k]) continue;
        IndexDimension I = grid.getIndexOfTable(k);
        Depth T(I);
        MultiDimFiveCompass mc;
        for (; mc.hasNext(); ++mc) {
            double w = 1.0;
            IndexDimension J = I.nextFiveP(&mc, T, &w);
            if (mc.goon()) {
                st_j.push_back((int32_t)lookup(grid, J));
                st_w.push_back(w);
            }
        }
    }
    st_off.push_back((int32_t)st_j.size());
    dump("stencil_j.i32", st_j);
    dump("stencil_w.f64", st_w);
    dump("stencil_off.i32", st_off);
    // cells of depth T+1 for every depth T, corners in CellIndexIterator order
    CellData cd(grid);
    std::vector<int32_t> cells, cells_off, corner_idx;
    for (Depth T : dv) {
        Depth Tc = T;
        ++Tc;
        cells_off.push_back((int32_t)(cells.size() >> D));
        const SingleDepthHashCellStructure &cg = cd.getGridForDepth(Tc);
        for (size_t i = 0; i < cg.getNumberOfEntries(); ++i) {
            CellDimension cell = cg._map.getIndexOfTable(i);
            for (CellIndexIterator it(&cell); it.goon(); ++it) {
                IndexDimension P = it.getIndex();
                cells.push_back(P.isNotAtBoundary() ? (int32_t)lookup(grid, P) : -1);
                for (int d = 0; d < D; ++d) corner_idx.push_back(P.getIndex(d));
            }
        }
    }
    cells_off.push_back((int32_t)(cells.size() >> D));
    dump("cells.i32", cells);
    dump("cells_off.i32", cells_off);
    dump("cell_corners.i32", corner_idx);
}

// ---------------------------------------------------------------- numerics
static MidpointDiffusion make_plugin(AdaptiveSparseGrid &grid) {
    int fam = atoi(opt("coef", "1").c_str());
    std::vector<double> p = parse_list(opt("cp", "1,0.5,1,1,1,1,1,1,1,1"));
    return MidpointDiffusion(grid, fam, p);
}

static void set_vec(VectorSparseG &v, const std::vector<double> &x) {
    for (unsigned long k = 0; k < x.size(); ++k) v.setValue(k, x[k]);
}
static std::vector<double> get_vec(VectorSparseG &v, unsigned long N) {
    std::vector<double> y(N);
    for (unsigned long k = 0; k < N; ++k) y[k] = v.getValue(k);
    return y;
}

int main(int argc, char **argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s grid|tables|matvec|poisson|diag|cg outdir [key=value ...]\n", argv[0]);
        return 2;
    }
    std::string cmd = argv[1];
    g_out = argv[2];
    for (int i = 3; i < argc; ++i) {
        std::string a = argv[i];
        size_t e = a.find('=');
        if (e != std::string::npos) g_opt[a.substr(0, e)] = a.substr(e + 1);
    }
    g_meta.open(g_out + "/meta_" + cmd + ".txt");
    AdaptiveSparseGrid grid;
    build_grid(grid);
    unsigned long N = grid.getMaximalOccupiedSecondTable();
    if (cmd == "grid") {
        dump_grid(grid);
    } else if (cmd == "tables") {
        dump_tables(grid);
    } else if (cmd == "h1norm" || cmd == "l2norm") {
        // H1::getValue / L2::getValue (applications/H1_Norm.cpp) of the nodal values x
        std::vector<double> x = read_f64(opt("x", ""), N);
        MultiLevelAdaptiveSparseGrid mgrid(&grid);
        VectorSparseG uv(grid);
        set_vec(uv, x);
        double val;
        if (cmd == "h1norm") {
            H1 norm(grid, mgrid);
            val = norm.getValue(uv);
        } else {
            L2 norm(grid, mgrid);
            val = norm.getValue(uv);
        }
        char buf[64];
        snprintf(buf, sizeof buf, "%.17g", val);
        g_meta << "value " << buf << "\n";
    } else if (cmd == "mass" || cmd == "helmholtz") {
        // mass: the midpoint plugin with the Q1 mass matrix; helmholtz: the
        // reference's own HelmHoltz stencil (Stencil.h:873-919, coefficient 1)
        std::vector<double> x = read_f64(opt("x", ""), N);
        MultiLevelAdaptiveSparseGrid mgrid(&grid);
        MatrixVectorHomogen m(grid, mgrid, true, false);
        VectorSparseG xv(grid), yv(grid);
        set_vec(xv, x);
        if (cmd == "helmholtz") {
            HelmHoltz helm(grid);
            m.multiplication(xv, yv, helm);
        } else {
            MidpointDiffusion plug = make_plugin(grid);
            plug.form = 1;
            LocalStiffnessMatricesMemoryDistribution lsm(grid, plug, 1);
            m.multiplication(xv, yv, lsm);
        }
        dump("y.f64", get_vec(yv, N));
    } else if (cmd == "matvec" || cmd == "poisson") {
        std::vector<double> x = read_f64(opt("x", ""), N);
        MultiLevelAdaptiveSparseGrid mgrid(&grid);
        MatrixVectorHomogen m(grid, mgrid, true, false);
        VectorSparseG xv(grid), yv(grid);
        set_vec(xv, x);
        auto t0 = std::chrono::steady_clock::now();
        double secs;
        if (cmd == "poisson") {
            Poisson pois(grid);
            t0 = std::chrono::steady_clock::now();
            m.multiplication(xv, yv, pois);
            secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        } else {
            MidpointDiffusion plug = make_plugin(grid);
            LocalStiffnessMatricesMemoryDistribution lsm(grid, plug, 1);
            int reps = atoi(opt("reps", "1").c_str());
            t0 = std::chrono::steady_clock::now();
            for (int r = 0; r < reps; ++r) m.multiplication(xv, yv, lsm);
            secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() / reps;
        }
        dump("y.f64", get_vec(yv, N));
        g_meta << "matvec_seconds " << secs << "\n";
    } else if (cmd == "diag" || cmd == "massdiag") {
        MidpointDiffusion plug = make_plugin(grid);
        if (cmd == "massdiag") plug.form = 1;
        LocalStiffnessMatricesMemoryDistribution lsm(grid, plug, 1);
        VectorSparseG z(grid);
        Preconditioning<LocalStiffnessMatricesMemoryDistribution> P(z, lsm);
        dump("diag.f64", get_vec(z, N));
    } else if (cmd == "cg") {
        std::vector<double> f = read_f64(opt("f", ""), N);
        double eps = atof(opt("eps", "1e-10").c_str());
        MultiLevelAdaptiveSparseGrid mgrid(&grid);
        MatrixVectorHomogen m(grid, mgrid, true, false);
        MidpointDiffusion plug = make_plugin(grid);
        LocalStiffnessMatricesMemoryDistribution lsm(grid, plug, 1);
        VectorSparseG fv(grid), xv(grid), usol(grid), r(grid);
        set_vec(fv, f);
        xv = 0.0;
        int it = 0;
        double tp = 0.0;
        auto t0 = std::chrono::steady_clock::now();
        CG::solveHomogen(eps, xv, fv, &it, usol, m, lsm, &tp);
        double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        m.multiplication(xv, r, lsm);
        std::vector<double> x = get_vec(xv, N), Ax = get_vec(r, N);
        double rr = 0.0, ff = 0.0;
        for (unsigned long k = 0; k < N; ++k) {
            rr += (f[k] - Ax[k]) * (f[k] - Ax[k]);
            ff += f[k] * f[k];
        }
        dump("x.f64", x);
        g_meta << "iterations " << it << "\nrelres " << sqrt(rr / ff) << "\nsolve_seconds " << secs
               << "\nprecond_seconds " << tp << "\n";
    } else if (cmd == "bdrhs") {
        // Boundary-data right-hand sides (MatrixVectorMultiplication/RHS.h:278-427,
        // RHS.cpp:6-41,697-1008): a second grid with boundary points, built like
        // the first and then completeNeumannGrid (sparseGrid.cc:654-677); boundary
        // values g = family gfam at the boundary points, 0 inside;
        // CalcHierarchicalBasisForRHS(g), then InHomoBoundaryRHSHierarchical
        // multiply / multiply_mass / multiply_mass_coeff onto this grid.
        AdaptiveSparseGrid ngrid;
        build_grid(ngrid);
        ngrid.completeNeumannGrid();
        unsigned long NN = ngrid.getMaximalOccupiedSecondTable();
        int gfam = atoi(opt("gfam", "1").c_str());
        std::vector<double> gp = parse_list(opt("gp", "1,0.5,1,1,1,1,1,1,1,1"));
        gp.resize(LSG_COEF_MAXPARAM, 0.0);
        std::vector<int32_t> nidx(NN * D);
        std::vector<uint8_t> nact(NN);
        std::vector<double> g(NN, 0.0);
        for (unsigned long k = 0; k < NN; ++k) {
            IndexDimension I = ngrid.getIndexOfTable(k);
            double x[D];
            bool boundary = false;
            for (int d = 0; d < D; ++d) {
                nidx[k * D + d] = I.getIndex(d);
                x[d] = I.coordinate(d);
                if (I.getIndex(d) < 2) boundary = true;
            }
            nact[k] = ngrid.getActiveTable()[k] ? 1 : 0;
            if (boundary) g[k] = lsg_coef_eval(gfam, gp.data(), D, x);
        }
        dump("npoints.i32", nidx);
        dump("nactive.u8", nact);
        dump("g.f64", g);
        VectorSparseG gv(ngrid), yv(grid);
        set_vec(gv, g);
        CalcHierarchicalBasisForRHS(gv);
        dump("g_hier.f64", get_vec(gv, NN));
        InHomoBoundaryRHSHierarchical rhs(grid);
        auto since = [](std::chrono::steady_clock::time_point t) {
            return std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
        };
        auto t0 = std::chrono::steady_clock::now();
        yv = 0.0;
        rhs.multiply(gv, yv);
        double secs = since(t0);
        dump("y_stiff.f64", get_vec(yv, N));
        yv = 0.0;
        t0 = std::chrono::steady_clock::now();
        rhs.multiply_mass(gv, yv);
        double secs_mass = since(t0);
        dump("y_mass.f64", get_vec(yv, N));
        yv = 0.0;
        t0 = std::chrono::steady_clock::now();
        rhs.multiply_mass_coeff(gv, yv);
        double secs_coeff = since(t0);
        dump("y_coeff.f64", get_vec(yv, N));
        g_meta << "NN " << NN << "\nstiff_seconds " << secs << "\nmass_seconds " << secs_mass
               << "\ncoeff_seconds " << secs_coeff << "\n";
    } else if (cmd == "pdesetup") {
        // Right-hand sides of problems with boundary data (applications/PDE.h,
        // PDE.cpp): f (family ffam) on every point of the grid with boundary
        // points, g (family gfam) on its boundary points; PDE_Poisson_InHomRHS
        // and PDE_Helmholtz_VariableCoeff SetUp, plus the two transforms they
        // use on their own: CalcHierarchicalBasis of f on that grid and
        // CalcNodalBasis of x on this one (BasisTransformations.cpp:174-198,390-409).
        AdaptiveSparseGrid ngrid;
        build_grid(ngrid);
        ngrid.completeNeumannGrid();
        unsigned long NN = ngrid.getMaximalOccupiedSecondTable();
        auto fam_vals = [&](const char *fk, const char *pk, bool boundary_only) {
            int fam = atoi(opt(fk, "1").c_str());
            std::vector<double> p = parse_list(opt(pk, "1,0.5,1,1,1,1,1,1,1,1"));
            p.resize(LSG_COEF_MAXPARAM, 0.0);
            std::vector<double> v(NN, 0.0);
            for (unsigned long k = 0; k < NN; ++k) {
                IndexDimension I = ngrid.getIndexOfTable(k);
                double x[D];
                bool boundary = false;
                for (int d = 0; d < D; ++d) {
                    x[d] = I.coordinate(d);
                    if (I.getIndex(d) < 2) boundary = true;
                }
                if (boundary || !boundary_only) v[k] = lsg_coef_eval(fam, p.data(), D, x);
            }
            return v;
        };
        std::vector<double> f = fam_vals("ffam", "fp", false), g = fam_vals("gfam", "gp", true);
        std::vector<int32_t> nidx(NN * D);
        std::vector<uint8_t> nact(NN);
        for (unsigned long k = 0; k < NN; ++k) {
            IndexDimension I = ngrid.getIndexOfTable(k);
            for (int d = 0; d < D; ++d) nidx[k * D + d] = I.getIndex(d);
            nact[k] = ngrid.getActiveTable()[k] ? 1 : 0;
        }
        dump("npoints.i32", nidx);
        dump("nactive.u8", nact);
        dump("f.f64", f);
        dump("g.f64", g);
        VectorSparseG fh(ngrid);
        set_vec(fh, f);
        CalcHierarchicalBasis(fh);
        dump("f_hier.f64", get_vec(fh, NN));
        std::vector<double> x = read_f64(opt("x", ""), N);
        VectorSparseG xv(grid);
        set_vec(xv, x);
        CalcNodalBasis(xv);
        dump("x_nodal.f64", get_vec(xv, N));
        MultiLevelAdaptiveSparseGrid mgrid(&grid);
        MatrixVectorHomogen m(grid, mgrid, true, false);
        for (int which = 0; which < 2; ++which) {
            VectorSparseG fv(ngrid), gv(ngrid);
            set_vec(fv, f);
            set_vec(gv, g);
            std::vector<double> rhs;
            if (which == 0) {
                PDE_Poisson_InHomRHS pde(ngrid, grid, m);
                pde.SetUp(fv, gv);
                rhs = get_vec(pde.getRHS(), N);
            } else {
                PDE_Helmholtz_VariableCoeff pde(ngrid, grid, m);
                pde.SetUp(fv, gv);
                rhs = get_vec(pde.getRHS(), N);
            }
            dump(which == 0 ? "rhs_poisson.f64" : "rhs_helmholtz.f64", rhs);
        }
        g_meta << "NN " << NN << "\n";
    } else if (cmd == "poissonex") {
        // The steps of examples_doxygen/poisson_regular.cpp through the
        // reference's API, for levels 1..levels: u = prod sin(pi x_d), f = d pi^2 u
        // at the active points; f to prewavelets (calcPrewByNodal), the
        // right-hand side by the HelmHoltz product, CG::solveHomogen with the
        // Poisson stencil at eps = 1e-10, the solution back to nodal values
        // (calcNodalByPrew); the error's maximum, L2 and L2 + H1 norms.
        int levels = atoi(opt("levels", "5").c_str());
        std::vector<double> dofs, iters, linf, l2v, h1v;
        for (int level = 1; level <= levels; ++level) {
            AdaptiveSparseGrid pg;
            IndexDimension c;
            pg.AddRecursiveSonsOfPoint(c, level);
            MultiLevelAdaptiveSparseGrid pm(&pg);
            unsigned long PN = pg.getMaximalOccupiedSecondTable();
            VectorSparseG u(pg), f(pg), rhs(pg), prew(pg), w(pg), err(pg);
            u = 0.0;
            f = 0.0;
            for (unsigned long k = 0; k < PN; ++k) {
                if (!pg.getActiveTable()[k]) continue;
                IndexDimension I = pg.getIndexOfTable(k);
                double s = 1.0;
                for (int d = 0; d < D; ++d) s *= sin(M_PI * I.coordinate(d));
                u.setValue(k, s);
                f.setValue(k, double(D) * M_PI * M_PI * s);
            }
            MatrixVectorHomogen mv(pg, pm, true, false);
            HelmHoltz helm(pg);
            Poisson pois(pg);
            prew = 0.0;
            calcPrewByNodal(prew, f);
            rhs = 0.0;
            mv.multiplication(prew, rhs, helm);
            prew = 0.0;
            int it = 0;
            double tp = 0.0;
            CG::solveHomogen(1e-10, prew, rhs, &it, u, mv, pois, &tp);
            w = 0.0;
            calcNodalByPrew(prew, w);
            err = u - w;
            L2 l2n(pg, pm);
            H1 h1n(pg, pm);
            double l2 = l2n.getValue(err);
            dofs.push_back(pg.getDOFS());
            iters.push_back(it);
            linf.push_back(L_infty(err));
            l2v.push_back(l2);
            h1v.push_back(h1n.getValue(err) + l2);
        }
        dump("dofs.f64", dofs);
        dump("iterations.f64", iters);
        dump("linfty.f64", linf);
        dump("l2.f64", l2v);
        dump("h1.f64", h1v);
    } else if (cmd == "complete") {
        // A caller's grid completed by the reference: the points of file `pts`
        // (np x D int32) added with AddPoint in order, then completeDirichletGrid
        // (mode=dirichlet, sgrid/sparseGrid.cc:771-787) or completeNeumannGrid
        // (mode=neumann, :654-740).  The grid built from level=... is not used.
        long np = atol(opt("np", "0").c_str());
        std::vector<int32_t> in(np * D);
        FILE *f = fopen(opt("pts", "").c_str(), "rb");
        if (!f || fread(in.data(), sizeof(int32_t), in.size(), f) != in.size()) { fprintf(stderr, "pts\n"); return 2; }
        fclose(f);
        AdaptiveSparseGrid cg;
        for (long k = 0; k < np; ++k) {
            IndexDimension I;
            for (int d = 0; d < D; ++d) I.replace(d, in[k * D + d]);
            cg.AddPoint(I);
        }
        if (opt("mode", "dirichlet") == "neumann") cg.completeNeumannGrid();
        else cg.completeDirichletGrid();
        dump_grid(cg);
    } else if (cmd == "prew2nodal" || cmd == "nodal2prew") {
        // prew2nodal: u = calcNodalByPrew(x); nodal2prew: p = calcPrewByNodal(x)
        std::vector<double> x = read_f64(opt("x", ""), N);
        VectorSparseG in(grid), out(grid);
        set_vec(in, x);
        auto t0 = std::chrono::steady_clock::now();
        if (cmd == "prew2nodal") calcNodalByPrew(in, out);
        else calcPrewByNodal(out, in);
        double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        dump("y.f64", get_vec(out, N));
        dump("x_after.f64", get_vec(in, N));
        g_meta << "seconds " << secs << "\n";
    } else {
        fprintf(stderr, "unknown command %s\n", cmd.c_str());
        return 2;
    }
    g_meta << "ok 1\n";
    return 0;
}
