// Drop-in usage of include/loadsg/loadsg.hpp, written the way a LoAdSG main
// (library/examples_doxygen/poisson_regular.cpp:43-131) calls the reference.
#include <cmath>
#include <cstdio>

#include "loadsg/loadsg.hpp"

int main() {
    lsg::AdaptiveSparseGrid<3> grid;
    grid.AddRecursiveSonsOfPoint(5);
    lsg::MatrixVectorHomogen<3> m(grid);
    lsg::MidpointDiffusion problem{LSG_COEF_SINPROD, {1.0, 0.5, 1.0, 1.0, 1.0}};
    lsg::VectorSparseG<3> f(grid), x(grid), Ax(grid);
    for (int64_t k = 0; k < grid.getMaximalOccupiedSecondTable(); ++k) f.setValue(k, std::sin(0.1 * k));
    int it = 0;
    double secs = 0;
    lsg::CG::solveHomogen<3>(1e-20, x, f, &it, m, problem, &secs);
    m.multiplication(x, Ax, problem);
    double rr = 0, ff = 0;
    for (int64_t k = 0; k < f.size(); ++k) {
        double r = f.getValue(k) - Ax.getValue(k);
        rr += r * r;
        ff += f.getValue(k) * f.getValue(k);
    }
    // solution read out as nodal values and back (calcNodalByPrew / calcPrewByNodal)
    lsg::VectorSparseG<3> u(grid), back(grid);
    lsg::calcNodalByPrew<3>(x, u, m);
    lsg::calcPrewByNodal<3>(back, u, m);
    double dmax = 0;
    for (int64_t k = 0; k < x.size(); ++k) dmax = std::fmax(dmax, std::fabs(back.getValue(k) - x.getValue(k)));
    // norms of the solution's nodal values (H1::getValue / L2::getValue)
    double h1 = lsg::H1<3>(m).getValue(u), l2 = lsg::L2<3>(m).getValue(u);
    if (!(h1 > 0.0 && l2 > 0.0 && std::isfinite(h1) && std::isfinite(l2))) return 2;
    // boundary data g = 1 (PDE_Poisson_InHomRHS::SetUp, applications/PDE.cpp):
    // its extension is the constant 1, so the gradient form vanishes and the
    // mass form at the root (the level-1 hat) is 2^-3
    lsg::AdaptiveSparseGrid<3> bgrid;
    bgrid.AddRecursiveSonsOfPoint(5);
    bgrid.completeNeumannGrid();
    lsg::VectorSparseG<3> g(bgrid), rhs(grid), mass(grid);
    for (int64_t k = 0; k < bgrid.getMaximalOccupiedSecondTable(); ++k) {
        auto I = bgrid.getIndexOfTable(k);
        bool boundary = I[0] < 2 || I[1] < 2 || I[2] < 2;
        g.setValue(k, boundary ? 1.0 : 0.0);
    }
    lsg::CalcHierarchicalBasisForRHS<3>(g);
    lsg::InHomoBoundaryRHSHierarchical<3> bd(m);
    bd.multiply(g, rhs);
    bd.multiply_mass(g, mass);
    double gmax = 0;
    for (int64_t k = 0; k < rhs.size(); ++k) gmax = std::fmax(gmax, std::fabs(rhs.getValue(k)));
    // the whole right-hand side of -lap u = 0, u = 1 on the boundary: zero
    lsg::VectorSparseG<3> f0(bgrid), g1(bgrid);
    for (int64_t k = 0; k < bgrid.getMaximalOccupiedSecondTable(); ++k) {
        auto I = bgrid.getIndexOfTable(k);
        g1.setValue(k, (I[0] < 2 || I[1] < 2 || I[2] < 2) ? 1.0 : 0.0);
    }
    lsg::PDE_Poisson_InHomRHS<3> pde(bgrid, grid, m);
    pde.SetUp(f0, g1);
    for (int64_t k = 0; k < grid.getMaximalOccupiedSecondTable(); ++k)
        gmax = std::fmax(gmax, std::fabs(pde.getRHS().getValue(k)));
    std::printf("N=%lld iterations=%d relres=%.3e transform round trip %.3e boundary: |grad| %.3e root mass %.6f\n",
                (long long)grid.getMaximalOccupiedSecondTable(), it, std::sqrt(rr / ff), dmax, gmax, mass.getValue(0));
    return (std::sqrt(rr / ff) < 1e-8 && dmax < 1e-10 && gmax < 1e-10 && mass.getValue(0) == 0.125) ? 0 : 1;
}
