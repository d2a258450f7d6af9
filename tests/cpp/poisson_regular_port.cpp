// The reference's Poisson example (examples_doxygen/poisson_regular.cpp: -lap u
// = f on regular grids, u = prod sin(pi x_d)) written against the C++ drop-in.
// The calls map one to one: AddRecursiveSonsOfPoint, calcPrewByNodal, the
// HelmHoltz product for the right-hand side, CG::solveHomogen with Poisson,
// calcNodalByPrew, L_infty / L2 / H1 of the error.  Prints the convergence
// table for levels 1..5 (the reference prints the same columns).
#include <cmath>
#include <cstdio>

#include "loadsg/loadsg.hpp"

int main() {
    constexpr int D = 3;
    for (int level = 1; level <= 5; ++level) {
        lsg::AdaptiveSparseGrid<D> grid;
        grid.AddRecursiveSonsOfPoint(level);
        lsg::VectorSparseG<D> u(grid), f(grid), rhs(grid), prew(grid), w(grid), d(grid);
        const double pi = std::acos(-1.0);
        for (int64_t k = 0; k < grid.getMaximalOccupiedSecondTable(); ++k) {
            if (!grid.getActiveTable()[k]) continue;
            auto I = grid.getIndexOfTable(k);
            double s = 1.0;
            for (int j = 0; j < D; ++j) {
                int t = 31 - __builtin_clz((unsigned)I[j]);
                s *= std::sin(pi * (2.0 * (I[j] - (1 << t)) + 1.0) / double(1 << t));
            }
            u.setValue(k, s);
            f.setValue(k, D * pi * pi * s);
        }
        lsg::MatrixVectorHomogen<D> m(grid);
        lsg::HelmHoltz helmHoltz(grid);
        lsg::Poisson stencilPoisson(grid);
        lsg::calcPrewByNodal<D>(prew, f, m);
        m.multiplication(prew, rhs, helmHoltz);
        prew = 0.0;
        int iterations = 0;
        double seconds = 0.0;
        lsg::CG::solveHomogen<D>(1e-10, prew, rhs, &iterations, m, stencilPoisson, &seconds);
        lsg::calcNodalByPrew<D>(prew, w, m);
        for (int64_t k = 0; k < d.size(); ++k) d.setValue(k, u.getValue(k) - w.getValue(k));
        double l2 = lsg::L2<D>(m).getValue(d);
        double h1 = lsg::H1<D>(m).getValue(d) + l2;
        std::printf("%d %lld %.6e %.6e %.6e %d\n", level, (long long)grid.getDOFS(), lsg::L_infty(d), l2, h1,
                    iterations);
    }
    return 0;
}
