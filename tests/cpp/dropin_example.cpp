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
    std::printf("N=%lld iterations=%d relres=%.3e\n", (long long)grid.getMaximalOccupiedSecondTable(), it,
                std::sqrt(rr / ff));
    return std::sqrt(rr / ff) < 1e-8 ? 0 : 1;
}
