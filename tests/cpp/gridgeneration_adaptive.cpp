// The reference's examples_doxygen/gridgeneration_adaptive.cpp written against
// the C++ drop-in: two points four levels below the centre, then
// completeDirichletGrid.  Prints the points (active flag, indices) and the
// counts; host code only, no GPU.
#include <cstdio>

#include "loadsg/loadsg.hpp"

int main() {
    lsg::AdaptiveSparseGrid<2> grid;
    lsg::AdaptiveSparseGrid<2>::Index bottomLeft{8, 8};  // centre.leftSon(0).leftSon(1).leftSon(0).leftSon(1)
    lsg::AdaptiveSparseGrid<2>::Index topRight{11, 11};  // the same with rightSon
    grid.AddPoint(bottomLeft);
    grid.AddPoint(topRight);
    grid.completeDirichletGrid();
    for (int64_t k = 0; k < grid.getMaximalOccupiedSecondTable(); ++k) {
        auto I = grid.getIndexOfTable(k);
        std::printf("%d %d %d\n", (int)grid.getActiveTable()[k], I[0], I[1]);
    }
    std::printf("# %lld %lld\n", (long long)grid.getDOFS(),
                (long long)(grid.getMaximalOccupiedSecondTable() - grid.getDOFS()));
    return 0;
}
