// Prints the boundary grid of the C++ drop-in's completeNeumannGrid (one point
// per line: active flag, then the 1D indices) for a regular grid of the level
// given as the only argument; host code only, no GPU.
#include <cstdio>
#include <cstdlib>

#include "loadsg/loadsg.hpp"

int main(int argc, char** argv) {
    int level = argc > 1 ? std::atoi(argv[1]) : 3;
    lsg::AdaptiveSparseGrid<3> grid;
    grid.AddRecursiveSonsOfPoint(level);
    grid.completeNeumannGrid();
    for (int64_t k = 0; k < grid.getMaximalOccupiedSecondTable(); ++k) {
        auto I = grid.getIndexOfTable(k);
        std::printf("%d %d %d %d\n", (int)grid.getActiveTable()[k], I[0], I[1], I[2]);
    }
    return 0;
}
