// Host-side grid generation (no GPU): regular sparse grids in the reference's
// storage order.  AdaptiveSparseGrid::AddRecursiveSonsOfPoint
// (sgrid/sparseGrid.cc:557-566) adds a point and recurses into the left and
// right son of every dimension; a point with sum_k (depth_k - 1) = s is always
// reached with remaining level L - s, so expanding each point once, in the
// same depth-first order, reproduces the reference's insertion order exactly
// while visiting O(N d) instead of O((2d)^L) nodes.
#include "../../include/lsg.h"

#include <cstring>
#include <string>
#include <unordered_set>
#include <vector>

namespace {
struct KeyHash {
    size_t operator()(const std::string& s) const { return std::hash<std::string>()(s); }
};
void rec(int d, std::vector<int32_t>& I, int level, std::unordered_set<std::string, KeyHash>& seen,
         std::vector<int32_t>& out) {
    std::string key(reinterpret_cast<const char*>(I.data()), I.size() * sizeof(int32_t));
    if (!seen.insert(key).second) return;
    out.insert(out.end(), I.begin(), I.end());
    if (level <= 0) return;
    for (int k = 0; k < d; ++k) {
        int32_t save = I[k];
        I[k] = save << 1;
        rec(d, I, level - 1, seen, out);
        I[k] = (save << 1) + 1;
        rec(d, I, level - 1, seen, out);
        I[k] = save;
    }
}
}  // namespace

extern "C" int lsg_grid_regular(int32_t d, int32_t level, int32_t* points, int64_t capacity, int64_t* n) {
    if (d < 1 || d > 8 || level < 0 || level > 24 || !n) return LSG_E_INVALID;
    std::vector<int32_t> I(d, 2), out;
    std::unordered_set<std::string, KeyHash> seen;
    rec(d, I, level, seen, out);
    *n = (int64_t)(out.size() / d);
    if (points) {
        if (capacity < *n) return LSG_E_INVALID;
        memcpy(points, out.data(), out.size() * sizeof(int32_t));
    }
    return 0;
}
