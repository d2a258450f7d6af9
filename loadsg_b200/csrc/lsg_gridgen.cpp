// Host-side adaptive grid generation: refinement plus the reference's
// completion of a locally adaptive sparse grid (AdaptiveSparseGrid::
// completeDirichletGrid, sgrid/sparseGrid.cc:771-787).  The stages, in order:
//   (a) completeGridWithoutBoundary   sparseGrid.cc:741-769
//   (b) CompleteToLocalTensorProductGrid  localTensorProduct.cc:189-224,
//       LocalForTensor::recursiveMarkArbeite2 / checkRechteck (:122-183)
//   (c) completeGridWithoutBoundary
//   (d) addHangingNodes              sparseGrid.cc:587-619
//   (e) addPoints2                   GridGeneration.cpp:333-392 (+ support,
//       overlap, refill :12-200)
// Points are kept in insertion (storage) order; the iteration orders of the
// reference are kept as well, so the result is the reference's grid, storage
// order included.  Stage (e) visits the reference's point pairs in the
// reference's order but finds them through the grid's index instead of a
// pairwise scan (add_points2 below).
#include "../../include/lsg.h"

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <vector>

namespace {

inline int depth1(int32_t i) { return i == 0 ? 0 : 31 - __builtin_clz((unsigned)i); }
inline int32_t next_left1(int32_t i) { return i >> (__builtin_ctz((unsigned)i) + 1); }
inline int32_t next_right1(int32_t i) { return i >> (__builtin_ctz(~(unsigned)i) + 1); }
inline bool interior1(int32_t i) { return i > 1; }
// level-t coordinate (coordinate * 2^t) of a 1D index of depth <= t; boundary 0 -> 0, 1 -> 2^t
inline int64_t coord_at(int32_t i, int t) {
    if (i == 0) return 0;
    if (i == 1) return (int64_t)1 << t;
    int ti = depth1(i);
    return (2 * (int64_t)(i - (1 << ti)) + 1) << (t - ti);
}
// 1D index of a level-t coordinate c (0 <= c <= 2^t)
inline int32_t index_of(int64_t c, int t) {
    if (c == 0) return 0;
    if (c == ((int64_t)1 << t)) return 1;
    int tz = __builtin_ctzll((unsigned long long)c);
    int tt = t - tz;
    int64_t odd = c >> tz;
    return (int32_t)((1 << tt) + (odd - 1) / 2);
}

struct Grid {
    int d;
    std::vector<int32_t> pts;
    std::vector<uint8_t> act;
    std::vector<int64_t> slot;  // open addressing, -1 empty
    // depth groups in first-appearance order with their members in insertion order
    std::map<std::vector<int32_t>, int> gid;
    std::vector<std::vector<int32_t>> gdepth;
    std::vector<std::vector<int64_t>> gmem;

    explicit Grid(int d_) : d(d_) { slot.assign(1 << 12, -1); }
    int64_t n() const { return (int64_t)act.size(); }
    const int32_t* P(int64_t k) const { return &pts[k * d]; }

    static uint64_t hsh(const int32_t* I, int d) {
        uint64_t h = 1469598103934665603ull;
        for (int k = 0; k < d; ++k) { h ^= (uint32_t)I[k]; h *= 1099511628211ull; h ^= h >> 29; }
        return h;
    }
    int64_t find(const int32_t* I) const {
        uint64_t m = slot.size() - 1, h = hsh(I, d) & m;
        for (;;) {
            int64_t s = slot[h];
            if (s < 0) return -1;
            if (!memcmp(P(s), I, sizeof(int32_t) * d)) return s;
            h = (h + 1) & m;
        }
    }
    void rehash() {
        std::vector<int64_t> ns(slot.size() * 2, -1);
        uint64_t m = ns.size() - 1;
        for (int64_t k = 0; k < n(); ++k) {
            uint64_t h = hsh(P(k), d) & m;
            while (ns[h] >= 0) h = (h + 1) & m;
            ns[h] = k;
        }
        slot.swap(ns);
    }
    // append a new point (caller checked absence)
    int64_t append(const int32_t* I, bool active) {
        if ((uint64_t)(n() + 1) * 2 > slot.size()) rehash();
        int64_t k = n();
        pts.insert(pts.end(), I, I + d);
        act.push_back(active ? 1 : 0);
        uint64_t m = slot.size() - 1, h = hsh(I, d) & m;
        while (slot[h] >= 0) h = (h + 1) & m;
        slot[h] = k;
        std::vector<int32_t> T(d);
        for (int j = 0; j < d; ++j) T[j] = depth1(I[j]);
        auto it = gid.find(T);
        int g;
        if (it == gid.end()) {
            g = (int)gdepth.size();
            gid[T] = g;
            gdepth.push_back(T);
            gmem.push_back({});
        } else g = it->second;
        gmem[g].push_back(k);
        return k;
    }
    // AdaptiveSparseGrid::AddPoint(I): new points active, existing ones made active
    bool add_active(const int32_t* I) {
        int64_t k = find(I);
        if (k >= 0) { act[k] = 1; return false; }
        append(I, true);
        return true;
    }
    // AddPoint(I, flag): new points active iff flag, existing ones untouched
    bool add_flag(const int32_t* I, bool flag) {
        if (find(I) >= 0) return false;
        append(I, flag);
        return true;
    }
};

void regular(Grid& g, std::vector<int32_t>& I, int level) {  // AddRecursiveSonsOfPoint, memoised
    if (g.find(I.data()) >= 0) return;
    g.add_active(I.data());
    if (level <= 0) return;
    for (int k = 0; k < g.d; ++k) {
        int32_t s = I[k];
        I[k] = s << 1;
        regular(g, I, level - 1);
        I[k] = (s << 1) + 1;
        regular(g, I, level - 1);
        I[k] = s;
    }
}

double coordinate(int32_t i) {
    if (i == 0) return 0.0;
    if (i == 1) return 1.0;
    int t = depth1(i);
    return (double)(2 * (i - (1 << t)) + 1) / (double)(1 << t);
}

// (a)/(c) completeGridWithoutBoundary: passes over the table adding missing
// interior same-level neighbours until nothing changes
void complete_without_boundary(Grid& g) {
    int d = g.d;
    std::vector<int32_t> J(d);
    for (bool changed = true; changed;) {
        changed = false;
        int64_t end = g.n();
        for (int64_t i = 0; i < end; ++i) {
            for (int k = 0; k < d; ++k) {
                for (int side = 0; side < 2; ++side) {
                    memcpy(J.data(), g.P(i), sizeof(int32_t) * d);
                    J[k] = side ? next_right1(J[k]) : next_left1(J[k]);
                    bool inner = true;
                    for (int j = 0; j < d; ++j) inner &= interior1(J[j]);
                    if (inner && g.find(J.data()) < 0) {
                        g.add_active(J.data());
                        changed = true;
                    }
                }
            }
        }
    }
}

// completeNeumannGrid = completeGrid (sparseGrid.cc:654-740): passes over the
// table in which every active point adds (or activates) its two same-level
// neighbours in each dimension where its depth is > 0, boundary points
// included, and the opposite boundary point in each dimension where its depth
// is 0.  Only a newly added point asks for another pass, as in the reference.
void complete_neumann(Grid& g) {
    int d = g.d;
    std::vector<int32_t> I(d), J(d);
    for (bool changed = true; changed;) {
        changed = false;
        int64_t end = g.n();
        for (int64_t i = 0; i < end; ++i) {
            if (!g.act[i]) continue;
            memcpy(I.data(), g.P(i), sizeof(int32_t) * d);
            for (int k = 0; k < d; ++k) {
                J = I;
                if (I[k] > 1) {
                    J[k] = next_left1(I[k]);
                    changed |= g.add_active(J.data());
                    J[k] = next_right1(I[k]);
                    changed |= g.add_active(J.data());
                } else {
                    J[k] = 1;
                    changed |= g.add_active(J.data());
                    J[k] = 0;
                    changed |= g.add_active(J.data());
                }
            }
        }
    }
}

// valid 1D stencil positions of an interior index i at its depth t
// (nextFive without weights): c, c-1, c+1, c-2, c+2 in level-t coordinates
int stencil_pos(int32_t i, int64_t* pos) {
    int t = depth1(i);
    int64_t c = coord_at(i, t), top = (int64_t)1 << t;
    int n = 0;
    bool lok = c - 1 > 0, rok = c + 1 < top;
    pos[n++] = c;
    if (lok) pos[n++] = c - 1;
    if (rok) pos[n++] = c + 1;
    if (lok) pos[n++] = c - 2;
    if (rok) pos[n++] = c + 2;
    return n;
}

// (b) CompleteToLocalTensorProductGrid
void complete_tensor(Grid& g) {
    int d = g.d;
    // depth groups present now, ordered by |T|_1, then first appearance
    std::vector<int> order(g.gdepth.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = (int)k;
    auto l1 = [&](int k) { int s = 0; for (int v : g.gdepth[k]) s += v; return s; };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return l1(a) < l1(b); });
    std::vector<uint8_t> marked;
    std::vector<int32_t> lo(d), hi(d), J(d);
    for (int gi : order) {
        std::vector<int32_t> T = g.gdepth[gi];
        // members of the group in storage order; points added to it meanwhile
        // are appended and visited too (LocalForTensor::findAnichtWithDepth)
        for (size_t mi = 0; mi < g.gmem[gi].size(); ++mi) {
            int64_t i = g.gmem[gi][mi];
            if ((int64_t)marked.size() < g.n()) marked.resize(g.n(), 0);
            if (marked[i] || !g.act[i]) continue;
            marked[i] = 1;
            // bounding box (level-T coordinates) of the point and its active stencil neighbours
            int64_t pos[8][5];
            int np[8];
            for (int k = 0; k < d; ++k) np[k] = stencil_pos(g.P(i)[k], pos[k]);
            int64_t bmin[8], bmax[8], emin[8], emax[8];
            for (int k = 0; k < d; ++k) {
                bmin[k] = bmax[k] = coord_at(g.P(i)[k], T[k]);
                emin[k] = *std::min_element(pos[k], pos[k] + np[k]);  // the stencil's extent
                emax[k] = *std::max_element(pos[k], pos[k] + np[k]);
            }
            int ctr[8] = {0};
            for (;;) {
                for (int k = 0; k < d; ++k) J[k] = index_of(pos[k][ctr[k]], T[k]);
                int64_t s = g.find(J.data());
                if (s >= 0 && g.act[s]) {
                    bool full = true;
                    for (int k = 0; k < d; ++k) {
                        bmin[k] = std::min(bmin[k], pos[k][ctr[k]]);
                        bmax[k] = std::max(bmax[k], pos[k][ctr[k]]);
                        full &= bmin[k] == emin[k] && bmax[k] == emax[k];
                    }
                    if (full) break;  // no further neighbour can widen the box
                }
                int k = 0;
                while (k < d && ++ctr[k] == np[k]) { ctr[k] = 0; ++k; }
                if (k == d) break;
            }
            // fill every level-T grid point of the box (dim 0 fastest)
            int64_t c[8];
            for (int k = 0; k < d; ++k) c[k] = bmin[k];
            for (;;) {
                for (int k = 0; k < d; ++k) J[k] = index_of(c[k], T[k]);
                int64_t s = g.find(J.data());
                if (s < 0) g.add_flag(J.data(), true);
                else g.act[s] = 1;
                int k = 0;
                while (k < d && ++c[k] > bmax[k]) { c[k] = bmin[k]; ++k; }
                if (k == d) break;
            }
        }
    }
}

// (d) addHangingNodes: the prewavelet stencil of every active point.  The
// points it adds are inactive and lie beyond the visited range, so the
// missing stencil positions of every point can be found in parallel on the
// grid as it was; they are then added in point order (a position missing for
// two points is added at the first, as in the sequential pass).
void add_hanging(Grid& g) {
    const int d = g.d;
    const int64_t end = g.n();
    const int64_t chunk = 4096;
    std::vector<std::vector<int32_t>> miss((size_t)((end + chunk - 1) / chunk));
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t cb = 0; cb < (int64_t)miss.size(); ++cb) {
        std::vector<int32_t> J(d);
        std::vector<int32_t>& out = miss[cb];
        for (int64_t i = cb * chunk; i < std::min(end, (cb + 1) * chunk); ++i) {
            if (!g.act[i]) continue;
            int64_t pos[8][5];
            int np[8], t[8];
            for (int k = 0; k < d; ++k) {
                t[k] = depth1(g.P(i)[k]);
                np[k] = stencil_pos(g.P(i)[k], pos[k]);
            }
            int ctr[8] = {0};
            for (;;) {
                for (int k = 0; k < d; ++k) J[k] = index_of(pos[k][ctr[k]], t[k]);
                if (g.find(J.data()) < 0) out.insert(out.end(), J.begin(), J.end());
                int k = 0;
                while (k < d && ++ctr[k] == np[k]) { ctr[k] = 0; ++k; }
                if (k == d) break;
            }
        }
    }
    for (const auto& out : miss)
        for (size_t o = 0; o < out.size(); o += d) g.add_flag(&out[o], false);
}

// support of a point (GridGeneration.cpp:12-40) in level-t_k coordinates per dim
void support(const int32_t* I, int d, int64_t* lo, int64_t* hi, int* t) {
    for (int k = 0; k < d; ++k) {
        t[k] = depth1(I[k]);
        int64_t c = coord_at(I[k], t[k]), top = (int64_t)1 << t[k];
        if (t[k] <= 2) { lo[k] = 0; hi[k] = top; continue; }
        lo[k] = (c - 1 == 0) ? 0 : c - 3;
        hi[k] = (c + 1 == top) ? top : c + 3;
    }
}

// (e) addPoints2 (GridGeneration.cpp:333-392): for pairs of depth groups T1,
// T2 (depth-list order, differing in >= 2 dims) and active P in T1, Q in T2
// with overlapping supports: if a depth-T point (T = max(T1, T2)) lies in the
// overlap, add every interior depth-T point of the overlap as a hanging node.
// The reference tests every pair of points; here, with the same visiting
// order and the same additions:
//   * a group pair is skipped when the depth-T group holds every point of
//     depth T (prod_k 2^(T_k - 1)): no overlap can miss one;
//   * for an active P, the Q of T2 whose supports can overlap P's lie on T2's
//     lattice inside P's support widened by Q's half support; they are looked
//     up by their indices, filtered by the exact overlap test and visited in
//     storage order, which is the order of the group's member list (points
//     are appended; points added by this stage are inactive and never become
//     a P or a Q).
void add_points2(Grid& g) {
    const int d = g.d;
    const int ngroups = (int)g.gdepth.size();
    std::vector<int32_t> J(d);
    std::vector<int64_t> cand;
    for (bool changed = true; changed;) {
        changed = false;
        for (int a = 0; a < ngroups; ++a) {
            for (int b = a + 1; b < ngroups; ++b) {
                const std::vector<int32_t> T1 = g.gdepth[a], T2 = g.gdepth[b];
                int lone = 0;
                int T[8];
                for (int k = 0; k < d; ++k) {
                    lone += T1[k] != T2[k];
                    T[k] = std::max(T1[k], T2[k]);
                }
                if (lone < 2) continue;
                auto tg = g.gid.find(std::vector<int32_t>(T, T + d));
                if (tg == g.gid.end()) continue;
                // every point of depth T present (prod_k 2^(T_k - 1) of them): no
                // overlap box can miss one, so this pair adds nothing
                int64_t full = 1;
                for (int k = 0; k < d && full > 0; ++k) full = T[k] >= 1 ? full << (T[k] - 1) : 0;
                if (full > 0 && (int64_t)g.gmem[tg->second].size() == full) continue;
                for (size_t ia = 0; ia < g.gmem[a].size(); ++ia) {
                    const int64_t p = g.gmem[a][ia];
                    if (!g.act[p]) continue;
                    int64_t plo[8], phi[8], c0[8], c1[8], cs[8];
                    int pt[8];
                    support(g.P(p), d, plo, phi, pt);
                    // candidate centres of Q per dimension: odd level-T2 coordinates,
                    // or both boundary coordinates 0 and 1 at depth 0
                    bool none = false;
                    for (int k = 0; k < d && !none; ++k) {
                        const int t = T2[k], sh = T[k] - t;
                        if (t == 0) {
                            c0[k] = 0;
                            c1[k] = 1;
                            cs[k] = 1;
                            continue;
                        }
                        cs[k] = 2;
                        const int64_t A0 = plo[k] << (T[k] - pt[k]), A1 = phi[k] << (T[k] - pt[k]);
                        const int64_t top = (int64_t)1 << t;
                        int64_t lo = std::max<int64_t>(1, ((A0 + ((int64_t)1 << sh) - 1) >> sh) - 3);
                        int64_t hi = std::min<int64_t>(top - 1, (A1 >> sh) + 3);
                        lo |= 1;
                        if (lo > hi) none = true;
                        c0[k] = lo;
                        c1[k] = hi;
                    }
                    if (none) continue;
                    cand.clear();
                    int64_t c[8];
                    for (int k = 0; k < d; ++k) c[k] = c0[k];
                    for (;;) {
                        for (int k = 0; k < d; ++k) J[k] = index_of(c[k], T2[k]);
                        const int64_t q = g.find(J.data());
                        if (q >= 0 && g.act[q]) cand.push_back(q);
                        int k = 0;
                        while (k < d && (c[k] += cs[k]) > c1[k]) { c[k] = c0[k]; ++k; }
                        if (k == d) break;
                    }
                    std::sort(cand.begin(), cand.end());
                    for (int64_t q : cand) {
                        int64_t qlo[8], qhi[8];
                        int qt[8];
                        support(g.P(q), d, qlo, qhi, qt);
                        int64_t lo[8], hi[8];
                        bool ov = true;
                        for (int k = 0; k < d && ov; ++k) {
                            int64_t a0 = plo[k] << (T[k] - pt[k]), a1 = phi[k] << (T[k] - pt[k]);
                            int64_t b0 = qlo[k] << (T[k] - qt[k]), b1 = qhi[k] << (T[k] - qt[k]);
                            if (b1 < a0 || a1 < b0) ov = false;
                            lo[k] = std::max(a0, b0);
                            hi[k] = std::min(a1, b1);
                        }
                        if (!ov) continue;
                        int64_t e0[8];
                        bool empty = false;
                        for (int k = 0; k < d; ++k) {
                            e0[k] = lo[k] | 1;
                            if (e0[k] > hi[k]) empty = true;
                        }
                        if (empty) continue;
                        bool any = false;
                        int64_t e[8];
                        for (int k = 0; k < d; ++k) e[k] = e0[k];
                        for (;;) {
                            for (int k = 0; k < d; ++k) J[k] = index_of(e[k], T[k]);
                            if (g.find(J.data()) >= 0) { any = true; break; }
                            int k = 0;
                            while (k < d && (e[k] += 2) > hi[k]) { e[k] = e0[k]; ++k; }
                            if (k == d) break;
                        }
                        if (!any) continue;
                        for (int k = 0; k < d; ++k) e[k] = e0[k];
                        for (;;) {
                            for (int k = 0; k < d; ++k) J[k] = index_of(e[k], T[k]);
                            if (g.add_flag(J.data(), false)) changed = true;
                            int k = 0;
                            while (k < d && (e[k] += 2) > hi[k]) { e[k] = e0[k]; ++k; }
                            if (k == d) break;
                        }
                    }
                }
            }
        }
    }
}

}  // namespace

// Refinement criteria of the benchmark/test grids: round r (1-based) refines
// every active point whose coordinates satisfy
//   target 0 (corner): max_k x_k < theta 2^(1-r)
//   target 1 (plane):  |x_0 - 1/2| < theta 2^(1-r)
// by adding its left and right son in every dimension.
namespace {
// the last generated grid of this thread, so that a size query followed by the
// fill call generates it once
struct LastGrid {
    int32_t d = -1, level = -1, refine = -1, target = -1, complete = -1;
    double theta = -1.0;
    std::vector<int32_t> pts;
    std::vector<uint8_t> act;
};
thread_local LastGrid g_last;
}  // namespace

// Completes a caller's grid: the points (n x d, in storage order, with their
// active flags) are taken as they are, then the completion stages of
// `complete` run on them and the result is returned in the same way as
// lsg_grid_adaptive returns its grid.
extern "C" int lsg_grid_complete(int32_t d, int64_t n, const int32_t* points, const uint8_t* active,
                                 int32_t complete, int32_t* out_points, uint8_t* out_active, int64_t capacity,
                                 int64_t* n_out) {
    if (d < 1 || d > 8 || n < 0 || (n > 0 && (!points || !active)) || !n_out) return LSG_E_INVALID;
    Grid g(d);
    for (int64_t k = 0; k < n; ++k) {
        const int32_t* I = points + k * d;
        for (int j = 0; j < d; ++j)
            if (I[j] < 0) return LSG_E_INVALID;
        if (g.find(I) >= 0) return LSG_E_INVALID;  // duplicate point
        g.append(I, active[k] != 0);
    }
    int mask = complete == 1 ? 0x3e : complete;
    if (mask & 2) complete_without_boundary(g);
    if (mask & 4) complete_tensor(g);
    if (mask & 8) complete_without_boundary(g);
    if (mask & 16) add_hanging(g);
    if (mask & 32) add_points2(g);
    if (mask & 64) complete_neumann(g);
    *n_out = g.n();
    if (out_points || out_active) {
        if (capacity < g.n()) return LSG_E_INVALID;
        if (out_points) memcpy(out_points, g.pts.data(), g.pts.size() * sizeof(int32_t));
        if (out_active) memcpy(out_active, g.act.data(), g.act.size());
    }
    return 0;
}

extern "C" int lsg_grid_adaptive(int32_t d, int32_t level, int32_t refine, double theta, int32_t target,
                                 int32_t complete, int32_t* points, uint8_t* active, int64_t capacity, int64_t* n) {
    if (d < 1 || d > 8 || level < 0 || level > 24 || refine < 0 || !n) return LSG_E_INVALID;
    LastGrid& L = g_last;
    if (L.d == d && L.level == level && L.refine == refine && L.theta == theta && L.target == target &&
        L.complete == complete) {
        *n = (int64_t)L.act.size();
        if (points || active) {
            if (capacity < *n) return LSG_E_INVALID;
            if (points) memcpy(points, L.pts.data(), L.pts.size() * sizeof(int32_t));
            if (active) memcpy(active, L.act.data(), L.act.size());
        }
        return 0;
    }
    Grid g(d);
    std::vector<int32_t> I(d, 2);
    regular(g, I, level);
    for (int r = 1; r <= refine; ++r) {
        double thr = theta / (double)(1 << (r - 1));
        std::vector<int64_t> todo;
        for (int64_t k = 0; k < g.n(); ++k) {
            if (!g.act[k]) continue;
            bool hit;
            if (target == 0) {
                hit = true;
                for (int j = 0; j < d; ++j) hit &= coordinate(g.P(k)[j]) < thr;
            } else {
                double x = coordinate(g.P(k)[0]) - 0.5;
                hit = (x < 0 ? -x : x) < thr;
            }
            if (hit) todo.push_back(k);
        }
        std::vector<int32_t> S(d);
        for (int64_t k : todo)
            for (int j = 0; j < d; ++j) {
                memcpy(S.data(), g.P(k), sizeof(int32_t) * d);
                S[j] = g.P(k)[j] << 1;
                g.add_active(S.data());
                S[j] = (g.P(k)[j] << 1) + 1;
                g.add_active(S.data());
            }
    }
    // complete: 0 none, 1 all stages, or a bit mask of stages a..e (bits 1..5)
    int mask = complete == 1 ? 0x3e : complete;
    if (mask & 2) complete_without_boundary(g);
    if (mask & 4) complete_tensor(g);
    if (mask & 8) complete_without_boundary(g);
    if (mask & 16) add_hanging(g);
    if (mask & 32) add_points2(g);
    if (mask & 64) complete_neumann(g);
    *n = g.n();
    L.d = d; L.level = level; L.refine = refine; L.theta = theta; L.target = target; L.complete = complete;
    L.pts = g.pts;
    L.act = g.act;
    if (points || active) {
        if (capacity < g.n()) return LSG_E_INVALID;
        if (points) memcpy(points, g.pts.data(), g.pts.size() * sizeof(int32_t));
        if (active) memcpy(active, g.act.data(), g.act.size());
    }
    return 0;
}
