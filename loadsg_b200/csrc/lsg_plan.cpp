// Host planner for the prewavelet matvec (see lsg_plan.h for the reference anchors).
#include "lsg_plan.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <numeric>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace lsg {

int depth1(int32_t i) { return i == 0 ? 0 : 31 - __builtin_clz((unsigned)i); }

namespace {

// level-t integer coordinate of a 1D index of depth <= t (coordinate * 2^t)
inline int64_t coord_at(int32_t idx, int t) {
    int ti = depth1(idx);
    int64_t c = 2 * (int64_t)(idx - (1 << ti)) + 1;
    return c << (t - ti);
}

struct Geometry {  // level-T interior grid: coordinates 1..2^T_k-1 per dim
    int d;
    int64_t ext[kMaxDim];     // 2^T_k - 1
    uint64_t stride[kMaxDim];
    int64_t cext[kMaxDim];    // cells per dim: 2^T_k
    uint64_t cstride[kMaxDim];
    int32_t T[kMaxDim];
    explicit Geometry(int d_, const int32_t* T_) : d(d_) {
        uint64_t s = 1, cs = 1;
        for (int k = 0; k < d; ++k) {
            T[k] = T_[k];
            ext[k] = ((int64_t)1 << T_[k]) - 1;
            stride[k] = s;
            s *= (uint64_t)ext[k];
            cext[k] = (int64_t)1 << T_[k];
            cstride[k] = cs;
            cs *= (uint64_t)cext[k];
        }
    }
    uint64_t key(const int64_t* c) const {
        uint64_t k = 0;
        for (int j = 0; j < d; ++j) k += (uint64_t)(c[j] - 1) * stride[j];
        return k;
    }
    void decode(uint64_t key, int64_t* c) const {
        for (int j = 0; j < d; ++j) {
            c[j] = (int64_t)(key % (uint64_t)ext[j]) + 1;
            key /= (uint64_t)ext[j];
        }
    }
    uint64_t total() const {
        uint64_t t = 1;
        for (int j = 0; j < d; ++j) t *= (uint64_t)ext[j];
        return t;
    }
};

inline int64_t find_key(const uint64_t* keys, int64_t n, uint64_t k) {
    const uint64_t* it = std::lower_bound(keys, keys + n, k);
    if (it != keys + n && *it == k) return it - keys;
    return -1;
}

// slab position of level-T coordinates c (interior), -1 if absent
inline int64_t slab_pos(const Plan& p, int t, const Geometry& g, const int64_t* c) {
    uint64_t k = g.key(c);
    const Slab& s = p.slabs[t];
    if (s.dense) return (int64_t)k;
    return find_key(p.slab_key.data() + s.off, s.n, k);
}

// One-dimensional prewavelet stencil of an odd level-t coordinate c
// (IndexDimension::nextFiveP, indices/index.cc:252-327) in level-t coordinates:
// positions {c, c-1, c+1, c-2, c+2} in the reference's direction order
// (Mitte, Links, Rechts, LinksLinks, RechtsRechts), weight codes
// 1: 1.0, 2: 0.9 (next to the boundary, depth > 1), 3: -0.6, 4: 0.1.
inline int stencil1(int64_t c, int t, int64_t* pos, int* code) {
    int64_t top = (int64_t)1 << t;
    int n = 0;
    bool lok = c - 1 > 0, rok = c + 1 < top;
    pos[n] = c;
    code[n++] = (t > 1 && (!lok || !rok)) ? 2 : 1;
    if (lok) { pos[n] = c - 1; code[n++] = 3; }
    if (rok) { pos[n] = c + 1; code[n++] = 3; }
    if (lok) { pos[n] = c - 2; code[n++] = 4; }
    if (rok) { pos[n] = c + 2; code[n++] = 4; }
    return n;
}
// weight code of stencil(i) at position q (0 if q is not in it)
inline int stencil_code(int64_t i, int t, int64_t q) {
    int64_t pos[5];
    int code[5];
    int n = stencil1(i, t, pos, code);
    for (int s = 0; s < n; ++s)
        if (pos[s] == q) return code[s];
    return 0;
}

void sort_unique(std::vector<uint64_t>& v) {
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
}

// Sum-factorised tensor stencil transform for one depth.
//  nodal   (forward=true):  in = active exact-depth points, out = all slab entries;
//          stage j maps odd coordinates in dim j to any coordinate in their stencil.
//  convert (forward=false): in = slab entries, out = active exact-depth points;
//          stage j gathers the stencil of an odd coordinate in dim j.
struct StageOut {
    std::vector<std::vector<uint64_t>> dom;  // d+1 domains (sorted keys)
    std::vector<std::vector<int32_t>> src;   // d stages
    std::vector<std::vector<int32_t>> code;
};

void build_transform(const Geometry& g, const std::vector<uint64_t>& in_keys, const std::vector<uint64_t>& out_keys,
                     bool nodal, int nsrc, StageOut& so) {
    int d = g.d;
    so.dom.assign(d + 1, {});
    so.src.assign(d, {});
    so.code.assign(d, {});
    // forward reachability
    std::vector<std::vector<uint64_t>> fwd(d + 1);
    fwd[0] = in_keys;
    int64_t c[kMaxDim], pos[5];
    int code[5];
    for (int j = 0; j < d; ++j) {
        std::vector<uint64_t> nxt;
        nxt.reserve(fwd[j].size() * (nodal ? 3 : 2));
        int64_t top = (int64_t)1 << g.T[j];
        for (uint64_t k : fwd[j]) {
            g.decode(k, c);
            int64_t cj = c[j];
            if (nodal) {  // odd cj spreads to its stencil
                int n = stencil1(cj, g.T[j], pos, code);
                for (int s = 0; s < n; ++s) { c[j] = pos[s]; nxt.push_back(g.key(c)); }
            } else {      // any cj reaches the odd coordinates whose stencil contains it
                for (int64_t o = -2; o <= 2; ++o) {
                    int64_t i = cj + o;
                    if (i < 1 || i >= top || !(i & 1)) continue;
                    if (stencil_code(i, g.T[j], cj)) { c[j] = i; nxt.push_back(g.key(c)); }
                }
            }
            c[j] = cj;
        }
        sort_unique(nxt);
        fwd[j + 1].swap(nxt);
    }
    // backward need, intersected with reachability
    so.dom[d] = out_keys;
    for (int j = d - 1; j >= 0; --j) {
        std::vector<uint64_t> need;
        need.reserve(so.dom[j + 1].size() * 3);
        int64_t top = (int64_t)1 << g.T[j];
        for (uint64_t k : so.dom[j + 1]) {
            g.decode(k, c);
            int64_t cj = c[j];
            if (nodal) {
                for (int64_t o = -2; o <= 2; ++o) {
                    int64_t i = cj + o;
                    if (i < 1 || i >= top || !(i & 1)) continue;
                    if (stencil_code(i, g.T[j], cj)) { c[j] = i; need.push_back(g.key(c)); }
                }
            } else {
                int n = stencil1(cj, g.T[j], pos, code);
                for (int s = 0; s < n; ++s) { c[j] = pos[s]; need.push_back(g.key(c)); }
            }
            c[j] = cj;
        }
        sort_unique(need);
        if (j == 0) {
            so.dom[0] = in_keys;  // stage-0 sources index the input list directly
        } else {
            std::vector<uint64_t> dom;
            std::set_intersection(need.begin(), need.end(), fwd[j].begin(), fwd[j].end(), std::back_inserter(dom));
            so.dom[j].swap(dom);
        }
    }
    // gather tables
    for (int j = 0; j < d; ++j) {
        const auto& out = so.dom[j + 1];
        const auto& in = so.dom[j];
        auto& src = so.src[j];
        auto& cod = so.code[j];
        src.assign(out.size() * nsrc, -1);
        cod.assign(out.size(), 0);
        int64_t top = (int64_t)1 << g.T[j];
        for (size_t e = 0; e < out.size(); ++e) {
            g.decode(out[e], c);
            int64_t cj = c[j];
            int ns = 0;
            int packed = 0;
            if (nodal) {
                for (int64_t o = -2; o <= 2; ++o) {
                    int64_t i = cj + o;
                    if (i < 1 || i >= top || !(i & 1)) continue;
                    int cd = stencil_code(i, g.T[j], cj);
                    if (!cd) continue;
                    c[j] = i;
                    int64_t at = find_key(in.data(), (int64_t)in.size(), g.key(c));
                    if (at >= 0) {
                        src[e * nsrc + ns] = (int32_t)at;
                        packed |= cd << (3 * ns);
                        ++ns;
                    }
                }
            } else {
                int n = stencil1(cj, g.T[j], pos, code);
                for (int s = 0; s < n; ++s) {
                    c[j] = pos[s];
                    int64_t at = find_key(in.data(), (int64_t)in.size(), g.key(c));
                    if (at >= 0) {
                        src[e * nsrc + ns] = (int32_t)at;
                        packed |= code[s] << (3 * ns);
                        ++ns;
                    }
                }
            }
            c[j] = cj;
            cod[e] = packed;
        }
    }
}

}  // namespace

// DepthList::recursiveDepth (iterator/depthIterator.cpp:7-45)
static void rec_depth(const Plan& p, const std::map<std::vector<int32_t>, int>& ids, int c, bool checkProl, int dd,
                      std::vector<int32_t>& T, std::vector<int32_t>& out) {
    int d = p.d;
    if (checkProl && dd > 0) {
        if (!((c >> dd) & 1)) {
            for (int t = 1; t <= p.maxdep[dd]; ++t) { T[dd] = t; rec_depth(p, ids, c, checkProl, dd - 1, T, out); }
        } else rec_depth(p, ids, c, checkProl, dd - 1, T, out);
    }
    if (checkProl && dd == 0) {
        if (!(c & 1)) {
            for (int t = 1; t <= p.maxdep[0]; ++t) { T[0] = t; rec_depth(p, ids, c, false, d - 1, T, out); }
        } else rec_depth(p, ids, c, false, d - 1, T, out);
    }
    if (!checkProl && dd >= 0) {
        if ((c >> dd) & 1) {
            for (int t = p.maxdep[dd]; t > 1; --t) { T[dd] = t; rec_depth(p, ids, c, checkProl, dd - 1, T, out); }
        } else rec_depth(p, ids, c, checkProl, dd - 1, T, out);
    }
    if (dd < 0) {
        auto it = ids.find(T);
        if (it != ids.end()) out.push_back(it->second);
    }
}

static std::map<std::vector<int32_t>, int> depth_ids(const Plan& p) {
    std::map<std::vector<int32_t>, int> ids;
    for (int t = 0; t < p.nD; ++t) ids[std::vector<int32_t>(p.D.begin() + t * p.d, p.D.begin() + (t + 1) * p.d)] = t;
    return ids;
}

std::vector<int32_t> sorted_depths(const Plan& p, int c) {
    auto ids = depth_ids(p);
    std::vector<int32_t> T(p.d, 0), out;
    rec_depth(p, ids, c, true, p.d - 1, T, out);
    return out;
}

bool build_plan(int d, int64_t n, const int32_t* points, const uint8_t* active, Plan& p) {
    auto t0 = std::chrono::steady_clock::now();
    if (d < 1 || d > kMaxDim || n < 1) { p.error = "dimension must be 1..8 and the grid non-empty"; return false; }
    p.d = d;
    p.n = n;
    p.pts.assign(points, points + n * d);
    p.act.assign(active, active + n);
    // ---- depths and depth list (first appearance, iterator/depthIterator.h:14-50)
    std::map<std::vector<int32_t>, int> ids;
    p.did.resize(n);
    std::vector<int32_t> Tk(d);
    for (int64_t k = 0; k < n; ++k) {
        for (int j = 0; j < d; ++j) {
            int32_t i = points[k * d + j];
            if (i < 2) { p.error = "boundary points (1D index 0 or 1) are not allowed in a Dirichlet grid"; return false; }
            if (depth1(i) > 30) { p.error = "depth too large"; return false; }
            Tk[j] = depth1(i);
        }
        auto it = ids.find(Tk);
        int t;
        if (it == ids.end()) {
            t = p.nD++;
            ids[Tk] = t;
            p.D.insert(p.D.end(), Tk.begin(), Tk.end());
        } else t = it->second;
        p.did[k] = t;
    }
    int nD = p.nD;
    p.maxdep.assign(d, 0);
    for (int t = 0; t < nD; ++t)
        for (int j = 0; j < d; ++j) p.maxdep[j] = std::max(p.maxdep[j], p.D[t * d + j]);
    p.ex_off.assign(nD + 1, 0);
    p.exa_off.assign(nD + 1, 0);
    for (int64_t k = 0; k < n; ++k) {
        p.ex_off[p.did[k] + 1]++;
        if (active[k]) p.exa_off[p.did[k] + 1]++;
    }
    for (int t = 0; t < nD; ++t) { p.ex_off[t + 1] += p.ex_off[t]; p.exa_off[t + 1] += p.exa_off[t]; }
    p.ex.resize(n);
    p.exa.resize(p.exa_off[nD]);
    {
        std::vector<int64_t> f(nD, 0), fa(nD, 0);
        for (int64_t k = 0; k < n; ++k) {
            int t = p.did[k];
            p.ex[p.ex_off[t] + f[t]++] = k;
            if (active[k]) p.exa[p.exa_off[t] + fa[t]++] = k;
        }
    }
    // duplicate points are invalid
    {
        std::vector<uint64_t> h(n);
        for (int64_t k = 0; k < n; ++k) {
            uint64_t x = 1469598103934665603ull;
            for (int j = 0; j < d; ++j) { x ^= (uint64_t)points[k * d + j]; x *= 1099511628211ull; }
            h[k] = x;
        }
        std::vector<int64_t> ord(n);
        std::iota(ord.begin(), ord.end(), 0);
        std::sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) {
            if (h[a] != h[b]) return h[a] < h[b];
            return std::lexicographical_compare(points + a * d, points + a * d + d, points + b * d, points + b * d + d);
        });
        for (int64_t k = 1; k < n; ++k)
            if (h[ord[k]] == h[ord[k - 1]] && std::equal(points + ord[k] * d, points + ord[k] * d + d, points + ord[k - 1] * d)) {
                p.error = "duplicate grid point";
                return false;
            }
    }
    // ---- slabs: points of depth <= T, ordered by level-T linear key
    p.slabs.resize(nD);
    std::vector<std::vector<uint64_t>> skeys(nD);
    std::vector<std::vector<int64_t>> spts(nD);
#pragma omp parallel for schedule(dynamic)
    for (int t = 0; t < nD; ++t) {
        const int32_t* T = &p.D[t * d];
        Geometry g(d, T);
        std::vector<std::pair<uint64_t, int64_t>> v;
        for (int u = 0; u < nD; ++u) {
            const int32_t* U = &p.D[u * d];
            bool le = true;
            for (int j = 0; j < d; ++j) le &= U[j] <= T[j];
            if (!le) continue;
            for (int64_t e = p.ex_off[u]; e < p.ex_off[u + 1]; ++e) {
                int64_t k = p.ex[e];
                int64_t c[kMaxDim];
                for (int j = 0; j < d; ++j) c[j] = coord_at(points[k * d + j], T[j]);
                v.emplace_back(g.key(c), k);
            }
        }
        std::sort(v.begin(), v.end());
        skeys[t].resize(v.size());
        spts[t].resize(v.size());
        for (size_t e = 0; e < v.size(); ++e) { skeys[t][e] = v[e].first; spts[t][e] = v[e].second; }
        Slab& s = p.slabs[t];
        std::copy(T, T + d, s.T);
        s.n = (int64_t)v.size();
        s.dense = (uint64_t)s.n == g.total();
    }
    p.M = 0;
    for (int t = 0; t < nD; ++t) { p.slabs[t].off = p.M; p.M += p.slabs[t].n; p.max_slab = std::max(p.max_slab, p.slabs[t].n); }
    p.slab_key.resize(p.M);
    p.slab_pt.resize(p.M);
    for (int t = 0; t < nD; ++t) {
        std::copy(skeys[t].begin(), skeys[t].end(), p.slab_key.begin() + p.slabs[t].off);
        std::copy(spts[t].begin(), spts[t].end(), p.slab_pt.begin() + p.slabs[t].off);
    }
    skeys.clear();
    spts.clear();
    // ---- cells of depth T+1 in the grid (cells/CellStructure.h:23-61)
    std::vector<std::vector<uint64_t>> ckeys(nD);
    std::vector<std::vector<int32_t>> ccorn(nD);
    int nc = 1 << d;
#pragma omp parallel for schedule(dynamic)
    for (int t = 0; t < nD; ++t) {
        Slab& s = p.slabs[t];
        Geometry g(d, s.T);
        if (s.dense) {
            uint64_t nc_all = 1;
            for (int j = 0; j < d; ++j) nc_all *= (uint64_t)g.cext[j];
            s.ncell = (int64_t)nc_all;
            continue;
        }
        std::vector<uint64_t> cand;
        cand.reserve(s.n * nc);
        int64_t c[kMaxDim], m[kMaxDim];
        for (int64_t e = 0; e < s.n; ++e) {
            g.decode(p.slab_key[s.off + e], c);
            for (int b = 0; b < nc; ++b) {
                uint64_t ck = 0;
                for (int j = 0; j < d; ++j) ck += (uint64_t)(c[j] - ((b >> j) & 1)) * g.cstride[j];
                cand.push_back(ck);
            }
        }
        sort_unique(cand);
        for (uint64_t ck : cand) {
            uint64_t r = ck;
            for (int j = 0; j < d; ++j) { m[j] = (int64_t)(r % (uint64_t)g.cext[j]); r /= (uint64_t)g.cext[j]; }
            int32_t corner[1 << kMaxDim];
            bool ok = true;
            for (int b = 0; b < nc && ok; ++b) {
                bool bnd = false;
                for (int j = 0; j < d; ++j) {
                    c[j] = m[j] + ((b >> j) & 1);
                    if (c[j] == 0 || c[j] == g.cext[j]) bnd = true;
                }
                if (bnd) { corner[b] = -1; continue; }
                int64_t at = find_key(p.slab_key.data() + s.off, s.n, g.key(c));
                if (at < 0) ok = false;
                else corner[b] = (int32_t)at;
            }
            if (!ok) continue;
            ckeys[t].push_back(ck);
            ccorn[t].insert(ccorn[t].end(), corner, corner + nc);
        }
        s.ncell = (int64_t)ckeys[t].size();
    }
    p.C = 0;
    int64_t ck_total = 0;
    for (int t = 0; t < nD; ++t) {
        Slab& s = p.slabs[t];
        s.cell_off = p.C;
        p.C += s.ncell;
        if (!s.dense) { s.corner_off = ck_total; ck_total += s.ncell; }
    }
    p.cell_key.resize(ck_total);
    p.cell_corner.resize(ck_total * nc);
    for (int t = 0; t < nD; ++t) {
        Slab& s = p.slabs[t];
        if (s.dense) continue;
        std::copy(ckeys[t].begin(), ckeys[t].end(), p.cell_key.begin() + s.corner_off);
        std::copy(ccorn[t].begin(), ccorn[t].end(), p.cell_corner.begin() + s.corner_off * nc);
    }
    ckeys.clear();
    ccorn.clear();
    // ---- tensor stencil transforms (calcNodal, MatrixVectorHomogen.cpp:43-74;
    //      ConvertToPrewavelet2, MatrixVectorHomogen.h:540-562)
    std::vector<StageOut> nod(nD), con(nD);
#pragma omp parallel for schedule(dynamic)
    for (int t = 0; t < nD; ++t) {
        Slab& s = p.slabs[t];
        Geometry g(d, s.T);
        std::vector<uint64_t> act_keys;
        for (int64_t e = p.exa_off[t]; e < p.exa_off[t + 1]; ++e) {
            int64_t k = p.exa[e];
            int64_t c[kMaxDim];
            for (int j = 0; j < d; ++j) c[j] = coord_at(points[k * d + j], s.T[j]);
            act_keys.push_back(g.key(c));
        }
        // active exact-depth points are stored in storage order; the transforms
        // use them sorted by key, so sort the list (exa) the same way
        std::vector<std::pair<uint64_t, int64_t>> kv;
        for (size_t e = 0; e < act_keys.size(); ++e) kv.emplace_back(act_keys[e], p.exa[p.exa_off[t] + e]);
        std::sort(kv.begin(), kv.end());
        for (size_t e = 0; e < kv.size(); ++e) { act_keys[e] = kv[e].first; p.exa[p.exa_off[t] + e] = kv[e].second; }
        std::vector<uint64_t> slab_keys(p.slab_key.begin() + s.off, p.slab_key.begin() + s.off + s.n);
        build_transform(g, act_keys, slab_keys, true, 3, nod[t]);
        build_transform(g, slab_keys, act_keys, false, 5, con[t]);
    }
    p.nodal.nsrc = 3;
    p.convert.nsrc = 5;
    p.nodal_dom.assign(nD * (d + 1), 0);
    p.convert_dom.assign(nD * (d + 1), 0);
    for (StageSet* ss : {&p.nodal, &p.convert}) {
        std::vector<StageOut>& so = ss == &p.nodal ? nod : con;
        std::vector<int64_t>& dom = ss == &p.nodal ? p.nodal_dom : p.convert_dom;
        ss->stage_off.assign(nD * d + 1, 0);
        int64_t tot = 0;
        for (int t = 0; t < nD; ++t) {
            for (int j = 0; j <= d; ++j) dom[t * (d + 1) + j] = (int64_t)so[t].dom[j].size();
            for (int j = 0; j < d; ++j) {
                ss->stage_off[t * d + j] = tot;
                tot += (int64_t)so[t].code[j].size();
            }
        }
        ss->stage_off[nD * d] = tot;
        ss->src.resize(tot * ss->nsrc);
        ss->code.resize(tot);
        for (int t = 0; t < nD; ++t)
            for (int j = 0; j < d; ++j) {
                int64_t o = ss->stage_off[t * d + j];
                std::copy(so[t].src[j].begin(), so[t].src[j].end(), ss->src.begin() + o * ss->nsrc);
                std::copy(so[t].code[j].begin(), so[t].code[j].end(), ss->code.begin() + o);
            }
    }
    nod.clear();
    con.clear();
    // ---- prolongation tables (MatrixVectorHomogen.h:444-474 + addMultiLevelValues)
    p.prol_tab.assign(nD * d, -1);
    {
        int64_t tot = 0;
        for (int t = 0; t < nD; ++t)
            for (int k = 0; k < d; ++k) {
                std::vector<int32_t> T(p.D.begin() + t * d, p.D.begin() + (t + 1) * d);
                T[k] += 1;
                auto it = ids.find(T);
                if (it == ids.end()) continue;
                p.prol_tab[t * d + k] = tot;
                tot += 2 * p.slabs[it->second].n;
            }
        p.prol.resize(tot);
#pragma omp parallel for schedule(dynamic)
        for (int tk = 0; tk < nD * d; ++tk) {
            if (p.prol_tab[tk] < 0) continue;
            int t = tk / d, k = tk % d;
            std::vector<int32_t> T(p.D.begin() + t * d, p.D.begin() + (t + 1) * d);
            Geometry gs(d, T.data());
            T[k] += 1;
            int tf = ids.at(T);
            Geometry gf(d, T.data());
            const Slab& sf = p.slabs[tf];
            int32_t* tab = &p.prol[p.prol_tab[tk]];
            int64_t c[kMaxDim];
            for (int64_t e = 0; e < sf.n; ++e) {
                gf.decode(p.slab_key[sf.off + e], c);
                int64_t ck = c[k];
                if (!(ck & 1)) {  // depth in dim k <= T_k: copy
                    c[k] = ck / 2;
                    int64_t at = slab_pos(p, t, gs, c);
                    tab[2 * e] = (int32_t)at;
                    tab[2 * e + 1] = -2;
                } else {          // new point: 0.5 (right + left)
                    int64_t top = gs.cext[k];
                    int64_t l = (ck - 1) / 2, r = (ck + 1) / 2;
                    c[k] = l;
                    tab[2 * e] = (l > 0 && l < top) ? (int32_t)slab_pos(p, t, gs, c) : -1;
                    c[k] = r;
                    tab[2 * e + 1] = (r > 0 && r < top) ? (int32_t)slab_pos(p, t, gs, c) : -1;
                }
            }
        }
    }
    // ---- per-case schedules
    p.ncase = 1 << d;
    p.sorted.resize(p.ncase);
    {
        std::vector<int32_t> T(d, 0);
        for (int c = 0; c < p.ncase; ++c) {
            std::vector<int32_t> out;
            std::fill(T.begin(), T.end(), 0);
            rec_depth(p, ids, c, true, d - 1, T, out);
            p.sorted[c] = out;
        }
    }
    p.p_slab_off.assign((size_t)p.ncase * nD, -1);
    p.gm_slab_off.assign((size_t)p.ncase * nD, -1);
    p.p_total = 0;
    p.gm_total = 0;
    std::map<std::tuple<int, int, int>, int64_t> restr_ids;  // (src, dst, dim) -> table offset
    std::vector<std::tuple<int, int, int, int64_t>> restr_list;
    int64_t restr_tot = 0;
    struct Pend { int c, t, s; };
    std::vector<std::vector<PhaseBItem>> blevels;
    std::vector<std::vector<std::vector<PhaseBStep>>> bsteps;
    int smax = 0;
    for (int t = 0; t < nD; ++t) {
        int s = 0;
        for (int j = 0; j < d; ++j) s += p.D[t * d + j];
        smax = std::max(smax, s);
    }
    blevels.assign(smax + 1, {});
    bsteps.assign(smax + 1, {});
    for (int c = 0; c < p.ncase; ++c) {
        for (int t : p.sorted[c]) {
            p.p_slab_off[(size_t)c * nD + t] = p.p_total;
            p.p_total += p.slabs[t].n;
        }
        auto gm_of = [&](int t) {
            int64_t& o = p.gm_slab_off[(size_t)c * nD + t];
            if (o < 0) { o = p.gm_total; p.gm_total += p.slabs[t].n; }
            return o;
        };
        for (int t : p.sorted[c]) {
            const int32_t* T = &p.D[t * d];
            int s = 0;
            for (int j = 0; j < d; ++j)
                if ((c >> j) & 1) s += T[j];
            PhaseBItem it{};
            it.c = c;
            it.t = t;
            it.p_off = p.p_slab_off[(size_t)c * nD + t];
            it.gm_off = gm_of(t);
            std::vector<PhaseBStep> steps;
            std::vector<int32_t> Tc(T, T + d);
            int cur = t;
            bool final_ok = true;
            for (int j = 0; j < d; ++j) {
                if (!((c >> j) & 1)) continue;
                Tc[j] -= 1;
                auto f = ids.find(Tc);
                if (f == ids.end()) { final_ok = false; continue; }
                final_ok = true;
                PhaseBStep st{};
                st.t_dst = f->second;
                st.dim = j;
                auto key = std::make_tuple(cur, f->second, j);
                auto rit = restr_ids.find(key);
                if (rit == restr_ids.end()) {
                    restr_ids[key] = restr_tot;
                    restr_list.emplace_back(cur, f->second, j, restr_tot);
                    st.tab_off = restr_tot;
                    restr_tot += 3 * p.slabs[f->second].n;
                } else st.tab_off = rit->second;
                st.n_src = p.slabs[cur].n;
                st.n_dst = p.slabs[f->second].n;
                st.gm_off = gm_of(f->second);
                steps.push_back(st);
                cur = f->second;
            }
            it.t_conv = final_ok ? cur : -1;
            if (it.t_conv >= 0 && !steps.empty() && cur != ids.at(Tc)) it.t_conv = -1;
            blevels[s].push_back(it);
            bsteps[s].push_back(steps);
        }
    }
    // restriction tables: z'[q] = z[self] + 0.5 z[q - h e_k] + 0.5 z[q + h e_k]
    p.restr.resize(restr_tot);
#pragma omp parallel for schedule(dynamic)
    for (size_t r = 0; r < restr_list.size(); ++r) {
        int ts, td, k;
        int64_t off;
        std::tie(ts, td, k, off) = restr_list[r];
        const Slab& ss = p.slabs[ts];
        const Slab& sd = p.slabs[td];
        Geometry gs(d, ss.T), gd(d, sd.T);
        int32_t* tab = &p.restr[off];
        int64_t c[kMaxDim], cs[kMaxDim];
        for (int64_t e = 0; e < sd.n; ++e) {
            gd.decode(p.slab_key[sd.off + e], c);
            for (int j = 0; j < d; ++j) cs[j] = c[j] << (ss.T[j] - sd.T[j]);
            tab[3 * e] = (int32_t)slab_pos(p, ts, gs, cs);
            // neighbours at level Tdst_k + 1 in dim k, expressed at the source level
            int sh = ss.T[k] - (sd.T[k] + 1);
            int64_t base = (2 * c[k]);
            int64_t top = gs.cext[k];
            int64_t lpos = (base - 1) << sh, rpos = (base + 1) << sh;
            cs[k] = lpos;
            tab[3 * e + 1] = (lpos > 0 && lpos < top) ? (int32_t)slab_pos(p, ts, gs, cs) : -1;
            cs[k] = rpos;
            tab[3 * e + 2] = (rpos > 0 && rpos < top) ? (int32_t)slab_pos(p, ts, gs, cs) : -1;
        }
    }
    // gM first-write flags, levels in descending restriction sum
    {
        std::vector<uint8_t> written((size_t)p.ncase * nD, 0);
        p.b_level_off.clear();
        int64_t scratch_max = 0;
        for (int s = smax; s >= 0; --s) {
            if (blevels[s].empty()) continue;
            p.b_level_off.push_back((int32_t)p.b_items.size());
            int64_t arena = 0;
            std::vector<std::pair<size_t, int>> writes;
            for (size_t i = 0; i < blevels[s].size(); ++i) {
                PhaseBItem it = blevels[s][i];
                it.gm_prev = written[(size_t)it.c * nD + it.t];
                it.step_begin = (int32_t)p.b_steps.size();
                int64_t scr = p.slabs[it.t].n;
                for (PhaseBStep st : bsteps[s][i]) {
                    st.gm_prev = written[(size_t)it.c * nD + st.t_dst];
                    writes.emplace_back((size_t)it.c * nD + st.t_dst, 1);
                    scr += st.n_dst;
                    p.b_steps.push_back(st);
                }
                it.step_end = (int32_t)p.b_steps.size();
                if (it.t_conv >= 0)
                    for (int j = 1; j < d; ++j) scr += p.convert_dom[it.t_conv * (d + 1) + j];
                it.scratch_off = arena;
                arena += scr;
                p.b_items.push_back(it);
            }
            for (auto& w : writes) written[w.first] = 1;
            scratch_max = std::max(scratch_max, arena);
        }
        p.b_level_off.push_back((int32_t)p.b_items.size());
        p.scratch_total = scratch_max;
    }
    // phase A: prolongation levels (dim k ascending, then T_k ascending)
    p.a_level_off.clear();
    for (int k = 0; k < d; ++k) {
        for (int tv = 1; tv <= p.maxdep[k]; ++tv) {
            size_t before = p.a_items.size();
            for (int c = 0; c < p.ncase; ++c) {
                if ((c >> k) & 1) continue;
                for (int t : p.sorted[c]) {
                    if (p.D[t * d + k] != tv) continue;
                    int64_t tab = p.prol_tab[t * d + k];
                    if (tab < 0) continue;
                    std::vector<int32_t> T(p.D.begin() + t * d, p.D.begin() + (t + 1) * d);
                    T[k] += 1;
                    int tf = ids.at(T);
                    PhaseAItem a{};
                    a.c = c;
                    a.t_src = t;
                    a.t_dst = tf;
                    a.dim = k;
                    a.src_off = p.p_slab_off[(size_t)c * nD + t];
                    a.dst_off = p.p_slab_off[(size_t)c * nD + tf];
                    a.n_dst = p.slabs[tf].n;
                    a.tab_off = tab;
                    p.a_items.push_back(a);
                }
            }
            if (p.a_items.size() > before) p.a_level_off.push_back((int32_t)before);
        }
    }
    p.a_level_off.push_back((int32_t)p.a_items.size());
    // nodal scratch: stage domains 1..d-1 of every depth
    p.nodal_scratch = 0;
    for (int t = 0; t < nD; ++t)
        for (int j = 1; j < d; ++j) p.nodal_scratch += p.nodal_dom[t * (d + 1) + j];
    p.inst_n_off = {0, n};
    p.inst_t_off = {0, nD};
    p.inst_c_off = {0, p.C};
    p.slab_inst.assign(nD, 0);
    p.plan_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return true;
}

namespace {
template <typename T>
void append_shift(std::vector<T>& dst, const std::vector<T>& src, T shift, bool keep_negative) {
    dst.reserve(dst.size() + src.size());
    for (T v : src) dst.push_back((keep_negative && v < 0) ? v : v + shift);
}

// scratch elements of one phase-B item (slab, restriction outputs, convert stages)
int64_t item_scratch(const Plan& p, const PhaseBItem& it) {
    int64_t scr = p.slabs[it.t].n;
    for (int32_t k = it.step_begin; k < it.step_end; ++k) scr += p.b_steps[k].n_dst;
    if (it.t_conv >= 0)
        for (int j = 1; j < p.d; ++j) scr += p.convert_dom[it.t_conv * (p.d + 1) + j];
    return scr;
}
}  // namespace

bool concat_plans(const std::vector<const Plan*>& parts, Plan& q) {
    if (parts.empty()) { q.error = "no plans to concatenate"; return false; }
    const int d = parts[0]->d;
    for (const Plan* p : parts)
        if (p->d != d) { q.error = "plans of different dimension"; return false; }
    q = Plan();
    q.d = d;
    q.ncase = 1 << d;
    q.maxdep.assign(d, 0);
    q.sorted.assign(q.ncase, {});
    q.inst_n_off.assign(1, 0);
    q.inst_t_off.assign(1, 0);
    q.inst_c_off.assign(1, 0);
    int64_t cornerb = 0, prolb = 0, restrb = 0, nsb = 0, csb = 0;
    std::vector<int64_t> pb, gmb, prolbv;
    std::vector<int32_t> stepb;
    for (size_t b = 0; b < parts.size(); ++b) {
        const Plan& p = *parts[b];
        const int64_t nb = q.n, Mb = q.M, Cb = q.C;
        const int32_t tb = q.nD;
        q.pts.insert(q.pts.end(), p.pts.begin(), p.pts.end());
        q.act.insert(q.act.end(), p.act.begin(), p.act.end());
        q.D.insert(q.D.end(), p.D.begin(), p.D.end());
        append_shift<int32_t>(q.did, p.did, tb, false);
        for (int j = 0; j < d; ++j) q.maxdep[j] = std::max(q.maxdep[j], p.maxdep[j]);
        // exact-depth lists: offsets arrays have nD+1 entries
        if (q.ex_off.empty()) { q.ex_off.push_back(0); q.exa_off.push_back(0); }
        for (int t = 1; t <= p.nD; ++t) {
            q.ex_off.push_back(p.ex_off[t] + (int64_t)q.ex.size());
            q.exa_off.push_back(p.exa_off[t] + (int64_t)q.exa.size());
        }
        append_shift<int64_t>(q.ex, p.ex, nb, false);
        append_shift<int64_t>(q.exa, p.exa, nb, false);
        // slabs and cells
        for (int t = 0; t < p.nD; ++t) {
            Slab s = p.slabs[t];
            s.off += Mb;
            s.cell_off += Cb;
            if (s.corner_off >= 0) s.corner_off += cornerb;
            q.slabs.push_back(s);
            q.slab_inst.push_back((int32_t)b);
        }
        append_shift<int64_t>(q.slab_pt, p.slab_pt, nb, false);
        q.slab_key.insert(q.slab_key.end(), p.slab_key.begin(), p.slab_key.end());
        q.cell_key.insert(q.cell_key.end(), p.cell_key.begin(), p.cell_key.end());
        q.cell_corner.insert(q.cell_corner.end(), p.cell_corner.begin(), p.cell_corner.end());
        cornerb += (int64_t)p.cell_key.size();
        // stencil stage tables: stage_off has nD*d+1 entries, sources are local
        for (int k = 0; k < p.nD * d; ++k) q.nodal.stage_off.push_back(p.nodal.stage_off[k] + nsb);
        for (int k = 0; k < p.nD * d; ++k) q.convert.stage_off.push_back(p.convert.stage_off[k] + csb);
        nsb += p.nodal.stage_off[p.nD * d];
        csb += p.convert.stage_off[p.nD * d];
        q.nodal.src.insert(q.nodal.src.end(), p.nodal.src.begin(), p.nodal.src.end());
        q.nodal.code.insert(q.nodal.code.end(), p.nodal.code.begin(), p.nodal.code.end());
        q.convert.src.insert(q.convert.src.end(), p.convert.src.begin(), p.convert.src.end());
        q.convert.code.insert(q.convert.code.end(), p.convert.code.begin(), p.convert.code.end());
        q.nodal_dom.insert(q.nodal_dom.end(), p.nodal_dom.begin(), p.nodal_dom.end());
        q.convert_dom.insert(q.convert_dom.end(), p.convert_dom.begin(), p.convert_dom.end());
        // prolongation / restriction tables (positions inside slabs are local)
        append_shift<int64_t>(q.prol_tab, p.prol_tab, prolb, true);
        q.prol.insert(q.prol.end(), p.prol.begin(), p.prol.end());
        q.restr.insert(q.restr.end(), p.restr.begin(), p.restr.end());
        for (int c = 0; c < q.ncase; ++c) append_shift<int32_t>(q.sorted[c], p.sorted[c], tb, false);
        pb.push_back(q.p_total);
        gmb.push_back(q.gm_total);
        prolbv.push_back(prolb);
        stepb.push_back((int32_t)q.b_steps.size());
        for (PhaseBStep st : p.b_steps) {
            st.t_dst += tb;
            st.tab_off += restrb;
            st.gm_off += q.gm_total;
            q.b_steps.push_back(st);
        }
        prolb += (int64_t)p.prol.size();
        restrb += (int64_t)p.restr.size();
        q.p_total += p.p_total;
        q.gm_total += p.gm_total;
        q.n += p.n;
        q.nD += p.nD;
        q.M += p.M;
        q.C += p.C;
        q.max_slab = std::max(q.max_slab, p.max_slab);
        q.nodal_scratch += p.nodal_scratch;
        q.plan_seconds += p.plan_seconds;
        q.inst_n_off.push_back(q.n);
        q.inst_t_off.push_back(q.nD);
        q.inst_c_off.push_back(q.C);
    }
    q.nodal.nsrc = 3;
    q.convert.nsrc = 5;
    q.nodal.stage_off.push_back(nsb);
    q.convert.stage_off.push_back(csb);
    // p_slab_off / gm_slab_off indexed (case, depth id) over the merged depth list
    q.p_slab_off.assign((size_t)q.ncase * q.nD, -1);
    q.gm_slab_off.assign((size_t)q.ncase * q.nD, -1);
    for (size_t b = 0; b < parts.size(); ++b) {
        const Plan& p = *parts[b];
        for (int c = 0; c < q.ncase; ++c)
            for (int t = 0; t < p.nD; ++t) {
                int64_t po = p.p_slab_off[(size_t)c * p.nD + t], go = p.gm_slab_off[(size_t)c * p.nD + t];
                size_t at = (size_t)c * q.nD + q.inst_t_off[b] + t;
                q.p_slab_off[at] = po < 0 ? -1 : po + pb[b];
                q.gm_slab_off[at] = go < 0 ? -1 : go + gmb[b];
            }
    }
    // phase A levels merged by index
    size_t la = 0;
    for (const Plan* p : parts) la = std::max(la, p->a_level_off.size() - 1);
    for (size_t L = 0; L < la; ++L) {
        q.a_level_off.push_back((int32_t)q.a_items.size());
        for (size_t b = 0; b < parts.size(); ++b) {
            const Plan& p = *parts[b];
            if (L + 1 >= p.a_level_off.size()) continue;
            for (int32_t i = p.a_level_off[L]; i < p.a_level_off[L + 1]; ++i) {
                PhaseAItem a = p.a_items[i];
                a.t_src += q.inst_t_off[b];
                a.t_dst += q.inst_t_off[b];
                a.src_off += pb[b];
                a.dst_off += pb[b];
                a.tab_off += prolbv[b];
                q.a_items.push_back(a);
            }
        }
    }
    q.a_level_off.push_back((int32_t)q.a_items.size());
    // phase B levels merged by index; scratch arenas laid out side by side
    size_t lb = 0;
    for (const Plan* p : parts) lb = std::max(lb, p->b_level_off.size() - 1);
    q.scratch_total = 0;
    for (size_t L = 0; L < lb; ++L) {
        q.b_level_off.push_back((int32_t)q.b_items.size());
        int64_t arena = 0;
        for (size_t b = 0; b < parts.size(); ++b) {
            const Plan& p = *parts[b];
            if (L + 1 >= p.b_level_off.size()) continue;
            for (int32_t i = p.b_level_off[L]; i < p.b_level_off[L + 1]; ++i) {
                PhaseBItem it = p.b_items[i];
                int64_t need = item_scratch(p, it);
                it.t += q.inst_t_off[b];
                if (it.t_conv >= 0) it.t_conv += q.inst_t_off[b];
                it.p_off += pb[b];
                it.gm_off += gmb[b];
                it.step_begin += stepb[b];
                it.step_end += stepb[b];
                it.scratch_off = arena;
                arena += need;
                q.b_items.push_back(it);
            }
        }
        q.scratch_total = std::max(q.scratch_total, arena);
    }
    q.b_level_off.push_back((int32_t)q.b_items.size());
    return true;
}


// ============================================================================= basis transforms
namespace {

inline int ctz64(int64_t v) { return __builtin_ctzll((unsigned long long)v); }

// LR decomposition without pivoting of a band matrix of half-bandwidth 2
// (sgoperation/matrix_operations.cc:34-60), same operation order; m holds the
// bands m[5k+0..4] = M[k][k-2..k+2] on entry.
void band_lr(int n, std::vector<double>& R, std::vector<double>& L) {
    auto at = [n](int i, int j) { return (size_t)i * 5 + (size_t)(j - i + 2); };
    L.assign((size_t)n * 5, 0.0);
    for (int i = 0; i < n; ++i) L[at(i, i)] = 1.0;
    for (int k = 0; k < n - 1; ++k)
        for (int i = k + 1; i < std::min(k + 3, n); ++i) {
            L[at(i, k)] = R[at(i, k)] / R[at(k, k)];
            for (int j = k; j < std::min(k + 3, n); ++j) R[at(i, j)] = R[at(i, j)] - L[at(i, k)] * R[at(k, j)];
        }
}

}  // namespace

std::vector<uint16_t> same_depth_neighbor_mask(const Plan& p) {
    const int d = p.d;
    std::vector<uint16_t> mask(p.n, 0);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < p.n; ++k) {
        const int t = p.did[k];
        const Slab& sl = p.slabs[t];
        Geometry g(d, sl.T);
        int64_t c[kMaxDim];
        for (int j = 0; j < d; ++j) c[j] = coord_at(p.pts[k * d + j], sl.T[j]);
        uint16_t m = 0;
        for (int j = 0; j < d; ++j) {
            const int64_t cj = c[j];
            if (cj - 2 >= 1) { c[j] = cj - 2; if (slab_pos(p, t, g, c) >= 0) m |= (uint16_t)(1u << (2 * j)); }
            if (cj + 2 < g.cext[j]) { c[j] = cj + 2; if (slab_pos(p, t, g, c) >= 0) m |= (uint16_t)(1u << (2 * j + 1)); }
            c[j] = cj;
        }
        mask[k] = m;
    }
    return mask;
}

bool build_basis_plan(const Plan& p, BasisPlan& b, std::string& error) {
    auto t0 = std::chrono::steady_clock::now();
    const int d = p.d, nD = p.nD;
    if (p.M >= ((int64_t)1 << 31) || p.n >= ((int64_t)1 << 29)) { error = "grid too large for the basis transforms"; return false; }
    b = BasisPlan();
    // ---- subgrid order: |T|_1 ascending, first appearance within equal norms
    b.order.resize(nD);
    for (int t = 0; t < nD; ++t) b.order[t] = t;
    auto l1 = [&](int t) { int s = 0; for (int j = 0; j < d; ++j) s += p.D[t * d + j]; return s; };
    std::stable_sort(b.order.begin(), b.order.end(), [&](int a, int c) { return l1(a) < l1(c); });
    // ---- nodal transform over all points of each depth
    b.ex_sorted.resize(p.ex.size());
    std::vector<StageOut> nod(nD);
#pragma omp parallel for schedule(dynamic)
    for (int t = 0; t < nD; ++t) {
        const Slab& sl = p.slabs[t];
        Geometry g(d, sl.T);
        std::vector<std::pair<uint64_t, int64_t>> kv;
        for (int64_t e = p.ex_off[t]; e < p.ex_off[t + 1]; ++e) {
            int64_t k = p.ex[e];
            int64_t c[kMaxDim];
            for (int j = 0; j < d; ++j) c[j] = coord_at(p.pts[k * d + j], sl.T[j]);
            kv.emplace_back(g.key(c), k);
        }
        std::sort(kv.begin(), kv.end());
        std::vector<uint64_t> keys(kv.size());
        for (size_t e = 0; e < kv.size(); ++e) { keys[e] = kv[e].first; b.ex_sorted[p.ex_off[t] + e] = kv[e].second; }
        std::vector<uint64_t> slab_keys(p.slab_key.begin() + sl.off, p.slab_key.begin() + sl.off + sl.n);
        build_transform(g, keys, slab_keys, true, 3, nod[t]);
    }
    b.nodal.nsrc = 3;
    b.nodal_dom.assign((size_t)nD * (d + 1), 0);
    b.nodal.stage_off.assign((size_t)nD * d + 1, 0);
    {
        int64_t tot = 0;
        for (int t = 0; t < nD; ++t) {
            for (int j = 0; j <= d; ++j) b.nodal_dom[t * (d + 1) + j] = (int64_t)nod[t].dom[j].size();
            for (int j = 0; j < d; ++j) { b.nodal.stage_off[t * d + j] = tot; tot += (int64_t)nod[t].code[j].size(); }
        }
        b.nodal.stage_off[nD * d] = tot;
        b.nodal.src.resize(tot * 3);
        b.nodal.code.resize(tot);
        for (int t = 0; t < nD; ++t)
            for (int j = 0; j < d; ++j) {
                int64_t o = b.nodal.stage_off[t * d + j];
                std::copy(nod[t].src[j].begin(), nod[t].src[j].end(), b.nodal.src.begin() + o * 3);
                std::copy(nod[t].code[j].begin(), nod[t].code[j].end(), b.nodal.code.begin() + o);
            }
    }
    nod.clear();
    // ---- slab hierarchization neighbours
    b.slab_nb.assign((size_t)p.M * d * 2, -1);
    b.slab_dep.assign((size_t)p.M * d, 0);
#pragma omp parallel for schedule(dynamic)
    for (int t = 0; t < nD; ++t) {
        const Slab& sl = p.slabs[t];
        Geometry g(d, sl.T);
        int64_t c[kMaxDim];
        for (int64_t e = 0; e < sl.n; ++e) {
            g.decode(p.slab_key[sl.off + e], c);
            for (int j = 0; j < d; ++j) {
                int own = sl.T[j] - ctz64(c[j]);
                b.slab_dep[(size_t)(sl.off + e) * d + j] = (uint8_t)own;
                int64_t step = (int64_t)1 << (sl.T[j] - own), cj = c[j];
                int32_t* nb = &b.slab_nb[((size_t)(sl.off + e) * d + j) * 2];
                if (cj - step > 0) {
                    c[j] = cj - step;
                    int64_t at = slab_pos(p, t, g, c);
                    nb[0] = at < 0 ? -1 : (int32_t)(sl.off + at);
                }
                if (cj + step < g.cext[j]) {
                    c[j] = cj + step;
                    int64_t at = slab_pos(p, t, g, c);
                    nb[1] = at < 0 ? -1 : (int32_t)(sl.off + at);
                }
                c[j] = cj;
            }
        }
    }
    // ---- point neighbours and per-(dim, depth) point lists
    b.pt_nb.assign((size_t)p.n * d * 2, -1);
    for (int j = 0; j < d; ++j) b.maxdep = std::max(b.maxdep, p.maxdep[j]);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < p.n; ++k) {
        int t = p.did[k];
        const Slab& sl = p.slabs[t];
        Geometry g(d, sl.T);
        int64_t c[kMaxDim];
        for (int j = 0; j < d; ++j) c[j] = coord_at(p.pts[k * d + j], sl.T[j]);  // odd: own level
        for (int j = 0; j < d; ++j) {
            int64_t cj = c[j];
            for (int side = 0; side < 2; ++side) {
                int64_t q = side ? cj + 1 : cj - 1;
                if (q <= 0 || q >= g.cext[j]) continue;
                c[j] = q;
                int64_t at = slab_pos(p, t, g, c);
                if (at >= 0) b.pt_nb[((size_t)k * d + j) * 2 + side] = (int32_t)p.slab_pt[sl.off + at];
            }
            c[j] = cj;
        }
    }
    {
        int nl = d * (b.maxdep + 1);
        b.lvl_off.assign(nl + 1, 0);
        // active points only: vector assignments of the reference touch active entries
        for (int64_t k = 0; k < p.n; ++k)
            if (p.act[k])
                for (int j = 0; j < d; ++j) b.lvl_off[j * (b.maxdep + 1) + p.D[p.did[k] * d + j] + 1]++;
        for (int i = 0; i < nl; ++i) b.lvl_off[i + 1] += b.lvl_off[i];
        b.lvl_pts.resize(b.lvl_off[nl]);
        std::vector<int64_t> fill(b.lvl_off.begin(), b.lvl_off.end() - 1);
        for (int64_t k = 0; k < p.n; ++k)
            if (p.act[k])
                for (int j = 0; j < d; ++j) b.lvl_pts[fill[j * (b.maxdep + 1) + p.D[p.did[k] * d + j]]++] = (int32_t)k;
    }
    // ---- calcPrewByNodal: components, bounding boxes and poles per depth, in
    // the reference's processing order (subgrids from the finest backwards,
    // BasisTransformations.cpp:486-545; SolvePrewavelet :468-484; components
    // sgrid/komponente.cpp; GetPrewaveletCoefficients :100-172; the pole matrix
    // sgoperation/matrix.cpp:76-150)
    std::vector<int32_t> mark(p.n, -1);
    for (int oi = nD - 1; oi >= 0; --oi) {
        const int t = b.order[oi];
        const Slab& sl = p.slabs[t];
        const int32_t* T = sl.T;
        Geometry g(d, T);
        b.step_t.push_back(t);
        b.step_group.push_back((int32_t)b.groups.size());
        auto lookup = [&](const int64_t* c) -> int64_t {  // storage index of level-T coords, -1 if none
            for (int j = 0; j < d; ++j)
                if (c[j] <= 0 || c[j] >= g.cext[j]) return -1;
            int64_t at = slab_pos(p, t, g, c);
            return at < 0 ? -1 : p.slab_pt[sl.off + at];
        };
        auto usable = [&](const int64_t* c) { int64_t k = lookup(c); return k >= 0 && p.act[k]; };
        for (int64_t e = p.ex_off[t]; e < p.ex_off[t + 1]; ++e) {
            int64_t seed = p.ex[e];
            if (!p.act[seed] || mark[seed] == t) continue;
            // component: depth-T points connected through their 5^d stencils
            int64_t mn[kMaxDim], mx[kMaxDim], c[kMaxDim], J[kMaxDim];
            for (int j = 0; j < d; ++j) mn[j] = mx[j] = coord_at(p.pts[seed * d + j], T[j]);
            std::vector<int64_t> stack{seed};
            mark[seed] = t;
            while (!stack.empty()) {
                int64_t k = stack.back();
                stack.pop_back();
                for (int j = 0; j < d; ++j) {
                    c[j] = coord_at(p.pts[k * d + j], T[j]);
                    mn[j] = std::min(mn[j], c[j]);
                    mx[j] = std::max(mx[j], c[j]);
                }
                // directions per dim: 0 centre, 1 left, 2 right, 3 left-left, 4 right-right
                int dir[kMaxDim] = {0};
                for (;;) {
                    bool ok = true;
                    for (int j = 0; j < d && ok; ++j) {
                        switch (dir[j]) {
                        case 0: J[j] = c[j]; break;
                        case 1: ok = c[j] - 1 > 0; J[j] = c[j] - 1; break;
                        case 2: ok = c[j] + 1 < g.cext[j]; J[j] = c[j] + 1; break;
                        case 3: ok = c[j] - 1 > 0; J[j] = c[j] - 2; break;
                        case 4: ok = c[j] + 1 < g.cext[j]; J[j] = c[j] + 2; break;
                        }
                    }
                    if (ok) {
                        int64_t q = lookup(J);
                        if (q >= 0 && p.act[q] && mark[q] != t) {
                            for (int j = 0; j < d; ++j) { mn[j] = std::min(mn[j], J[j]); mx[j] = std::max(mx[j], J[j]); }
                            if (p.did[q] == t) { mark[q] = t; stack.push_back(q); }
                        }
                    }
                    int j = 0;
                    while (j < d && ++dir[j] == 5) { dir[j] = 0; ++j; }
                    if (j == d) break;
                }
            }
            // per dimension: pole length and matrix from the box's minimum corner
            for (int dim = 0; dim < d; ++dim) {
                const int64_t top = g.cext[dim];
                int size = 1;
                {
                    int64_t w[kMaxDim];
                    std::copy(mn, mn + d, w);
                    while (w[dim] + 1 < top) {
                        w[dim] += 1;
                        if (!usable(w)) break;
                        ++size;
                    }
                }
                std::vector<double> R((size_t)size * 5, 0.0), L;
                auto setM = [&](int i, int j, double v) {  // M[i][j]; entries outside the matrix are dropped
                    if (i < 0 || i >= size || j < 0 || j >= size) return;
                    R[(size_t)i * 5 + (size_t)(j - i + 2)] = v;
                };
                {
                    int64_t w[kMaxDim];
                    std::copy(mn, mn + d, w);
                    int k = -1;
                    const int depth = T[dim];
                    while (w[dim] < top && usable(w)) {
                        ++k;
                        int64_t cp = w[dim];
                        int pd = T[dim] - ctz64(cp);  // depth of the position in dim
                        auto at = [&](int64_t off) { int64_t s2 = w[dim]; w[dim] = cp + off; bool u = w[dim] > 0 && w[dim] < top && usable(w); w[dim] = s2; return u; };
                        if (pd == depth) {
                            if (cp - 1 == 0) {
                                setM(k, k, 0.9);
                                if (pd == 1 && depth == 1) { setM(k, k, 1.0); break; }
                                if (at(1)) setM(k + 1, k, -0.6);
                                if (at(2)) setM(k + 2, k, 0.1);
                            } else if (cp + 1 == top) {
                                setM(k, k, 0.9);
                                if (at(-1)) setM(k - 1, k, -0.6);
                                if (at(-2)) setM(k - 2, k, 0.1);
                            } else {
                                setM(k, k, 1.0);
                                if (at(-1)) setM(k - 1, k, -0.6);
                                if (at(-2)) setM(k - 2, k, 0.1);
                                if (at(1)) setM(k + 1, k, -0.6);
                                if (at(2)) setM(k + 2, k, 0.1);
                            }
                        }
                        if (pd < depth) {
                            setM(k, k, 1.0);
                            if (at(-1)) setM(k - 1, k, 0.5);
                            if (at(1)) setM(k + 1, k, 0.5);
                        }
                        w[dim] += 1;
                    }
                }
                PoleGroup pg{};
                pg.t = t;
                pg.dim = dim;
                pg.size = size;
                pg.lu_off = (int64_t)b.lu.size();
                if (size >= 2) {
                    band_lr(size, R, L);
                    for (int k2 = 0; k2 < size; ++k2) {
                        b.lu.push_back(k2 + 1 < size ? L[(size_t)(k2 + 1) * 5 + 1] : 0.0);
                        b.lu.push_back(k2 + 2 < size ? L[(size_t)(k2 + 2) * 5 + 0] : 0.0);
                        b.lu.push_back(R[(size_t)k2 * 5 + 2]);
                        b.lu.push_back(k2 + 1 < size ? R[(size_t)k2 * 5 + 3] : 0.0);
                        b.lu.push_back(k2 + 2 < size ? R[(size_t)k2 * 5 + 4] : 0.0);
                    }
                } else {
                    b.lu.insert(b.lu.end(), {0.0, 0.0, R[2], 0.0, 0.0});
                }
                // poles: box positions with dim fixed at the minimum, dim 0 fastest
                pg.pos_off = (int64_t)b.pole_pos.size();
                int64_t w[kMaxDim];
                std::copy(mn, mn + d, w);
                int64_t np = 0;
                for (;;) {
                    int64_t q[kMaxDim];
                    std::copy(w, w + d, q);
                    for (int i = 0; i < size; ++i) {
                        q[dim] = mn[dim] + i;
                        int64_t k = lookup(q);
                        bool isT = true;
                        for (int j = 0; j < d; ++j) isT = isT && (q[j] & 1);
                        b.pole_pos.push_back(k < 0 ? -1 : (int32_t)(4 * k + (p.act[k] ? 2 : 0) + (isT ? 1 : 0)));
                    }
                    ++np;
                    int j = 0;
                    for (; j < d; ++j) {
                        if (j == dim) continue;
                        if (w[j] == mx[j]) { w[j] = mn[j]; continue; }
                        w[j] += 1;
                        break;
                    }
                    if (j == d) break;
                }
                pg.npoles = np;
                b.max_pole_elems = std::max(b.max_pole_elems, np * size);
                b.groups.push_back(pg);
            }
        }
    }
    b.step_group.push_back((int32_t)b.groups.size());
    b.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return true;
}

}  // namespace lsg
