// Planning of the factorised dense-slab cell operator (descriptors in lsg_sf.h)
// and its host emulation, which the CPU tests compare with the cell-by-cell
// form of LocalStiffnessMatrices::applyLocalMatrix
// (localStiffnessMatrices/LocalStiffnessMatrices.cpp:555-582).
#include "lsg_sf.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace lsg {

SfDiv sf_div(uint32_t d) {
    SfDiv r;
    r.d = d ? d : 1;
    uint32_t s = 0;
    while (((uint64_t)1 << s) < r.d) ++s;
    r.s = s;
    r.m = (uint32_t)((((uint64_t)1 << 32) * (((uint64_t)1 << s) - r.d)) / r.d + 1);
    return r;
}

static inline uint32_t sf_quot(const SfDiv& v, uint32_t q) {
    uint32_t t = (uint32_t)(((uint64_t)q * v.m) >> 32);
    return (t + q) >> v.s;
}

SfCoefLayout sf_coef_layout(const Plan& p) {
    SfCoefLayout L;
    L.coef_off.assign(p.nD, -1);
    for (int t = 0; t < p.nD; ++t) {
        const Slab& s = p.slabs[t];
        if (!s.dense) continue;
        int64_t c = 1;
        for (int k = 0; k < p.d; ++k)
            if (s.T[k] >= 2) c *= ((int64_t)1 << s.T[k]);
        L.coef_off[t] = L.ccount;
        L.ccount += c;
    }
    return L;
}

// per-dimension 1D factors of mode type 0 = P, 1 = M, 2 = B, 3 = I (virtual)
static inline void fac1(int T, int type, double& kap, double& mu) {
    if (type == 3) { kap = 0.0; mu = 1.0; return; }
    double h = std::ldexp(1.0, -T), ih = std::ldexp(1.0, T);
    if (type == 0) { kap = 0.0; mu = h / 4.0; }
    else if (type == 1) { kap = ih; mu = h / 12.0; }
    else { kap = ih; mu = h / 3.0; }
}

std::vector<SfSlab> sf_plan(const Plan& p, const SfCoefLayout& L, int64_t wcap, int na_max) {
    const int d = p.d;
    std::vector<SfSlab> out(p.nD);
    for (int t = 0; t < p.nD; ++t) {
        const Slab& s = p.slabs[t];
        SfSlab& D = out[t];
        D.na_max = na_max;
        if (!s.dense) { D.nm = D.nq = -1; continue; }
        D.coef_off = L.coef_off[t];
        // non-collapsed dimensions, inner to outer, with their position strides
        // (coefficient strides are set once the roles are known)
        std::vector<SfDim> nc;
        int64_t pst = 1;
        double S = 0.0, M = 1.0, unit = 1.0;
        for (int k = 0; k < d; ++k) {
            int32_t n = (1 << s.T[k]) - 1;
            if (n == 1) {  // one interior node: collapses into the coefficient (B factors)
                double kap, mu;
                fac1(s.T[k], 2, kap, mu);
                double S2 = S * mu + M * kap, M2 = M * mu;
                S = S2;
                M = M2;
                unit *= 2.0;
                continue;
            }
            SfDim x;
            x.n = n;
            x.pstride = (int32_t)pst;
            x.T = s.T[k];
            x.div2n = sf_div((uint32_t)(2 * n));
            nc.push_back(x);
            pst *= n;
        }
        D.S0 = S;
        D.M0 = M;
        D.unit_sum = unit;
        SfDim virt;
        virt.n = 1;
        virt.T = -1;
        // chunk set: every subset of the non-collapsed dimensions is a
        // candidate; keep the one whose plan fits with the lowest estimated
        // cost (stages and syncs per chunk, idle threads of the fused step)
        const int nn = (int)nc.size();
        double best = 1e300;
        unsigned best_set = 0;
        bool found = false;
        for (unsigned set = 0; set < (1u << nn); ++set) {
            std::vector<SfDim> rest;
            int64_t nch = 1;
            for (int i = 0; i < nn; ++i) {
                if ((set >> i) & 1) nch *= 2 * nc[i].n;
                else rest.push_back(nc[i]);
            }
            size_t pos = 0;
            int64_t na = 1, nb = 1;
            if (pos < rest.size() && rest[pos].n <= na_max) na = rest[pos++].n;
            if (pos < rest.size()) nb = rest[pos++].n;
            int m = (int)(rest.size() - pos);
            int64_t sl = na * nb, npl = 1;
            for (size_t i = pos; i < rest.size(); ++i) { sl *= rest[i].n; npl *= 2 * rest[i].n; }
            int64_t top = sl << m;
            int64_t w = m == 0 ? sl : top + top / 2;
            if (w > wcap || nch > (1 << 28)) continue;
            const double T = 256.0;
            double per = 2.0 * m + 4.0;                                          // stages (syncs)
            per += std::ceil(npl / T) * (double)nb * (double)na * 0.1;          // fused step, rows in series
            for (int k = 0; k <= m; ++k) per += std::ceil((double)(sl << k) / T) * 0.3;  // sweeps / gather / scatter
            double cost = (double)nch * per;
            if (cost < best) { best = cost; best_set = set; found = true; }
        }
        if (!found) { D.nm = D.nq = -1; continue; }  // a x b alone does not fit
        std::vector<SfDim> rest, chunks;
        for (int i = 0; i < nn; ++i) (((best_set >> i) & 1) ? chunks : rest).push_back(nc[i]);
        size_t pos = 0;
        if (pos < rest.size() && rest[pos].n <= na_max) D.a = rest[pos++];
        else D.a = virt;
        if (pos < rest.size()) D.b = rest[pos++];
        else D.b = virt;
        std::vector<SfDim> mids(rest.begin() + pos, rest.end());
        D.nm = (int32_t)mids.size();
        D.nq = (int32_t)chunks.size();
        for (int i = 0; i < D.nm; ++i) D.mid[i] = mids[i];
        for (int i = 0; i < D.nq; ++i) D.q[i] = chunks[i];
        const int64_t ab = (int64_t)D.a.n * D.b.n;
        int64_t sl = ab;
        for (const auto& x : mids) sl *= x.n;
        D.slice = (int32_t)sl;
        for (int i = 0; i < D.nq; ++i) {  // slice extent below each chunked dimension
            int64_t below = 1;
            for (const auto& x : rest)
                if (x.pstride < D.q[i].pstride) below *= x.n;
            D.qB[i] = sf_div((uint32_t)below);
            D.qmult[i] = (int32_t)(below * (D.q[i].n - 1));
        }
        D.nchunk = 1;
        for (const auto& x : chunks) D.nchunk *= 2 * x.n;
        D.npl = 1;
        for (const auto& x : mids) D.npl *= 2 * x.n;
        int64_t I = ab;
        for (int k = 0; k <= D.nm; ++k) D.stage[k] = (int32_t)(sl << k);
        for (int k = 0; k < D.nm; ++k) {
            D.inner[k] = sf_div((uint32_t)I);
            I *= 2 * D.mid[k].n;
        }
        D.hi_off = D.stage[D.nm];
        D.wtotal = D.nm == 0 ? D.stage[0] : D.stage[D.nm] + D.stage[D.nm - 1];
        // b segments of the fused step: as many as fill the CTA's 256 threads,
        // each of at least two b cells; the two parts of every row between
        // segments go to the idle ping-pong region (nm >= 1 only)
        D.nseg = 1;
        if (D.nm >= 1 && D.b.T >= 0 && D.a.n < 7) {  // the 7-node a path has no registers to spare
            const int64_t cells = (int64_t)D.b.n + 1;
            while ((int64_t)D.npl * D.nseg * 2 <= 256 && D.nseg * 2 * 2 <= cells &&
                   (int64_t)D.npl * (D.nseg * 2 - 1) * 2 * D.a.n <= D.stage[D.nm - 1])
                D.nseg *= 2;
        }
        // coefficient order of the slab: mid dimensions fastest, then a, b and
        // the chunked dimensions (n + 1 cells each)
        int32_t cs = 1;
        for (int i = 0; i < D.nm; ++i) { D.mid[i].cstride = cs; cs *= D.mid[i].n + 1; }
        if (D.a.T >= 0) { D.a.cstride = cs; cs *= D.a.n + 1; } else D.a.cstride = 0;
        if (D.b.T >= 0) { D.b.cstride = cs; cs *= D.b.n + 1; } else D.b.cstride = 0;
        for (int i = 0; i < D.nq; ++i) { D.q[i].cstride = cs; cs *= D.q[i].n + 1; }
    }
    return out;
}

void sf_cell_strides(const Plan& p, int t, const SfSlab& D, int32_t* by_dim) {
    const Slab& s = p.slabs[t];
    int64_t pst = 1;
    for (int k = 0; k < p.d; ++k) {
        by_dim[k] = 0;
        const int32_t n = (1 << s.T[k]) - 1;
        if (n == 1) continue;  // collapsed
        auto match = [&](const SfDim& x) {
            if (x.T >= 0 && x.pstride == pst) by_dim[k] = x.cstride;
        };
        match(D.a);
        match(D.b);
        for (int i = 0; i < D.nm; ++i) match(D.mid[i]);
        for (int i = 0; i < D.nq; ++i) match(D.q[i]);
        pst *= n;
    }
}

void sf_collapse_host(const Plan& p, int t, const SfSlab& D, const double* acell, double* coef) {
    const Slab& s = p.slabs[t];
    const int d = p.d;
    int64_t cstr[kMaxDim], ext[kMaxDim];
    int32_t ostr[kMaxDim];
    sf_cell_strides(p, t, D, ostr);
    int64_t st = 1;
    for (int k = 0; k < d; ++k) { cstr[k] = st; ext[k] = (int64_t)1 << s.T[k]; st *= ext[k]; }
    std::vector<int> ncd, cd;
    for (int k = 0; k < d; ++k) (s.T[k] >= 2 ? ncd : cd).push_back(k);
    int64_t cnt = 1;
    for (int k : ncd) cnt *= ext[k];
    for (int64_t c = 0; c < cnt; ++c) {
        int64_t r = c, base = 0, pos = 0;
        for (int k : ncd) {
            const int64_t ck = r % ext[k];
            base += ck * cstr[k];
            pos += ck * ostr[k];
            r /= ext[k];
        }
        double acc = 0.0;
        for (int b = 0; b < (1 << cd.size()); ++b) {  // collapsed cells in binary order
            int64_t key = base;
            for (size_t i = 0; i < cd.size(); ++i)
                if ((b >> i) & 1) key += cstr[cd[i]];
            acc += acell[key];
        }
        coef[pos] = acc;
    }
}

// ---------------------------------------------------------------- host emulation of k_sf
namespace {

// reduced-mode index r of a dimension with n nodes -> (cell, type)
inline void mode_of(int n, int r, int& cell, int& type) {
    cell = (r + 1) >> 1;
    type = (r == 0 || r == 2 * n - 1) ? 2 : ((r & 1) ? 0 : 1);
}

// nodes (1-based) and signs a reduced mode touches
inline int mode_nodes(int n, int r, int* j, double* sg) {
    if (r == 0) { j[0] = 1; sg[0] = 1.0; return 1; }
    if (r == 2 * n - 1) { j[0] = n; sg[0] = 1.0; return 1; }
    int c = (r + 1) >> 1;
    j[0] = c; sg[0] = 1.0;
    j[1] = c + 1; sg[1] = (r & 1) ? 1.0 : -1.0;
    return 2;
}

inline void combine(double& S, double& M, const SfDim& x, int type) {
    double kap, mu;
    fac1(x.T, x.T < 0 ? 3 : type, kap, mu);
    double S2 = S * mu + M * kap;
    M = M * mu;
    S = S2;
}

// forward 1D transform of n nodes (stride st) into 2n modes (stride st2)
inline void fwd1(const double* in, int64_t st, int n, double* out, int64_t st2) {
    out[0] = in[0];
    for (int j = 1; j < n; ++j) {
        out[(2 * j - 1) * st2] = in[(j - 1) * st] + in[j * st];
        out[(2 * j) * st2] = in[(j - 1) * st] - in[j * st];
    }
    out[(2 * n - 1) * st2] = in[(n - 1) * st];
}

// transposed 1D transform: 2n modes -> n nodes
inline void bwd1(const double* in, int64_t st2, int n, double* out, int64_t st) {
    for (int j = 1; j <= n; ++j) {
        double l = j == 1 ? in[0] : in[(2 * j - 3) * st2] - in[(2 * j - 2) * st2];
        double r = j == n ? in[(2 * n - 1) * st2] : in[(2 * j - 1) * st2] + in[(2 * j) * st2];
        out[(j - 1) * st] = l + r;
    }
}

}  // namespace

void sf_apply_host(const SfSlab& D, int form, const double* coef, const double* u, double* z) {
    const int nm = D.nm, nq = D.nq;
    std::vector<double> W(std::max(D.wtotal, 1));
    double* L = W.data();
    double* H = W.data() + D.hi_off;
    auto region = [&](int k) { return ((nm - k) & 1) ? H : L; };
    int64_t N = (int64_t)D.slice;
    for (int i = 0; i < nq; ++i) N *= D.q[i].n;
    if (nq > 0) std::fill(z, z + N, 0.0);
    const int na = D.a.n, nb = D.b.n;
    for (int ch = 0; ch < D.nchunk; ++ch) {
        // chunk tuple: per chunk dimension its reduced mode
        double cS = D.S0, cM = D.M0;
        int64_t cbase = 0;
        int64_t off[1 << kMaxDim];
        double sgn[1 << kMaxDim];
        int ncomb = 1;
        off[0] = 0;
        sgn[0] = 1.0;
        int rem = ch;
        for (int i = 0; i < nq; ++i) {
            const SfDim& x = D.q[i];
            int r = rem % (2 * x.n);
            rem /= 2 * x.n;
            int cell, type;
            mode_of(x.n, r, cell, type);
            combine(cS, cM, x, type);
            cbase += (int64_t)cell * x.cstride;
            int j[2];
            double sg[2];
            int k = mode_nodes(x.n, r, j, sg);
            int nn = ncomb;
            for (int c = 0; c < nn; ++c) {
                for (int e = k - 1; e >= 0; --e) {
                    int idx = e == 0 ? c : ncomb + c;
                    off[idx] = off[c] + (int64_t)(j[e] - 1) * x.pstride;
                    sgn[idx] = sgn[c] * sg[e];
                }
            }
            if (k == 2) ncomb *= 2;
        }
        auto upos = [&](int64_t e) {  // insert the chunked dimensions, outer to inner
            uint32_t x = (uint32_t)e;
            for (int i = nq - 1; i >= 0; --i) x += sf_quot(D.qB[i], x) * (uint32_t)D.qmult[i];
            return (int64_t)x;
        };
        // gather
        double* s0 = region(0);
        for (int64_t e = 0; e < D.slice; ++e) {
            double acc = 0.0;
            for (int c = 0; c < ncomb; ++c) acc += sgn[c] * u[off[c] + upos(e)];
            s0[e] = acc;
        }
        // mid forward sweeps
        for (int k = 0; k < nm; ++k) {
            const int n = D.mid[k].n;
            const int64_t I = D.inner[k].d, O = D.stage[k] / (I * n);
            const double* src = region(k);
            double* dst = region(k + 1);
            for (int64_t o = 0; o < O; ++o)
                for (int64_t i = 0; i < I; ++i) fwd1(src + i + I * n * o, I, n, dst + i + I * 2 * n * o, I);
        }
        // fused step (a, b) on every pencil plane
        double* F = region(nm);
        for (int pl = 0; pl < D.npl; ++pl) {
            double S = cS, M = cM;
            int64_t cb = cbase;
            int r = pl;
            for (int k = 0; k < nm; ++k) {
                const SfDim& x = D.mid[k];
                int rk = r % (2 * x.n);
                r /= 2 * x.n;
                int cell, type;
                mode_of(x.n, rk, cell, type);
                combine(S, M, x, type);
                cb += (int64_t)cell * x.cstride;
            }
            double* P = F + (int64_t)pl * na * nb;
            const int ma = D.a.T < 0 ? 1 : 2 * na, mb = D.b.T < 0 ? 1 : 2 * nb;
            // full a x b mode block (emulation: materialised)
            std::vector<double> Fa(ma * nb), G(ma * mb), Gb(ma * nb);
            for (int jb = 0; jb < nb; ++jb) {
                if (D.a.T < 0) Fa[jb * ma] = P[jb * na];
                else fwd1(P + jb * na, 1, na, Fa.data() + jb * ma, 1);
            }
            for (int ra = 0; ra < ma; ++ra) {
                if (D.b.T < 0) G[ra] = Fa[ra];
                else fwd1(Fa.data() + ra, ma, nb, G.data() + ra, ma);
            }
            for (int rb = 0; rb < mb; ++rb)
                for (int ra = 0; ra < ma; ++ra) {
                    int ca = 0, ta = 3, cbb = 0, tb = 3;
                    if (D.a.T >= 0) mode_of(na, ra, ca, ta);
                    if (D.b.T >= 0) mode_of(nb, rb, cbb, tb);
                    double S2 = S, M2 = M;
                    combine(S2, M2, D.a, ta);
                    combine(S2, M2, D.b, tb);
                    double lam = form == 1 ? M2 : S2;
                    double a = coef[cb + (int64_t)ca * D.a.cstride + (int64_t)cbb * D.b.cstride];
                    G[rb * ma + ra] *= a * lam;
                }
            for (int ra = 0; ra < ma; ++ra) {
                if (D.b.T < 0) Gb[ra] = G[ra];
                else bwd1(G.data() + ra, ma, nb, Gb.data() + ra, ma);
            }
            for (int jb = 0; jb < nb; ++jb) {
                if (D.a.T < 0) P[jb * na] = Gb[jb * ma];
                else bwd1(Gb.data() + jb * ma, 1, na, P + jb * na, 1);
            }
        }
        // mid backward sweeps
        for (int k = nm - 1; k >= 0; --k) {
            const int n = D.mid[k].n;
            const int64_t I = D.inner[k].d, O = D.stage[k] / (I * n);
            const double* src = region(k + 1);
            double* dst = region(k);
            for (int64_t o = 0; o < O; ++o)
                for (int64_t i = 0; i < I; ++i) bwd1(src + i + I * 2 * n * o, I, n, dst + i + I * n * o, I);
        }
        // scatter
        for (int64_t e = 0; e < D.slice; ++e)
            for (int c = 0; c < ncomb; ++c) {
                if (nq == 0) z[off[c] + e] = s0[e];
                else z[off[c] + upos(e)] += sgn[c] * s0[e];
            }
    }
}

// ---------------------------------------------------------------- direct cell loop
static double q1_entry(int form, int d, const double* h, unsigned pp, unsigned qq) {
    if (form == 1) {
        double prod = 1.0;
        for (int j = 0; j < d; ++j) prod *= (((pp >> j) & 1u) == ((qq >> j) & 1u)) ? h[j] / 3.0 : h[j] / 6.0;
        return prod;
    }
    double sum = 0.0;
    for (int i = 0; i < d; ++i) {
        double prod = 1.0;
        for (int j = 0; j < d; ++j) {
            bool same = ((pp >> j) & 1u) == ((qq >> j) & 1u);
            if (i == j) prod *= same ? 1.0 / h[j] : -1.0 / h[j];
            else prod *= same ? h[j] / 3.0 : h[j] / 6.0;
        }
        sum += prod;
    }
    return sum;
}

void cells_apply_host(const Plan& p, int t, int form, const double* acell, const double* u, double* z) {
    const Slab& s = p.slabs[t];
    const int d = p.d, nc = 1 << d;
    int64_t ext[kMaxDim], pstr[kMaxDim], cext[kMaxDim];
    double h[kMaxDim];
    int64_t st = 1;
    for (int k = 0; k < d; ++k) {
        ext[k] = ((int64_t)1 << s.T[k]) - 1;
        cext[k] = ext[k] + 1;
        pstr[k] = st;
        st *= ext[k];
        h[k] = std::ldexp(1.0, -s.T[k]);
    }
    std::vector<double> K((size_t)nc * nc);
    for (int a = 0; a < nc; ++a)
        for (int b = 0; b < nc; ++b) K[(size_t)a * nc + b] = q1_entry(form, d, h, a, b);
    std::fill(z, z + s.n, 0.0);
    std::vector<int64_t> pos(nc);
    for (int64_t c = 0; c < s.ncell; ++c) {
        int64_t m[kMaxDim], r = c;
        for (int k = 0; k < d; ++k) { m[k] = r % cext[k]; r /= cext[k]; }
        for (int b = 0; b < nc; ++b) {
            int64_t pp = 0;
            bool in = true;
            for (int k = 0; k < d && in; ++k) {
                int64_t j = m[k] + ((b >> k) & 1);
                if (j < 1 || j > ext[k]) in = false;
                else pp += (j - 1) * pstr[k];
            }
            pos[b] = in ? pp : -1;
        }
        for (int qq = 0; qq < nc; ++qq) {
            if (pos[qq] < 0) continue;
            double acc = 0.0;
            for (int pp = 0; pp < nc; ++pp)
                if (pos[pp] >= 0) acc += K[(size_t)qq * nc + pp] * u[pos[pp]];
            z[pos[qq]] += acell[c] * acc;
        }
    }
}

}  // namespace lsg
