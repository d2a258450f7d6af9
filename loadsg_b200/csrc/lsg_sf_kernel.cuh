// k_sf: the factorised level-T cell operator of a dense slab (see lsg_sf.h for
// the mathematics and the host emulation in lsg_sf.cpp that the CPU tests
// check against the cell-by-cell form).  One CTA per (case, slab) item:
//   chunk loop (reduced modes of the outermost dimensions, one tuple at a time)
//     gather   W0 = signed sum of <= 2^nq strided blocks of u
//     sweeps   W(k+1) = E_k W(k) for the mid dimensions (shared memory, ping-pong)
//     fused    per pencil plane: E_a and E_b, a~ * Lambda, E_b^T and E_a^T in
//              registers, streaming along b (in place)
//     sweeps   W(k) = E_k^T W(k+1)
//     scatter  z (+)= signed W0 into the same blocks
// No atomics: each stage writes every element from one thread, stages are
// separated by __syncthreads, and chunks add into z in a fixed order.
#pragma once
#include "lsg_sf.h"

namespace lsg_sfk {

constexpr int kMaxComb = 64;  // 2^nq signed blocks of one chunk (nq <= 6)

template <typename V>
__device__ __forceinline__ V pow2(int e);
template <>
__device__ __forceinline__ float pow2<float>(int e) { return __int_as_float((127 + e) << 23); }
template <>
__device__ __forceinline__ double pow2<double>(int e) { return __longlong_as_double((long long)(1023 + e) << 52); }

// 1D factors of mode type 0 = P, 1 = M, 2 = B; T < 0 is a virtual dimension
template <typename V>
__device__ __forceinline__ void fac(int T, int type, V& kap, V& mu) {
    if (T < 0) { kap = V(0); mu = V(1); return; }
    const V h = pow2<V>(-T);
    if (type == 0) { kap = V(0); mu = h * V(0.25); }
    else if (type == 1) { kap = pow2<V>(T); mu = h * V(1.0 / 12.0); }
    else { kap = pow2<V>(T); mu = h * V(1.0 / 3.0); }
}

template <typename V>
__device__ __forceinline__ void combine(V& S, V& M, int T, int type) {
    V kap, mu;
    fac<V>(T, type, kap, mu);
    V S2 = S * mu + M * kap;
    M = M * mu;
    S = S2;
}

__device__ __forceinline__ uint32_t quot(const lsg::SfDiv& v, uint32_t q) { return (__umulhi(q, v.m) + q) >> v.s; }

__device__ __forceinline__ void mode_of(int n, int r, int& cell, int& type) {
    cell = (r + 1) >> 1;
    type = (r == 0 || r == 2 * n - 1) ? 2 : ((r & 1) ? 0 : 1);
}

// reduced modes of the register dimension a: BL, P_i, M_i (i < NA-1), BR
template <typename V, int NA>
struct Modes {
    V bl, br;
    V p[NA - 1], m[NA - 1];
};

template <typename V, int NA>
__device__ __forceinline__ void fwd_a(const V* X, int na, bool virt, Modes<V, NA>& F) {
    F.bl = X[0];
    F.br = V(0);
#pragma unroll
    for (int i = 0; i < NA - 1; ++i) {
        bool ok = !virt && i < na - 1;
        F.p[i] = ok ? X[i] + X[i + 1] : V(0);
        F.m[i] = ok ? X[i] - X[i + 1] : V(0);
    }
#pragma unroll
    for (int i = 0; i < NA; ++i)
        if (!virt && i == na - 1) F.br = X[i];
}

template <typename V, int NA>
__device__ __forceinline__ void bwd_a(const Modes<V, NA>& G, int na, bool virt, V* Y) {
    if (virt) { Y[0] = G.bl; return; }
#pragma unroll
    for (int j = 0; j < NA; ++j) {
        V l = j == 0 ? G.bl : G.p[j > 0 ? j - 1 : 0] - G.m[j > 0 ? j - 1 : 0];
        V r = j < NA - 1 ? G.p[j < NA - 1 ? j : 0] + G.m[j < NA - 1 ? j : 0] : V(0);
        if (j == na - 1) r = G.br;
        Y[j] = l + r;
    }
}

// G = coefficient(cell of each a mode) * Lambda(a type, b type) * F
template <typename V, int NA>
__device__ __forceinline__ void scale_a(const Modes<V, NA>& F, const V* c, int na, V lP, V lM, V lB,
                                        Modes<V, NA>& G) {
    G.bl = c[0] * lB * F.bl;
#pragma unroll
    for (int i = 0; i < NA - 1; ++i) {
        G.p[i] = c[i + 1] * lP * F.p[i];
        G.m[i] = c[i + 1] * lM * F.m[i];
    }
    V cbr = c[0];
#pragma unroll
    for (int i = 1; i <= NA; ++i)
        if (i == na) cbr = c[i];
    G.br = cbr * lB * F.br;
}

template <typename V, int NA>
__device__ __forceinline__ void add_modes(Modes<V, NA>& A, const Modes<V, NA>& B, V s) {
    A.bl += s * B.bl;
    A.br += s * B.br;
#pragma unroll
    for (int i = 0; i < NA - 1; ++i) { A.p[i] += s * B.p[i]; A.m[i] += s * B.m[i]; }
}

// The fused (a, b) step of one pencil plane P (a fastest, rows of na values,
// nb rows), in place.  (S, M): pair of every other dimension; cf: coefficient
// of the plane's cell in the other dimensions (a and b cell 0).
template <typename V, int NA>
__device__ __forceinline__ void fused_plane(V* P, const lsg::SfSlab& D, V S, V M, const V* cf, bool unit, V unit_v,
                                            int form) {
    const int na = D.a.n, nb = D.b.n;
    const bool avirt = D.a.T < 0, bvirt = D.b.T < 0;
    const int csa = D.a.cstride, csb = D.b.cstride;
    // a factors by a type, folded with (S, M)
    V SAt[3], MAt[3];
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        V kap, mu;
        fac<V>(D.a.T, t, kap, mu);
        SAt[t] = S * mu + M * kap;
        MAt[t] = M * mu;
    }
    auto lam = [&](int tb, V& lP, V& lM, V& lB) {
        V kb, mb;
        fac<V>(D.b.T, tb, kb, mb);
        if (form == 1) {
            lP = MAt[0] * mb; lM = MAt[1] * mb; lB = MAt[2] * mb;
        } else {
            lP = SAt[0] * mb + MAt[0] * kb;
            lM = SAt[1] * mb + MAt[1] * kb;
            lB = SAt[2] * mb + MAt[2] * kb;
        }
    };
    auto coefs = [&](int mb_cell, V* c) {
        const V* q = cf + (int64_t)mb_cell * csb;
#pragma unroll
        for (int i = 0; i <= NA; ++i) c[i] = (i <= na && (i == 0 || !avirt)) ? (unit ? unit_v : q[(int64_t)i * csa]) : V(0);
    };
    V X[NA], Y[NA], c[NA + 1];
    auto load = [&](int row) {
#pragma unroll
        for (int i = 0; i < NA; ++i) X[i] = i < na ? P[row * na + i] : V(0);
    };
    auto store = [&](int row) {
#pragma unroll
        for (int i = 0; i < NA; ++i)
            if (i < na) P[row * na + i] = Y[i];
    };
    Modes<V, NA> Fp, Fc, acc;
    V lP, lM, lB;
    if (bvirt) {
        load(0);
        fwd_a<V, NA>(X, na, avirt, Fc);
        coefs(0, c);
        lam(3, lP, lM, lB);  // virtual b: identity factors
        scale_a<V, NA>(Fc, c, na, lP, lM, lB, acc);
        bwd_a<V, NA>(acc, na, avirt, Y);
        store(0);
        return;
    }
    load(0);
    fwd_a<V, NA>(X, na, avirt, Fp);
    coefs(0, c);
    lam(2, lP, lM, lB);
    scale_a<V, NA>(Fp, c, na, lP, lM, lB, acc);  // left boundary cell of b: row 0 only
    V pP, pM, pB, mP, mM, mB;  // Lambda(a type, b type) of the interior b cells
    lam(0, pP, pM, pB);
    lam(1, mP, mM, mB);
    for (int jb = 1; jb < nb; ++jb) {
        load(jb);
        fwd_a<V, NA>(X, na, avirt, Fc);
        coefs(jb, c);  // interior b cell jb between rows jb-1 and jb
        // per a mode: b modes P = Fp + Fc, M = Fp - Fc, scaled; row jb-1 gets
        // P' + M' (complete), row jb starts with P' - M'
        auto step = [&](V& ac, V& fp, V f, V cc, V lp, V lm) {
            V gp = cc * lp * (fp + f), gm = cc * lm * (fp - f);
            V done = ac + gp + gm;
            ac = gp - gm;
            fp = f;
            return done;
        };
        Modes<V, NA> out;
        out.bl = step(acc.bl, Fp.bl, Fc.bl, c[0], pB, mB);
#pragma unroll
        for (int i = 0; i < NA - 1; ++i) {
            out.p[i] = step(acc.p[i], Fp.p[i], Fc.p[i], c[i + 1], pP, mP);
            out.m[i] = step(acc.m[i], Fp.m[i], Fc.m[i], c[i + 1], pM, mM);
        }
        V cbr = c[0];
#pragma unroll
        for (int i = 1; i <= NA; ++i)
            if (i == na) cbr = c[i];
        out.br = step(acc.br, Fp.br, Fc.br, cbr, pB, mB);
        bwd_a<V, NA>(out, na, avirt, Y);
        store(jb - 1);
    }
    coefs(nb, c);  // right boundary cell of b: row nb-1 only
    lam(2, lP, lM, lB);
    scale_a<V, NA>(Fp, c, na, lP, lM, lB, Fc);
    add_modes<V, NA>(acc, Fc, V(1));
    bwd_a<V, NA>(acc, na, avirt, Y);
    store(nb - 1);
}

}  // namespace lsg_sfk

// One CTA per dense (case, slab) item.  sf: per-slab plans of this precision;
// coef: collapsed coefficients (or unit: the slab's 2^#collapsed).
template <typename V, int NA>
__global__ void __launch_bounds__(256) k_sf(const lsg::PhaseBItem* __restrict__ items, const lsg::SfSlab* __restrict__ sf,
                                            const V* __restrict__ pc, V* __restrict__ zb, const V* __restrict__ coef,
                                            const int32_t* __restrict__ order, int32_t ord0, int unit, int form) {
    using namespace lsg_sfk;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(16) unsigned char draw[sizeof(lsg::SfSlab)];
    __shared__ int64_t s_off[kMaxComb];
    __shared__ V s_sgn[kMaxComb];
    __shared__ int s_ncomb;
    __shared__ V s_cS, s_cM;
    __shared__ int64_t s_cbase;
    const lsg::PhaseBItem it = items[order[ord0 + blockIdx.x]];
    {
        const int* src = reinterpret_cast<const int*>(sf + it.t);
        int* dst = reinterpret_cast<int*>(draw);
        for (int i = threadIdx.x; i < (int)(sizeof(lsg::SfSlab) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const lsg::SfSlab& D = *reinterpret_cast<const lsg::SfSlab*>(draw);
    const V* u = pc + it.p_off;
    V* z = zb + it.p_off;
    const V* cf0 = coef + D.coef_off;
    const V unit_v = V(D.unit_sum);
    V* Wl = reinterpret_cast<V*>(smem_raw);
    V* Wh = Wl + D.hi_off;
    const int nm = D.nm, nq = D.nq;
    auto region = [&](int k) { return ((nm - k) & 1) ? Wh : Wl; };
    const int tid = threadIdx.x, T = blockDim.x;
    if (nq > 0) {
        int64_t N = D.slice;
        for (int i = 0; i < nq; ++i) N *= D.q[i].n;
        for (int64_t e = tid; e < N; e += T) z[e] = V(0);
    }
    for (int ch = 0; ch < D.nchunk; ++ch) {
        if (tid == 0) {  // chunk tuple -> signed blocks, (S, M) and coefficient offset
            V cS = V(D.S0), cM = V(D.M0);
            int64_t cbase = 0;
            int ncomb = 1;
            s_off[0] = 0;
            s_sgn[0] = V(1);
            int rem = ch;
            for (int i = 0; i < nq; ++i) {
                const lsg::SfDim& x = D.q[i];
                int r = rem % (2 * x.n);
                rem /= 2 * x.n;
                int cell, type;
                mode_of(x.n, r, cell, type);
                combine<V>(cS, cM, x.T, type);
                cbase += (int64_t)cell * x.cstride;
                if (type == 2) {
                    int j = r == 0 ? 1 : x.n;
                    for (int c = 0; c < ncomb; ++c) s_off[c] += (int64_t)(j - 1) * x.pstride;
                } else {
                    V sg = type == 0 ? V(1) : V(-1);
                    for (int c = 0; c < ncomb; ++c) {
                        s_off[ncomb + c] = s_off[c] + (int64_t)cell * x.pstride;  // node cell + 1
                        s_sgn[ncomb + c] = s_sgn[c] * sg;
                        s_off[c] += (int64_t)(cell - 1) * x.pstride;              // node cell
                    }
                    ncomb *= 2;
                }
            }
            s_ncomb = ncomb;
            s_cS = cS;
            s_cM = cM;
            s_cbase = cbase;
        }
        __syncthreads();
        const int ncomb = s_ncomb;
        // slice position -> u position: insert the chunked dimensions, outer to inner
        auto upos = [&](uint32_t x) {
            for (int i = nq - 1; i >= 0; --i) x += quot(D.qB[i], x) * (uint32_t)D.qmult[i];
            return (int64_t)x;
        };
        // gather
        V* s0 = region(0);
        for (int e = tid; e < D.slice; e += T) {
            const int64_t ue = upos((uint32_t)e);
            V acc = V(0);
            for (int c = 0; c < ncomb; ++c) acc += s_sgn[c] * u[s_off[c] + ue];
            s0[e] = acc;
        }
        __syncthreads();
        // mid sweeps, forward
        for (int k = 0; k < nm; ++k) {
            const int n = D.mid[k].n;
            const uint32_t I = D.inner[k].d;
            const uint32_t cnt = (uint32_t)D.stage[k] / (uint32_t)n;
            const V* src = region(k);
            V* dst = region(k + 1);
            for (uint32_t p = tid; p < cnt; p += T) {
                uint32_t o = quot(D.inner[k], p), i = p - o * I;
                const V* in = src + i + (size_t)I * n * o;
                V* out = dst + i + (size_t)I * 2 * n * o;
                V xp = in[0];
                out[0] = xp;
                for (int j = 1; j < n; ++j) {
                    V x = in[(size_t)j * I];
                    out[(size_t)(2 * j - 1) * I] = xp + x;
                    out[(size_t)(2 * j) * I] = xp - x;
                    xp = x;
                }
                out[(size_t)(2 * n - 1) * I] = xp;
            }
            __syncthreads();
        }
        // fused (a, b) step on every pencil plane
        {
            V* F = region(nm);
            const int plane = D.a.n * D.b.n;
            for (int pl = tid; pl < D.npl; pl += T) {
                V S = s_cS, M = s_cM;
                int64_t cb = s_cbase;
                uint32_t r = (uint32_t)pl;
                for (int k = 0; k < nm; ++k) {
                    const lsg::SfDim& x = D.mid[k];
                    uint32_t q2 = quot(x.div2n, r);
                    int rk = (int)(r - q2 * (uint32_t)(2 * x.n));
                    r = q2;
                    int cell, type;
                    mode_of(x.n, rk, cell, type);
                    combine<V>(S, M, x.T, type);
                    cb += (int64_t)cell * x.cstride;
                }
                fused_plane<V, NA>(F + (size_t)pl * plane, D, S, M, cf0 + cb, unit != 0, unit_v, form);
            }
            __syncthreads();
        }
        // mid sweeps, transposed
        for (int k = nm - 1; k >= 0; --k) {
            const int n = D.mid[k].n;
            const uint32_t I = D.inner[k].d;
            const uint32_t cnt = (uint32_t)D.stage[k] / (uint32_t)n;
            const V* src = region(k + 1);
            V* dst = region(k);
            for (uint32_t p = tid; p < cnt; p += T) {
                uint32_t o = quot(D.inner[k], p), i = p - o * I;
                const V* in = src + i + (size_t)I * 2 * n * o;
                V* out = dst + i + (size_t)I * n * o;
                V l = in[0];
                for (int j = 1; j < n; ++j) {
                    V pp = in[(size_t)(2 * j - 1) * I], mm = in[(size_t)(2 * j) * I];
                    out[(size_t)(j - 1) * I] = l + (pp + mm);
                    l = pp - mm;
                }
                out[(size_t)(n - 1) * I] = l + in[(size_t)(2 * n - 1) * I];
            }
            __syncthreads();
        }
        // scatter
        for (int e = tid; e < D.slice; e += T) {
            V v = s0[e];
            if (nq == 0) z[e] = v;
            else {
                const int64_t ue = upos((uint32_t)e);
                for (int c = 0; c < ncomb; ++c) z[s_off[c] + ue] += s_sgn[c] * v;
            }
        }
        __syncthreads();
    }
}

// Collapsed coefficients of every dense slab: per non-collapsed cell the sum of
// a over the collapsed dimensions' cells in binary order (FP64, rounded once
// for FP32), for the collapsed cells [lo, hi); coll_slab: slab of each
// collapsed cell, coll_off: first collapsed cell of each slab.
__global__ void k_sf_collapse(const int32_t* __restrict__ slab_T, int d, const int64_t* __restrict__ cell_off,
                              const int64_t* __restrict__ coll_off, const int32_t* __restrict__ coll_slab, int64_t lo,
                              int64_t hi, const double* __restrict__ acell, double* __restrict__ c64,
                              float* __restrict__ c32) {
    int64_t gi = lo + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (gi >= hi) return;
    const int t = coll_slab[gi];
    const int32_t* T = slab_T + (size_t)t * d;
    int64_t r = gi - coll_off[t], base = 0, st = 1;
    int ncd = 0;
    int64_t cstr[lsg::kMaxDim];
    for (int k = 0; k < d; ++k) {
        int64_t ext = (int64_t)1 << T[k];
        if (T[k] >= 2) { base += (r % ext) * st; r /= ext; }
        else cstr[ncd++] = st;
        st *= ext;
    }
    const double* a = acell + cell_off[t];
    double acc = 0.0;
    for (int b = 0; b < (1 << ncd); ++b) {
        int64_t key = base;
        for (int i = 0; i < ncd; ++i)
            if ((b >> i) & 1) key += cstr[i];
        acc += a[key];
    }
    c64[gi] = acc;
    c32[gi] = (float)acc;
}
