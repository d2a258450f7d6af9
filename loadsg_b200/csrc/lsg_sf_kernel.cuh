// k_sf: the factorised level-T cell operator of a dense slab (see lsg_sf.h for
// the mathematics and the host emulation in lsg_sf.cpp that the CPU tests
// check against the cell-by-cell form).  One CTA per (case, slab) item:
//   chunk loop (reduced modes of the chunked dimensions, one tuple at a time)
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

// elements per thread in flight in the gather and scatter of a chunk
constexpr int kGS = 4;


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

// Pairs of values (the P and M mode of one a cell): packed f32x2 arithmetic in
// FP32 (Blackwell FADD2/FMUL2/FFMA2), two scalar operations in FP64.
template <typename V>
struct PairT;
template <>
struct PairT<float> { using T = float2; };
template <>
struct PairT<double> { using T = double2; };

__device__ __forceinline__ float2 mk2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mk2(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 psub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ double2 padd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 psub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 pmul(double2 a, double2 b) { return make_double2(a.x * b.x, a.y * b.y); }

// Reduced modes of the register dimension a with NX nodes: BL, the (P_i, M_i)
// pairs of the interior cells i = 1 .. NX-1, BR.
template <typename V, int NX>
struct ModesX {
    using V2 = typename PairT<V>::T;
    V bl, br;
    V2 pm[NX - 1];
};

template <typename V, int NX>
__device__ __forceinline__ void fwd_x(const V* X, ModesX<V, NX>& F) {
    F.bl = X[0];
    F.br = X[NX - 1];
#pragma unroll
    for (int i = 0; i < NX - 1; ++i) F.pm[i] = mk2(X[i] + X[i + 1], X[i] - X[i + 1]);
}

template <typename V, int NX>
__device__ __forceinline__ void bwd_x(const ModesX<V, NX>& G, V* Y) {
    V l = G.bl;
#pragma unroll
    for (int j = 0; j < NX - 1; ++j) {
        Y[j] = l + (G.pm[j].x + G.pm[j].y);
        l = G.pm[j].x - G.pm[j].y;
    }
    Y[NX - 1] = l + G.br;
}

// The fused (a, b) step of one pencil plane P (a fastest, rows of NX values,
// nb rows), in place, for an a dimension of exactly NX nodes (NX = 1: no a
// dimension), over the b cells [c0, c1) of the cells 0 .. nb (cell 0 and nb:
// the boundary cells; cell c: rows c - 1 and c).  (S, M): pair of every other
// dimension; cf: coefficient of the plane's cell in the other dimensions (a and
// b cell 0).  Rows with both cells in the range are written in place.  With
// c0 > 0, row c0 - 1 gets only cell c0's part: it goes to bnd[-NX .. -1] (value
// space); with c1 <= nb, row c1 - 1 gets only cell c1 - 1's part: it goes to
// bnd[0 .. NX-1].  The whole plane (c0 = 0, c1 = nb + 1) has neither.
template <typename V, int NX>
__device__ __forceinline__ void fused_plane(V* P, const lsg::SfSlab& D, V S, V M, const V* cf, bool unit, V unit_v,
                                            int form, int c0, int c1, V* bnd) {
    using V2 = typename PairT<V>::T;
    const int nb = D.b.n;
    const bool bvirt = D.b.T < 0;
    const int64_t csa = D.a.cstride, csb = D.b.cstride;
    // a factors by a type (P, M, B), folded with (S, M); no a dimension: identity
    V SAt[3], MAt[3];
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        V kap, mu;
        fac<V>(NX == 1 ? -1 : D.a.T, t, kap, mu);
        SAt[t] = S * mu + M * kap;
        MAt[t] = M * mu;
    }
    // Lambda(a type, b type) for the b type tb
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
    V X[NX], Y[NX], c[NX + 1];
    auto coefs = [&](int mb_cell) {
        const V* q = cf + mb_cell * csb;
#pragma unroll
        for (int i = 0; i <= NX; ++i)
            if (NX > 1 || i == 0) c[i] = unit ? unit_v : q[i * csa];
    };
    auto load = [&](int row) {
#pragma unroll
        for (int i = 0; i < NX; ++i) X[i] = P[row * NX + i];
    };
    auto store = [&](int row) {
#pragma unroll
        for (int i = 0; i < NX; ++i) P[row * NX + i] = Y[i];
    };
    const int ce = c1 < nb ? c1 : nb;  // interior cells [cs, ce)
    if constexpr (NX == 1) {
        // one value per row: the b stream alone
        V lP, lM, lB;
        if (bvirt) {
            coefs(0);
            lam(3, lP, lM, lB);
            P[0] = c[0] * lB * P[0];
            return;
        }
        V pP, pM, pB, mP, mM, mB;
        lam(0, pP, pM, pB);
        lam(1, mP, mM, mB);
        lam(2, lP, lM, lB);
        V fp, acc;
        int cs;
        if (c0 == 0) {  // left boundary cell: row 0 only
            fp = P[0];
            coefs(0);
            acc = c[0] * lB * fp;
            cs = 1;
        } else {        // row c0 - 1: this segment's part starts empty
            fp = P[c0 - 1];
            acc = V(0);
            cs = c0;
        }
        auto cell = [&](int jb) {
            V f = P[jb];
            coefs(jb);
            V gp = c[0] * pB * (fp + f), gm = c[0] * mB * (fp - f);
            V o = acc + gp + gm;
            acc = gp - gm;
            fp = f;
            return o;
        };
        if (c0 > 0) bnd[-1] = cell(cs++);
        for (int jb = cs; jb < ce; ++jb) P[jb - 1] = cell(jb);
        if (c1 > nb) {  // right boundary cell nb: row nb-1 only
            coefs(nb);
            P[nb - 1] = acc + c[0] * lB * fp;
        } else {
            bnd[0] = acc;
        }
    } else {
        ModesX<V, NX> Fp{}, acc{};
        V lP, lM, lB;
        if (bvirt) {
            ModesX<V, NX> Fc;
            load(0);
            fwd_x<V, NX>(X, Fc);
            coefs(0);
            lam(3, lP, lM, lB);  // virtual b: identity factors
            acc.bl = c[0] * lB * Fc.bl;
            acc.br = c[NX] * lB * Fc.br;
#pragma unroll
            for (int i = 0; i < NX - 1; ++i) acc.pm[i] = mk2(c[i + 1] * lP * Fc.pm[i].x, c[i + 1] * lM * Fc.pm[i].y);
            bwd_x<V, NX>(acc, Y);
            store(0);
            return;
        }
        V pP, pM, pB, mP, mM, mB;  // Lambda of the interior b cells: b type P (p..) and M (m..)
        lam(0, pP, pM, pB);
        lam(1, mP, mM, mB);
        lam(2, lP, lM, lB);        // ... and of the boundary b cells
        const V2 lp2 = mk2(pP, pM), lm2 = mk2(mP, mM);
        // interior b cell jb between rows jb-1 and jb: per a mode, b modes
        // P = Fp + Fc, M = Fp - Fc, scaled; row jb-1 gets P' + M' (complete, into
        // Y), row jb starts with P' - M'
        auto cell = [&](int jb) {
            load(jb);
            coefs(jb);
            ModesX<V, NX> Fc, out;
            fwd_x<V, NX>(X, Fc);
            {
                V gp = c[0] * pB * (Fp.bl + Fc.bl), gm = c[0] * mB * (Fp.bl - Fc.bl);
                out.bl = acc.bl + gp + gm;
                acc.bl = gp - gm;
                gp = c[NX] * pB * (Fp.br + Fc.br);
                gm = c[NX] * mB * (Fp.br - Fc.br);
                out.br = acc.br + gp + gm;
                acc.br = gp - gm;
            }
#pragma unroll
            for (int i = 0; i < NX - 1; ++i) {
                const V2 cc = mk2(c[i + 1], c[i + 1]);
                const V2 gp = pmul(pmul(cc, lp2), padd(Fp.pm[i], Fc.pm[i]));
                const V2 gm = pmul(pmul(cc, lm2), psub(Fp.pm[i], Fc.pm[i]));
                out.pm[i] = padd(padd(acc.pm[i], gp), gm);
                acc.pm[i] = psub(gp, gm);
            }
            Fp = Fc;
            bwd_x<V, NX>(out, Y);
        };
        int cs;
        if (c0 == 0) {
            load(0);
            fwd_x<V, NX>(X, Fp);
            coefs(0);  // left boundary b cell: row 0 only
            acc.bl = c[0] * lB * Fp.bl;
            acc.br = c[NX] * lB * Fp.br;
#pragma unroll
            for (int i = 0; i < NX - 1; ++i) acc.pm[i] = mk2(c[i + 1] * lP * Fp.pm[i].x, c[i + 1] * lM * Fp.pm[i].y);
            cs = 1;
        } else {  // row c0 - 1: this segment's part starts empty and goes to bnd[-NX ..]
            load(c0 - 1);
            fwd_x<V, NX>(X, Fp);
            acc.bl = V(0);
            acc.br = V(0);
#pragma unroll
            for (int i = 0; i < NX - 1; ++i) acc.pm[i] = mk2(V(0), V(0));
            cell(c0);
#pragma unroll
            for (int i = 0; i < NX; ++i) bnd[i - NX] = Y[i];
            cs = c0 + 1;
        }
        for (int jb = cs; jb < ce; ++jb) {
            cell(jb);
            store(jb - 1);
        }
        if (c1 > nb) {
            coefs(nb);  // right boundary b cell nb: row nb-1 only
            acc.bl += c[0] * lB * Fp.bl;
            acc.br += c[NX] * lB * Fp.br;
#pragma unroll
            for (int i = 0; i < NX - 1; ++i)
                acc.pm[i] = padd(acc.pm[i], mk2(c[i + 1] * lP * Fp.pm[i].x, c[i + 1] * lM * Fp.pm[i].y));
            bwd_x<V, NX>(acc, Y);
            store(nb - 1);
        } else {
            bwd_x<V, NX>(acc, Y);
#pragma unroll
            for (int i = 0; i < NX; ++i) bnd[i] = Y[i];
        }
    }
}

}  // namespace lsg_sfk

// One CTA per dense (case, slab) item.  sf: per-slab plans of this precision;
// coef: collapsed coefficients (or unit: the slab's 2^#collapsed).
template <typename V, int NA>
__global__ void __launch_bounds__(256, (sizeof(V) == 4 ? 3 : 2)) k_sf(const lsg::PhaseBItem* __restrict__ items, const lsg::SfSlab* __restrict__ sf,
                                            const V* __restrict__ pc, V* __restrict__ zb, const V* __restrict__ coef,
                                            const int32_t* __restrict__ order, int32_t ord0, int unit, int form) {
    using namespace lsg_sfk;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(16) unsigned char draw[sizeof(lsg::SfSlab)];
    __shared__ int s_ncomb[2];
    __shared__ V s_cS[2], s_cM[2];
    __shared__ int64_t s_cbase[2];
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
    // the signed blocks (2^nq of them) of this chunk and the next one, after the
    // work space: offsets of buffer 0 and 1, then signs of buffer 0 and 1
    const int ncmax = 1 << nq;
    int64_t* s_off0 = reinterpret_cast<int64_t*>(smem_raw + lsg::sf_comb_offset(D, sizeof(V)));
    V* s_sgn0 = reinterpret_cast<V*>(s_off0 + 2 * ncmax);
    auto region = [&](int k) { return ((nm - k) & 1) ? Wh : Wl; };
    const int tid = threadIdx.x, T = blockDim.x;
    // chunk tuple -> signed blocks, (S, M) and coefficient offset, into buffer bf
    // (one thread)
    auto combos = [&](int ch, int bf) {
        int64_t* so = s_off0 + bf * ncmax;
        V* sg = s_sgn0 + bf * ncmax;
        V cS = V(D.S0), cM = V(D.M0);
        int64_t cbase = 0;
        int ncomb = 1;
        so[0] = 0;
        sg[0] = V(1);
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
                for (int c = 0; c < ncomb; ++c) so[c] += (int64_t)(j - 1) * x.pstride;
            } else {
                V sv = type == 0 ? V(1) : V(-1);
                for (int c = 0; c < ncomb; ++c) {
                    so[ncomb + c] = so[c] + (int64_t)cell * x.pstride;  // node cell + 1
                    sg[ncomb + c] = sg[c] * sv;
                    so[c] += (int64_t)(cell - 1) * x.pstride;           // node cell
                }
                ncomb *= 2;
            }
        }
        s_ncomb[bf] = ncomb;
        s_cS[bf] = cS;
        s_cM[bf] = cM;
        s_cbase[bf] = cbase;
    };
    if (nq > 0) {
        int64_t N = D.slice;
        for (int i = 0; i < nq; ++i) N *= D.q[i].n;
        for (int64_t e = tid; e < N; e += T) z[e] = V(0);
    }
    if (tid == T - 1) combos(0, 0);
    __syncthreads();
    for (int ch = 0; ch < D.nchunk; ++ch) {
        const int bf = ch & 1;
        const int ncomb = s_ncomb[bf];
        const int64_t* s_off = s_off0 + bf * ncmax;
        const V* s_sgn = s_sgn0 + bf * ncmax;
        // slice position -> u position: insert the chunked dimensions, outer to inner
        auto upos = [&](uint32_t x) {
            for (int i = nq - 1; i >= 0; --i) x += quot(D.qB[i], x) * (uint32_t)D.qmult[i];
            return (int64_t)x;
        };
        // gather the slice of u for this chunk tuple into stage 0: kGS elements
        // per thread, all their loads issued before the sums
        {
            V* s0 = region(0);
            for (int e0 = tid; e0 < D.slice; e0 += kGS * T) {
                int64_t ue[kGS];
                V acc[kGS];
#pragma unroll
                for (int k = 0; k < kGS; ++k) {
                    const int e = e0 + k * T;
                    ue[k] = e < D.slice ? upos((uint32_t)e) : -1;
                    acc[k] = V(0);
                }
                for (int c = 0; c < ncomb; ++c) {
                    const V sg = s_sgn[c];
                    const V* uc = u + s_off[c];
                    V x[kGS];
#pragma unroll
                    for (int k = 0; k < kGS; ++k) x[k] = ue[k] >= 0 ? uc[ue[k]] : V(0);
#pragma unroll
                    for (int k = 0; k < kGS; ++k) acc[k] += sg * x[k];
                }
#pragma unroll
                for (int k = 0; k < kGS; ++k)
                    if (ue[k] >= 0) s0[e0 + k * T] = acc[k];
            }
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
                int j = 1;
                if constexpr (sizeof(V) == 8) {  // FP64: four loads in flight before the stores
                    for (; j + 3 < n; j += 4) {
                        const V x0 = in[(size_t)j * I], x1 = in[(size_t)(j + 1) * I];
                        const V x2 = in[(size_t)(j + 2) * I], x3 = in[(size_t)(j + 3) * I];
                        out[(size_t)(2 * j - 1) * I] = xp + x0;
                        out[(size_t)(2 * j) * I] = xp - x0;
                        out[(size_t)(2 * j + 1) * I] = x0 + x1;
                        out[(size_t)(2 * j + 2) * I] = x0 - x1;
                        out[(size_t)(2 * j + 3) * I] = x1 + x2;
                        out[(size_t)(2 * j + 4) * I] = x1 - x2;
                        out[(size_t)(2 * j + 5) * I] = x2 + x3;
                        out[(size_t)(2 * j + 6) * I] = x2 - x3;
                        xp = x3;
                    }
                }
                for (; j < n; ++j) {
                    V x = in[(size_t)j * I];
                    out[(size_t)(2 * j - 1) * I] = xp + x;
                    out[(size_t)(2 * j) * I] = xp - x;
                    xp = x;
                }
                out[(size_t)(2 * n - 1) * I] = xp;
            }
            __syncthreads();
        }
        // fused (a, b) step on every pencil plane; with G > 1 segments per
        // plane, each row between two segments is completed after a barrier
        // from the two parts the segments left in the idle ping-pong region:
        // the left segment's, then the right segment's
        {
            V* F = region(nm);
            const int plane = D.a.n * D.b.n, na = D.a.n;
            // FP64 only: the FP32 kernel (80 registers for three CTAs per SM) has none to spare
            const int G = (sizeof(V) == 8 && D.nseg > 1 && D.npl * D.nseg <= T) ? D.nseg : 1;
            const int lg = 31 - __clz(G);
            const int L = (D.b.n + 1) >> lg;  // b cells per segment (nb + 1 = 2^T_b when G > 1)
            V* Wr = region(nm > 0 ? nm - 1 : 0);  // per boundary row: [left part | right part]
            for (int w = tid; w < D.npl * G; w += T) {
                const int pl = w >> lg, sg = w & (G - 1);
                V S = s_cS[bf], M = s_cM[bf];
                int64_t cb = s_cbase[bf];
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
                V* Pp = F + (size_t)pl * plane;
                const int c0 = sg * L, c1 = G == 1 ? D.b.n + 1 : c0 + L;
                // boundary row sg (after this segment): [this segment's part | the next one's]
                V* bnd = Wr + (size_t)2 * na * ((size_t)pl * (G - 1) + sg);
                if (D.a.T < 0) fused_plane<V, 1>(Pp, D, S, M, cf0 + cb, unit != 0, unit_v, form, c0, c1, bnd);
                else if (NA >= 7 && D.a.n == 7)  // never segmented (register budget)
                    fused_plane<V, (NA >= 7 ? 7 : 3)>(Pp, D, S, M, cf0 + cb, unit != 0, unit_v, form, 0, D.b.n + 1, bnd);
                else fused_plane<V, 3>(Pp, D, S, M, cf0 + cb, unit != 0, unit_v, form, c0, c1, bnd);
            }
            __syncthreads();
            if (G > 1) {
                const int g1 = G - 1 > 0 ? G - 1 : 1;  // boundary rows per plane
                const int nbr = D.npl * g1 * na;       // boundary-row values
                for (int e = tid; e < nbr; e += T) {
                    const int i = e % na, rowid = e / na;  // rowid = pl * (G - 1) + (sg - 1)
                    const int pl = rowid / g1, sg = rowid - pl * g1 + 1;
                    const V* part = Wr + (size_t)2 * na * rowid;
                    F[(size_t)pl * plane + (size_t)(sg * L - 1) * na + i] = part[i] + part[na + i];
                }
                __syncthreads();
            }
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
                int j = 1;
                if constexpr (sizeof(V) == 8) {  // FP64: eight loads in flight before the stores
                    for (; j + 3 < n; j += 4) {
                        V pp[4], mm[4];
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            pp[u] = in[(size_t)(2 * (j + u) - 1) * I];
                            mm[u] = in[(size_t)(2 * (j + u)) * I];
                        }
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            out[(size_t)(j + u - 1) * I] = l + (pp[u] + mm[u]);
                            l = pp[u] - mm[u];
                        }
                    }
                }
                for (; j < n; ++j) {
                    V pp = in[(size_t)(2 * j - 1) * I], mm = in[(size_t)(2 * j) * I];
                    out[(size_t)(j - 1) * I] = l + (pp + mm);
                    l = pp - mm;
                }
                out[(size_t)(n - 1) * I] = l + in[(size_t)(2 * n - 1) * I];
            }
            __syncthreads();
        }
        // scatter stage 0 into z (its transpose of the gather), kGS elements per
        // thread: per signed block all loads of z before the stores
        {
            const V* s0 = region(0);
            for (int e0 = tid; e0 < D.slice; e0 += kGS * T) {
                int64_t ue[kGS];
                V v[kGS];
#pragma unroll
                for (int k = 0; k < kGS; ++k) {
                    const int e = e0 + k * T;
                    ue[k] = e < D.slice ? upos((uint32_t)e) : -1;
                    v[k] = ue[k] >= 0 ? s0[e] : V(0);
                }
                if (nq == 0) {
#pragma unroll
                    for (int k = 0; k < kGS; ++k)
                        if (ue[k] >= 0) z[ue[k]] = v[k];
                } else {
                    for (int c = 0; c < ncomb; ++c) {
                        const V sg = s_sgn[c];
                        V* zc = z + s_off[c];
                        V old[kGS];
#pragma unroll
                        for (int k = 0; k < kGS; ++k) old[k] = ue[k] >= 0 ? zc[ue[k]] : V(0);
#pragma unroll
                        for (int k = 0; k < kGS; ++k)
                            if (ue[k] >= 0) zc[ue[k]] = old[k] + sg * v[k];
                    }
                }
            }
        }
        // the next chunk's signed blocks into the other buffer (its last reader,
        // chunk ch - 1, finished before the previous barrier)
        if (tid == T - 1 && ch + 1 < D.nchunk) combos(ch + 1, bf ^ 1);
        __syncthreads();
    }
}

// Collapsed coefficients of every dense slab: per non-collapsed cell the sum of
// a over the collapsed dimensions' cells in binary order (FP64, rounded once
// for FP32), for the collapsed cells [lo, hi) enumerated in slab-dimension
// order; coll_slab: slab of each collapsed cell, coll_off: first collapsed cell
// of each slab; str64 / str32: per (slab, dim) the coefficient stride of the
// FP64 / FP32 plan, which place the value in that plan's order.
__global__ void k_sf_collapse(const int32_t* __restrict__ slab_T, int d, const int64_t* __restrict__ cell_off,
                              const int64_t* __restrict__ coll_off, const int32_t* __restrict__ coll_slab, int64_t lo,
                              int64_t hi, const double* __restrict__ acell, const int32_t* __restrict__ str64,
                              const int32_t* __restrict__ str32, double* __restrict__ c64, float* __restrict__ c32) {
    int64_t gi = lo + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (gi >= hi) return;
    const int t = coll_slab[gi];
    const int32_t* T = slab_T + (size_t)t * d;
    const int32_t* s64 = str64 + (size_t)t * d;
    const int32_t* s32 = str32 + (size_t)t * d;
    int64_t r = gi - coll_off[t], base = 0, st = 1, p64 = 0, p32 = 0;
    int ncd = 0;
    int64_t cstr[lsg::kMaxDim];
    for (int k = 0; k < d; ++k) {
        int64_t ext = (int64_t)1 << T[k];
        if (T[k] >= 2) {
            const int64_t ck = r % ext;
            base += ck * st;
            p64 += ck * s64[k];
            p32 += ck * s32[k];
            r /= ext;
        } else cstr[ncd++] = st;
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
    c64[coll_off[t] + p64] = acc;
    c32[coll_off[t] + p32] = (float)acc;
}
