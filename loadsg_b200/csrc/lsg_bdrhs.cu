// Boundary-data right-hand sides on the device (MatrixVectorMultiplication/
// RHS.h:278-427 and RHS.cpp, paths relative to LoAdSG's library/source/).
//
// A problem -div(grad u) + c u = f with u = g on the boundary is reduced to
// zero boundary values; its right-hand side needs the products of the interior
// prewavelets with the boundary data.  g is given on a second grid that holds
// boundary points (a 1D index 0 or 1 in some dimension; completeNeumannGrid of
// the interior grid), as hierarchical coefficients of its boundary points
// (CalcHierarchicalBasisForRHS, RHS.cpp:6-41).
//
//   lsg_hierarchize_boundary   CalcHierarchicalBasisForRHS: per dimension, the
//       boundary points lose half the sum of their two 1D parents, finest depth
//       first; one launch per (dimension, depth) over host-built
//       (point, left, right) lists.
//   lsg_boundary_rhs           InHomoBoundaryRHSHierarchical::multiply,
//       multiply_mass, multiply_mass_coeff (RHS.cpp:697-1008): for every depth
//       T of the interior grid and every point J of depth <= T the level-T hat
//       of J is integrated against every hierarchical boundary hat (closed
//       forms of RHS.cpp:43-695, gradients / values / values weighted by
//       prod (1 - x_k^2)), and ConvertToPrewavelet2 (RHS.h:397-420) combines
//       these nodal values into the prewavelet entries of the points of depth T.
//
// Only the (J, T) pairs that some 5^d stencil reads are evaluated: the host
// builds the stencil of every active point once per operator (entries and CSR
// rows).  k_bd_nodal gives every entry one warp; the lanes test 32 boundary
// points at a time for overlapping supports (most pairs do not overlap and
// contribute an exact zero), evaluate the ones that do, and the partial
// products are added in the reference's order (depth list of the boundary
// grid, then storage order) by shuffles, so the sums are the reference's to
// the bit.  The integrals use the reference's antiderivative forms with every
// product and sum rounded on its own (no contraction into FMAs).
#include "lsg_internal.h"
#include "../../include/lsg.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

using lsg_internal::fail_msg;

#define BD_TRY(expr)                                                                                    \
    do {                                                                                                \
        cudaError_t _e = (expr);                                                                        \
        if (_e != cudaSuccess)                                                                          \
            return fail_msg(LSG_E_CUDA, (std::string(#expr) + ": " + cudaGetErrorString(_e)).c_str());  \
    } while (0)

struct DevArr {
    void* p = nullptr;
    size_t bytes = 0;
    DevArr() = default;
    DevArr(const DevArr&) = delete;
    DevArr& operator=(const DevArr&) = delete;
    DevArr(DevArr&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    ~DevArr() { if (p) cudaFree(p); }
    int alloc(size_t b) {
        if (p) { cudaFree(p); p = nullptr; }
        bytes = b;
        if (!b) return 0;
        cudaError_t e = cudaMalloc(&p, b);
        return e == cudaSuccess ? 0 : fail_msg(LSG_E_CUDA, (std::string("cudaMalloc: ") + cudaGetErrorString(e)).c_str());
    }
    template <typename T>
    int upload(const std::vector<T>& v, cudaStream_t st) {
        int rc = alloc(v.size() * sizeof(T));
        if (rc || v.empty()) return rc;
        cudaError_t e = cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st);
        return e == cudaSuccess ? 0 : fail_msg(LSG_E_CUDA, cudaGetErrorString(e));
    }
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

// ------------------------------------------------------------------ host index algebra
// indices/index.h:656-871: root 2, sons 2i and 2i+1, boundary indices 0 and 1
inline int h_depth1(int32_t i) { return i < 2 ? 0 : 31 - __builtin_clz((unsigned)i); }
inline int32_t h_left1(int32_t i) { return i >> (__builtin_ctz((unsigned)i) + 1); }
inline int32_t h_right1(int32_t i) { return i >> (__builtin_ctz(~(unsigned)i) + 1); }
inline int32_t h_left_lv(int32_t i, int level) {  // index.h:834-847
    int lv = level - h_depth1(i);
    if (lv == 0) return h_left1(i);
    i <<= 1;
    for (int k = 1; k < lv; ++k) i = (i << 1) + 1;
    return i;
}
inline int32_t h_right_lv(int32_t i, int level) {  // index.h:855-866
    int lv = level - h_depth1(i);
    if (lv == 0) return h_right1(i);
    i = (i << 1) + 1;
    for (int k = 1; k < lv; ++k) i <<= 1;
    return i;
}

// open-addressing map from a point (d 1D indices) to its position
struct PointMap {
    int d = 0;
    const int32_t* pts = nullptr;
    std::vector<int64_t> slot;
    static uint64_t hsh(const int32_t* I, int d) {
        uint64_t h = 0xcbf29ce484222325ull;
        for (int k = 0; k < d; ++k) { h ^= (uint32_t)I[k]; h *= 0x100000001b3ull; h ^= h >> 31; }
        return h;
    }
    void build(int d_, const int32_t* p, int64_t n) {
        d = d_;
        pts = p;
        size_t cap = 16;
        while (cap < (size_t)(2 * n)) cap <<= 1;
        slot.assign(cap, -1);
        for (int64_t k = 0; k < n; ++k) {
            uint64_t m = cap - 1, h = hsh(p + k * d, d) & m;
            while (slot[h] >= 0) h = (h + 1) & m;
            slot[h] = k;
        }
    }
    int64_t find(const int32_t* I) const {
        uint64_t m = slot.size() - 1, h = hsh(I, d) & m;
        for (;;) {
            int64_t s = slot[h];
            if (s < 0) return -1;
            if (!memcmp(pts + s * d, I, sizeof(int32_t) * d)) return s;
            h = (h + 1) & m;
        }
    }
};

// ------------------------------------------------------------------ device arithmetic
__device__ __forceinline__ double M(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double A(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double S(double a, double b) { return __dsub_rn(a, b); }

__device__ __forceinline__ int d_depth1(int32_t i) { return i < 2 ? 0 : 31 - __clz(i); }
__device__ __forceinline__ double d_coord1(int32_t i) {  // index.h:718-730 (dyadic, exact)
    if (i == 0) return 0.0;
    int t = d_depth1(i);
    return (double)(2 * (i & ~(1 << t)) + 1) / (double)(1 << t);
}

// integral over [a,b] of (mp x + cp)(mq x + cq), antiderivative form (RHS.cpp:47-54)
__device__ double int_vv(double a, double b, double mp, double mq, double cp, double cq) {
    const double c3 = 1.0 / 3.0;
    double t1 = S(M(M(M(M(M(c3, b), b), b), mp), mq), M(M(M(M(M(c3, a), a), a), mp), mq));
    double t2 = S(M(M(M(M(0.5, b), b), mp), cq), M(M(M(M(0.5, a), a), mp), cq));
    double t3 = S(M(M(M(M(0.5, b), b), mq), cp), M(M(M(M(0.5, a), a), mq), cp));
    double t4 = M(M(S(b, a), cp), cq);
    return A(A(A(t1, t2), t3), t4);
}
// the same weighted by (1 - x^2) (RHS.cpp:285-300): int_vv minus the x^2 moments
__device__ double int_vw(double a, double b, double mp, double mq, double cp, double cq) {
    const double c3 = 1.0 / 3.0, c5 = 1.0 / 5.0;
    double r1 = int_vv(a, b, mp, mq, cp, cq);
    double t1 = S(M(M(M(M(M(M(M(c5, b), b), b), b), b), mp), mq), M(M(M(M(M(M(M(c5, a), a), a), a), a), mp), mq));
    double t2 = S(M(M(M(M(M(M(0.25, b), b), b), b), mp), cq), M(M(M(M(M(M(0.25, a), a), a), a), mp), cq));
    double t3 = S(M(M(M(M(M(M(0.25, b), b), b), b), mq), cp), M(M(M(M(M(M(0.25, a), a), a), a), mq), cp));
    double t4 = S(M(M(M(M(M(c3, b), b), b), cp), cq), M(M(M(M(M(c3, a), a), a), cp), cq));
    return S(r1, A(A(A(t1, t2), t3), t4));
}

// One dimension of the hat of J at level t (centre xp, half width hp) against
// the hierarchical boundary hat of 1D index iq: the four pairs of linear
// pieces (left-left, left-right, right-left, right-right, RHS.cpp:126-268),
// of which a boundary index keeps only the half inside [0,1].
// kind 0: values, 1: derivatives, 2: values weighted by (1 - x^2).
template <int KIND>
__device__ double hat_factor(double xp, double hp, double mp, int32_t iq) {
    int tq = d_depth1(iq);
    double mq = (double)(1 << tq), hq = 1.0 / mq, xq = d_coord1(iq);
    double lp[2] = {S(xp, hp), xp}, rp[2] = {xp, A(xp, hp)};
    double lq[2] = {S(xq, hq), xq}, rq[2] = {xq, A(xq, hq)};
    double mps[2] = {mp, M(-1.0, mp)}, mqs[2] = {mq, M(-1.0, mq)};
    // (x -+ h) / h of the reference: h is a power of two, so the quotient is
    // the exact product with 1/h = m (same bits, no division)
    double cps[2] = {-M(S(xp, hp), mp), M(A(xp, hp), mp)};
    double cqs[2] = {-M(S(xq, hq), mq), M(A(xq, hq), mq)};
    double s = 0.0;
#pragma unroll
    for (int sp = 0; sp < 2; ++sp)
#pragma unroll
        for (int sq = 0; sq < 2; ++sq) {
            double v = 0.0;
            bool skip = (iq == 0 && sq == 0) || (iq == 1 && sq == 1);
            if (!skip && !(rp[sp] < lq[sq]) && !(rq[sq] < lp[sp])) {
                double a = lq[sq] > lp[sp] ? lq[sq] : lp[sp];
                double b = rp[sp] < rq[sq] ? rp[sp] : rq[sq];
                if (KIND == 1) v = M(M(S(b, a), mps[sp]), mqs[sq]);
                else if (KIND == 0) v = int_vv(a, b, mps[sp], mqs[sq], cps[sp], cqs[sq]);
                else v = int_vw(a, b, mps[sp], mqs[sq], cps[sp], cqs[sq]);
            }
            s = A(s, v);
        }
    return s;
}

// Nodal value of every entry (J, T): sum over the boundary points b of
// I(J at level T, b) hier[b].  One warp per entry; bq holds the boundary
// points' 1D indices dimension-major (bq[k * nb + b]).
// KIND 0: CalcIntegral (sum over the derivative dimension of the products),
// 1: CalcIntegral_mass, 2: CalcIntegral_coeff.
// bsup[(2k) * nb + b], bsup[(2k+1) * nb + b]: the support of boundary point b
// in dimension k, [lo, hi] in units of 2^-30 (exact: depths are at most 30)
constexpr double kSupUnit = 1073741824.0;  // 2^30

template <int D, int KIND>
__global__ void __launch_bounds__(256) k_bd_nodal(int64_t ne, const int32_t* __restrict__ ej,
                                                  const int8_t* __restrict__ et, int64_t nb,
                                                  const int32_t* __restrict__ bq, const int32_t* __restrict__ bsup,
                                                  const double* __restrict__ bh, double* __restrict__ z) {
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t e = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); e < ne; e += nwarps) {
        double xp[D], hp[D], mp[D];
        int32_t plo[D], phi[D];
#pragma unroll
        for (int k = 0; k < D; ++k) {
            int t = et[e * D + k];
            mp[k] = (double)(1 << t);
            hp[k] = 1.0 / mp[k];
            xp[k] = d_coord1(ej[e * D + k]);
            plo[k] = (int32_t)((xp[k] - hp[k]) * kSupUnit);
            phi[k] = (int32_t)((xp[k] + hp[k]) * kSupUnit);
        }
        double sum = 0.0;
        for (int64_t base = 0; base < nb; base += 32) {
            const int64_t b = base + lane;
            bool hit = b < nb;
            double c = 0.0;
            // the supports must overlap with positive length in every dimension;
            // otherwise each piece integral is exactly zero
#pragma unroll
            for (int k = 0; k < D; ++k)
                if (hit) hit = plo[k] < bsup[(2 * k + 1) * nb + b] && bsup[(2 * k) * nb + b] < phi[k];
            if (hit) {
                int32_t iq[D];
#pragma unroll
                for (int k = 0; k < D; ++k) iq[k] = bq[k * nb + b];
                double val;
                if (KIND == 0) {
                    double fv[D], fg[D];
#pragma unroll
                    for (int k = 0; k < D; ++k) {
                        fv[k] = hat_factor<0>(xp[k], hp[k], mp[k], iq[k]);
                        fg[k] = hat_factor<1>(xp[k], hp[k], mp[k], iq[k]);
                    }
                    val = 0.0;
#pragma unroll
                    for (int o = 0; o < D; ++o) {
                        double prod = 1.0;
#pragma unroll
                        for (int k = 0; k < D; ++k) prod = M(prod, k == o ? fg[k] : fv[k]);
                        val = A(val, prod);
                    }
                } else {
                    val = 1.0;
#pragma unroll
                    for (int k = 0; k < D; ++k) val = M(val, hat_factor<KIND == 1 ? 0 : 2>(xp[k], hp[k], mp[k], iq[k]));
                }
                c = M(val, bh[b]);
            }
            // add the lanes' products in boundary-point order
            unsigned mask = __ballot_sync(0xffffffffu, hit);
            while (mask) {
                int src = __ffs(mask) - 1;
                mask &= mask - 1;
                sum = A(sum, __shfl_sync(0xffffffffu, c, src));
            }
        }
        if (lane == 0) z[e] = sum;
    }
}

// ConvertToPrewavelet2 (RHS.h:397-420): rhs[out[r]] = sum over the stencil of
// row r, in stencil order, of z[entry] * weight
__global__ void k_bd_convert(int64_t nr, const int64_t* __restrict__ off, const int32_t* __restrict__ col,
                             const double* __restrict__ w, const int64_t* __restrict__ out,
                             const double* __restrict__ z, double* __restrict__ rhs) {
    int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= nr) return;
    double c = 0.0;
    for (int64_t j = off[r]; j < off[r + 1]; ++j) c = A(c, M(z[col[j]], w[j]));
    rhs[out[r]] = c;
}

__global__ void k_gather(int64_t n, const int64_t* __restrict__ idx, const double* __restrict__ src,
                         double* __restrict__ dst) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[idx[i]];
}

// ------------------------------------------------------------------ per-operator tables
struct BdState {
    int d = 0;
    int64_t ne = 0, nr = 0;
    DevArr ej, et, off, col, w, out, z;
};

int build_state(lsg_operator* op, BdState& S, cudaStream_t st) {
    const lsg::Plan& P = lsg_internal::plan(op);
    if (P.inst_n_off.size() != 2) return fail_msg(LSG_E_INVALID, "boundary right-hand sides take a single-grid operator");
    const int d = P.d;
    S.d = d;
    PointMap pm;
    pm.build(d, P.pts.data(), P.n);
    std::map<std::vector<int32_t>, int32_t> tid;
    std::unordered_map<int64_t, int32_t> eid;
    std::vector<int32_t> ej;
    std::vector<int8_t> et;
    std::vector<int64_t> off{0}, out;
    std::vector<int32_t> col;
    std::vector<double> w;
    std::vector<int32_t> T(d), J(d);
    int32_t j1[lsg::kMaxDim][5];
    double w1[lsg::kMaxDim][5];
    int n1[lsg::kMaxDim];
    for (int64_t k = 0; k < P.n; ++k) {
        if (!P.act[k]) continue;
        const int32_t* I = &P.pts[k * d];
        for (int q = 0; q < d; ++q) T[q] = h_depth1(I[q]);
        auto ti = tid.emplace(T, (int32_t)tid.size()).first->second;
        // 1D prewavelet stencils at the point's own depth (nextFiveP,
        // indices/index.cc:252-327): the point itself 1 (0.9 when a parent is
        // on the boundary and the depth is above 1), its two parents -0.6, the
        // level-t points beyond them 0.1; boundary positions are left out
        for (int q = 0; q < d; ++q) {
            int32_t i = I[q];
            int t = T[q];
            int32_t l = h_left1(i), r = h_right1(i);
            bool lok = l > 1, rok = r > 1;
            int n = 0;
            j1[q][n] = i;
            w1[q][n++] = (t > 1 && (!lok || !rok)) ? 0.9 : 1.0;
            if (lok) { j1[q][n] = l; w1[q][n++] = -0.6; }
            if (rok) { j1[q][n] = r; w1[q][n++] = -0.6; }
            if (lok) { j1[q][n] = h_left_lv(l, t); w1[q][n++] = 0.1; }
            if (rok) { j1[q][n] = h_right_lv(r, t); w1[q][n++] = 0.1; }
            n1[q] = n;
        }
        int pos[lsg::kMaxDim] = {0};
        for (;;) {  // combinations with dimension 0 fastest (MultiDimFiveCompass order)
            double val = 1.0;
            for (int q = 0; q < d; ++q) {
                J[q] = j1[q][pos[q]];
                val = val * w1[q][pos[q]];
            }
            int64_t jk = pm.find(J.data());
            if (jk >= 0) {
                int64_t key = jk * (int64_t)P.nD + ti;
                auto it = eid.find(key);
                int32_t e;
                if (it == eid.end()) {
                    e = (int32_t)(ej.size() / d);
                    eid.emplace(key, e);
                    ej.insert(ej.end(), J.begin(), J.end());
                    for (int q = 0; q < d; ++q) et.push_back((int8_t)T[q]);
                } else e = it->second;
                col.push_back(e);
                w.push_back(val);
            }
            int q = 0;
            while (q < d && ++pos[q] == n1[q]) { pos[q] = 0; ++q; }
            if (q == d) break;
        }
        off.push_back((int64_t)col.size());
        out.push_back(k);
    }
    S.ne = (int64_t)ej.size() / d;
    S.nr = (int64_t)out.size();
    int rc = 0;
    rc = rc ? rc : S.ej.upload(ej, st);
    rc = rc ? rc : S.et.upload(et, st);
    rc = rc ? rc : S.off.upload(off, st);
    rc = rc ? rc : S.col.upload(col, st);
    rc = rc ? rc : S.w.upload(w, st);
    rc = rc ? rc : S.out.upload(out, st);
    rc = rc ? rc : S.z.alloc(std::max<int64_t>(S.ne, 1) * sizeof(double));
    if (rc) return rc;
    BD_TRY(cudaStreamSynchronize(st));  // the host vectors go out of scope
    return 0;
}

int ensure_state(lsg_operator* op, BdState** out, cudaStream_t st) {
    auto& slot = lsg_internal::bdrhs_slot(op);
    if (!slot) {
        auto s = std::make_shared<BdState>();
        int rc = build_state(op, *s, st);
        if (rc) return rc;
        slot = s;
    }
    *out = static_cast<BdState*>(slot.get());
    return 0;
}

// boundary points of the second grid in the reference's summation order: the
// depth list in first-appearance order, then storage order within a depth
std::vector<int64_t> boundary_order(int d, int64_t nn, const int32_t* pts) {
    std::map<std::vector<int32_t>, int32_t> tid;
    std::vector<int32_t> id(nn);
    std::vector<int32_t> T(d);
    for (int64_t k = 0; k < nn; ++k) {
        for (int q = 0; q < d; ++q) T[q] = h_depth1(pts[k * d + q]);
        id[k] = tid.emplace(T, (int32_t)tid.size()).first->second;
    }
    std::vector<int64_t> b;
    for (int64_t k = 0; k < nn; ++k) {
        bool boundary = false;
        for (int q = 0; q < d; ++q) boundary |= pts[k * d + q] < 2;
        if (boundary) b.push_back(k);
    }
    std::stable_sort(b.begin(), b.end(), [&](int64_t x, int64_t y) { return id[x] < id[y]; });
    return b;
}

template <int D>
int launch_nodal(int kind, const BdState& S, int64_t nb, const int32_t* bq, const int32_t* bsup, const double* bh,
                 cudaStream_t st) {
    int64_t warps = S.ne;
    unsigned grid = (unsigned)std::min<int64_t>((warps + 7) / 8, 148 * 64);
    if (grid == 0) return 0;
    const int32_t* ej = S.ej.as<int32_t>();
    const int8_t* et = S.et.as<int8_t>();
    double* z = S.z.as<double>();
    if (kind == LSG_BDRHS_GRADIENT) k_bd_nodal<D, 0><<<grid, 256, 0, st>>>(S.ne, ej, et, nb, bq, bsup, bh, z);
    else if (kind == LSG_BDRHS_MASS) k_bd_nodal<D, 1><<<grid, 256, 0, st>>>(S.ne, ej, et, nb, bq, bsup, bh, z);
    else k_bd_nodal<D, 2><<<grid, 256, 0, st>>>(S.ne, ej, et, nb, bq, bsup, bh, z);
    return 0;
}

// bh: hierarchical coefficients of the boundary points, in boundary order (device)
int boundary_rhs_run(lsg_operator* op, int32_t kind, int64_t nb, const int32_t* bq, const int32_t* bsup,
                     const double* bh, double* rhs, cudaStream_t st) {
    BdState* Sp = nullptr;
    int rc = ensure_state(op, &Sp, st);
    if (rc) return rc;
    const BdState& S = *Sp;
    if (S.ne > 0 && nb > 0) {
        switch (S.d) {
        case 1: rc = launch_nodal<1>(kind, S, nb, bq, bsup, bh, st); break;
        case 2: rc = launch_nodal<2>(kind, S, nb, bq, bsup, bh, st); break;
        case 3: rc = launch_nodal<3>(kind, S, nb, bq, bsup, bh, st); break;
        case 4: rc = launch_nodal<4>(kind, S, nb, bq, bsup, bh, st); break;
        case 5: rc = launch_nodal<5>(kind, S, nb, bq, bsup, bh, st); break;
        case 6: rc = launch_nodal<6>(kind, S, nb, bq, bsup, bh, st); break;
        case 7: rc = launch_nodal<7>(kind, S, nb, bq, bsup, bh, st); break;
        case 8: rc = launch_nodal<8>(kind, S, nb, bq, bsup, bh, st); break;
        default: return fail_msg(LSG_E_INVALID, "unsupported dimension");
        }
    } else if (S.ne > 0) {
        BD_TRY(cudaMemsetAsync(S.z.p, 0, S.ne * sizeof(double), st));
    }
    if (rc) return rc;
    if (S.nr > 0)
        k_bd_convert<<<nblk(S.nr), 256, 0, st>>>(S.nr, S.off.as<int64_t>(), S.col.as<int32_t>(), S.w.as<double>(),
                                                  S.out.as<int64_t>(), S.z.as<double>(), rhs);
    BD_TRY(cudaGetLastError());
    return 0;
}

int check_points(int d, int64_t nn, const int32_t* pts) {
    for (int64_t k = 0; k < nn * d; ++k)
        if (pts[k] < 0 || (pts[k] >= 2 && h_depth1(pts[k]) > 30))
            return fail_msg(LSG_E_INVALID, "invalid 1D index in the boundary grid");
    return 0;
}

// (De)hierarchization sweeps: per dimension, one (point, left, right) list per
// depth in that dimension, finest first (hierarchization) or coarsest first
// (dehierarchization).  Points of equal depth in a dimension never read each
// other there, so each list is one launch.
//   kBoundary: the boundary points, each needs both 1D parents
//              (CalcHierarchicalBasisForRHS, RHS.cpp:6-41);
//   kActive:   the active points, an absent neighbour reads 0 (the expression
//              assignments of CalcHierarchicalBasis / CalcNodalBasis,
//              BasisTransformations.cpp:174-198,390-409).
enum class SweepSet { kBoundary, kActive };

int build_sweeps(int d, int64_t n, const int32_t* pts, const uint8_t* act, SweepSet set, bool fine_first,
                 std::vector<std::vector<int64_t>>& steps) {
    PointMap pm;
    pm.build(d, pts, n);
    std::vector<int32_t> J(d);
    for (int q = 0; q < d; ++q) {
        int maxt = 0;
        for (int64_t k = 0; k < n; ++k) maxt = std::max(maxt, h_depth1(pts[k * d + q]));
        for (int s = 0; s < maxt; ++s) {
            const int t = fine_first ? maxt - s : s + 1;
            std::vector<int64_t> klr;
            for (int64_t k = 0; k < n; ++k) {
                const int32_t* I = pts + k * d;
                if (h_depth1(I[q]) != t) continue;
                if (set == SweepSet::kBoundary) {
                    bool boundary = false;
                    for (int j = 0; j < d; ++j) boundary |= I[j] < 2;
                    if (!boundary) continue;
                } else if (!act[k]) {
                    continue;
                }
                memcpy(J.data(), I, d * sizeof(int32_t));
                J[q] = h_left1(I[q]);
                int64_t l = pm.find(J.data());
                J[q] = h_right1(I[q]);
                int64_t r = pm.find(J.data());
                if (set == SweepSet::kBoundary && (l < 0 || r < 0))
                    return fail_msg(LSG_E_INVALID, "a boundary point lacks a 1D parent in the grid");
                klr.insert(klr.end(), {k, l, r});
            }
            if (!klr.empty()) steps.push_back(std::move(klr));
        }
    }
    return 0;
}

// u[k] -/+= (u[l] + u[r]) / 2 over one list; an absent neighbour reads 0
__global__ void k_bd_sweep(int64_t n, const int64_t* __restrict__ klr, double* __restrict__ u, int sign) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t k = klr[3 * i], l = klr[3 * i + 1], r = klr[3 * i + 2];
    double s = M(0.5, A(l >= 0 ? u[l] : 0.0, r >= 0 ? u[r] : 0.0));
    u[k] = sign < 0 ? S(u[k], s) : A(u[k], s);
}

// tables: one device list per step, owned by the caller until the stream is done
int run_sweeps(const std::vector<std::vector<int64_t>>& steps, double* u, int sign, std::vector<DevArr>& tables,
               cudaStream_t st) {
    size_t base = tables.size();
    tables.resize(base + steps.size());
    for (size_t i = 0; i < steps.size(); ++i) {
        int rc = tables[base + i].upload(steps[i], st);
        if (rc) return rc;
        int64_t n = (int64_t)steps[i].size() / 3;
        k_bd_sweep<<<nblk(n), 256, 0, st>>>(n, tables[base + i].as<int64_t>(), u, sign);
    }
    BD_TRY(cudaGetLastError());
    return 0;
}

// boundary points of a grid in the reference's summation order, their 1D
// indices dimension-major, and the gather of a coefficient vector into that order
struct BoundarySet {
    int64_t nb = 0;
    DevArr dq, dsup, di;
    int build(int d, int64_t nn, const int32_t* pts, cudaStream_t st) {
        std::vector<int64_t> b = boundary_order(d, nn, pts);
        nb = (int64_t)b.size();
        std::vector<int32_t> bq((size_t)nb * d), sup((size_t)nb * d * 2);
        for (int64_t i = 0; i < nb; ++i)
            for (int q = 0; q < d; ++q) {
                int32_t iq = pts[b[i] * d + q];
                bq[(size_t)q * nb + i] = iq;
                // support in units of 2^-30: [0, 1] for the boundary indices (their
                // half inside the domain), [2j, 2j + 2] 2^-t for index 2^t + j
                int64_t lo = 0, hi = (int64_t)1 << 30;
                if (iq >= 2) {
                    int t = h_depth1(iq);
                    int64_t j = iq - ((int64_t)1 << t), s = (int64_t)1 << (30 - t);
                    lo = 2 * j * s;
                    hi = (2 * j + 2) * s;
                }
                sup[(size_t)(2 * q) * nb + i] = (int32_t)lo;
                sup[(size_t)(2 * q + 1) * nb + i] = (int32_t)hi;
            }
        int rc = dq.upload(bq, st);
        rc = rc ? rc : dsup.upload(sup, st);
        rc = rc ? rc : di.upload(b, st);
        if (rc) return rc;
        BD_TRY(cudaStreamSynchronize(st));  // the host vectors go out of scope
        return 0;
    }
    void gather(const double* src, double* dst, cudaStream_t st) const {
        if (nb > 0) k_gather<<<nblk(nb), 256, 0, st>>>(nb, di.as<int64_t>(), src, dst);
    }
};

__global__ void k_split_interior(int64_t n, const int64_t* __restrict__ kj, double* __restrict__ f,
                                 double* __restrict__ fd) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t k = kj[2 * i], j = kj[2 * i + 1];
    if (j >= 0) fd[j] = f[k];
    f[k] = 0.0;
}

__global__ void k_add_active(int64_t n, const uint8_t* __restrict__ act, double* __restrict__ y,
                             const double* __restrict__ x, int sign) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n && act[i]) y[i] = sign < 0 ? S(y[i], x[i]) : A(y[i], x[i]);
}

int hierarchize_host(int32_t d, int64_t n, const int32_t* points, const uint8_t* active, double* u, SweepSet set,
                     int sign) {
    if (d < 1 || d > lsg::kMaxDim || n < 0 || (n > 0 && (!points || !u || (set == SweepSet::kActive && !active))))
        return fail_msg(LSG_E_INVALID, "bad argument");
    if (n == 0) return 0;
    int rc = check_points(d, n, points);
    if (rc) return rc;
    std::vector<std::vector<int64_t>> steps;
    rc = build_sweeps(d, n, points, active, set, sign < 0, steps);
    if (rc) return rc;
    cudaStream_t st;
    BD_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct Guard { cudaStream_t s; ~Guard() { cudaStreamDestroy(s); } } guard{st};
    DevArr du;
    std::vector<double> hu(u, u + n);
    std::vector<DevArr> tables;
    rc = du.upload(hu, st);
    rc = rc ? rc : run_sweeps(steps, du.as<double>(), sign, tables, st);
    if (rc) return rc;
    BD_TRY(cudaMemcpyAsync(u, du.p, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    BD_TRY(cudaStreamSynchronize(st));
    return 0;
}

}  // namespace

extern "C" {

int lsg_hierarchize_boundary(int32_t d, int64_t nn, const int32_t* points, double* u) {
    return hierarchize_host(d, nn, points, nullptr, u, SweepSet::kBoundary, -1);
}

int lsg_hierarchize(int32_t d, int64_t n, const int32_t* points, const uint8_t* active, double* u) {
    return hierarchize_host(d, n, points, active, u, SweepSet::kActive, -1);
}

int lsg_dehierarchize(int32_t d, int64_t n, const int32_t* points, const uint8_t* active, double* u) {
    return hierarchize_host(d, n, points, active, u, SweepSet::kActive, +1);
}

int lsg_boundary_rhs_device(lsg_operator* op, int32_t kind, int64_t nn, const int32_t* points, const double* hier,
                            double* rhs, void* stream) {
    if (!op || nn < 0 || (nn > 0 && (!points || !hier)) || !rhs) return fail_msg(LSG_E_INVALID, "null argument");
    if (kind < LSG_BDRHS_GRADIENT || kind > LSG_BDRHS_MASS_COEFF) return fail_msg(LSG_E_INVALID, "bad kind");
    const int d = lsg_internal::plan(op).d;
    int rc = check_points(d, nn, points);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    BoundarySet B;
    DevArr dh;
    if ((rc = B.build(d, nn, points, st)) || (rc = dh.alloc(std::max<int64_t>(B.nb, 1) * 8))) return rc;
    B.gather(hier, dh.as<double>(), st);
    rc = boundary_rhs_run(op, kind, B.nb, B.dq.as<int32_t>(), B.dsup.as<int32_t>(), dh.as<double>(), rhs, st);
    if (rc) return rc;
    BD_TRY(cudaStreamSynchronize(st));  // the device tables go out of scope
    return 0;
}

int lsg_boundary_rhs(lsg_operator* op, int32_t kind, int64_t nn, const int32_t* points, const double* hier,
                     double* rhs) {
    if (!op || nn < 0 || (nn > 0 && (!points || !hier)) || !rhs) return fail_msg(LSG_E_INVALID, "null argument");
    const int64_t n = lsg_internal::plan(op).n;
    DevArr dh, dr;
    std::vector<double> hh(hier, hier + nn), hr(rhs, rhs + n);
    int rc = 0;
    if ((rc = dh.upload(hh, 0)) || (rc = dr.upload(hr, 0))) return rc;
    rc = lsg_boundary_rhs_device(op, kind, nn, points, dh.as<double>(), dr.as<double>(), nullptr);
    if (rc) return rc;
    BD_TRY(cudaMemcpy(rhs, dr.p, n * sizeof(double), cudaMemcpyDeviceToHost));
    return 0;
}

int lsg_pde_boundary_rhs(lsg_operator* op, int32_t kind, int64_t nn, const int32_t* npoints, const uint8_t* nactive,
                         double* f, double* g, double* rhs) {
    if (!op || nn < 1 || !npoints || !nactive || !f || !g || !rhs) return fail_msg(LSG_E_INVALID, "null argument");
    if (kind != LSG_PDE_POISSON && kind != LSG_PDE_HELMHOLTZ) return fail_msg(LSG_E_INVALID, "bad kind");
    const lsg::Plan& P = lsg_internal::plan(op);
    if (P.inst_n_off.size() != 2) return fail_msg(LSG_E_INVALID, "boundary right-hand sides take a single-grid operator");
    const int d = P.d;
    const int64_t n = P.n;
    int rc = check_points(d, nn, npoints);
    if (rc) return rc;
    // host tables: the three sweeps and the interior points shared by both grids
    std::vector<std::vector<int64_t>> sw_f, sw_fd, sw_g;
    if ((rc = build_sweeps(d, nn, npoints, nactive, SweepSet::kActive, true, sw_f)) ||
        (rc = build_sweeps(d, n, P.pts.data(), P.act.data(), SweepSet::kActive, false, sw_fd)) ||
        (rc = build_sweeps(d, nn, npoints, nullptr, SweepSet::kBoundary, true, sw_g)))
        return rc;
    PointMap pm;
    pm.build(d, P.pts.data(), n);
    std::vector<int64_t> kj;
    for (int64_t k = 0; k < nn; ++k) {
        const int32_t* I = npoints + k * d;
        bool interior = nactive[k] != 0;
        for (int q = 0; q < d; ++q) interior &= I[q] >= 2;
        if (interior) kj.insert(kj.end(), {k, pm.find(I)});
    }
    cudaStream_t st;
    BD_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct Guard { cudaStream_t s; ~Guard() { cudaStreamDestroy(s); } } guard{st};
    BoundarySet B;
    DevArr df, dg, dfd, dprew, drhs, dy, dbh, dkj;
    std::vector<DevArr> tables;
    std::vector<double> hf(f, f + nn), hg(g, g + nn);
    if ((rc = B.build(d, nn, npoints, st)) || (rc = df.upload(hf, st)) || (rc = dg.upload(hg, st)) ||
        (rc = dkj.upload(kj, st)) || (rc = dfd.alloc(n * 8)) || (rc = dprew.alloc(n * 8)) ||
        (rc = drhs.alloc(n * 8)) || (rc = dy.alloc(n * 8)) || (rc = dbh.alloc(std::max<int64_t>(B.nb, 1) * 8)))
        return rc;
    double *F = df.as<double>(), *G = dg.as<double>(), *FD = dfd.as<double>(), *R = drhs.as<double>(),
           *Y = dy.as<double>();
    const uint8_t* act = lsg_internal::active(op);
    // f in the hierarchical basis of the boundary grid; its interior part moves
    // to this grid and back to nodal values (PDE.cpp:12-33)
    BD_TRY(cudaMemsetAsync(FD, 0, n * 8, st));
    if ((rc = run_sweeps(sw_f, F, -1, tables, st))) return rc;
    int64_t nkj = (int64_t)kj.size() / 2;
    if (nkj > 0) k_split_interior<<<nblk(nkj), 256, 0, st>>>(nkj, dkj.as<int64_t>(), F, FD);
    if ((rc = run_sweeps(sw_fd, FD, +1, tables, st))) return rc;
    // <f_inner, psi_i>: prewavelet coefficients, then the coefficient-1 mass product (HelmHoltz)
    if ((rc = lsg_internal::prew_by_nodal_dev(op, dprew.as<double>(), FD, st))) return rc;
    BD_TRY(cudaMemsetAsync(R, 0, n * 8, st));
    if ((rc = lsg_internal::matvec64_unit(op, LSG_FORM_MASS, dprew.as<double>(), R, st))) return rc;
    // + <f_boundary, psi_i> (multiply_mass of the boundary coefficients of f)
    B.gather(F, dbh.as<double>(), st);
    BD_TRY(cudaMemsetAsync(Y, 0, n * 8, st));
    rc = boundary_rhs_run(op, LSG_BDRHS_MASS, B.nb, B.dq.as<int32_t>(), B.dsup.as<int32_t>(), dbh.as<double>(), Y, st);
    if (rc) return rc;
    k_add_active<<<nblk(n), 256, 0, st>>>(n, act, R, Y, +1);
    // - <grad g, grad psi_i> (- <c g, psi_i> for the Helmholtz problem)
    if ((rc = run_sweeps(sw_g, G, -1, tables, st))) return rc;
    B.gather(G, dbh.as<double>(), st);
    BD_TRY(cudaMemsetAsync(Y, 0, n * 8, st));
    rc = boundary_rhs_run(op, LSG_BDRHS_GRADIENT, B.nb, B.dq.as<int32_t>(), B.dsup.as<int32_t>(), dbh.as<double>(), Y, st);
    if (rc) return rc;
    k_add_active<<<nblk(n), 256, 0, st>>>(n, act, R, Y, -1);
    if (kind == LSG_PDE_HELMHOLTZ) {
        BD_TRY(cudaMemsetAsync(Y, 0, n * 8, st));
        rc = boundary_rhs_run(op, LSG_BDRHS_MASS_COEFF, B.nb, B.dq.as<int32_t>(), B.dsup.as<int32_t>(),
                              dbh.as<double>(), Y, st);
        if (rc) return rc;
        k_add_active<<<nblk(n), 256, 0, st>>>(n, act, R, Y, -1);
    }
    BD_TRY(cudaGetLastError());
    BD_TRY(cudaMemcpyAsync(rhs, R, n * 8, cudaMemcpyDeviceToHost, st));
    BD_TRY(cudaMemcpyAsync(f, F, nn * 8, cudaMemcpyDeviceToHost, st));
    BD_TRY(cudaMemcpyAsync(g, G, nn * 8, cudaMemcpyDeviceToHost, st));
    BD_TRY(cudaStreamSynchronize(st));
    return 0;
}

}  // extern "C"
