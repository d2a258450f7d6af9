// B200 (sm_100a) prewavelet matvec, Jacobi diagonal and CG behind the C-ABI of
// include/lsg.h.  The host planner (lsg_plan.cpp) produces integer tables and a
// static level schedule; this file uploads them and runs:
//   k_nodal      prewavelet -> nodal values per depth (calcNodal,
//                MatrixVectorHomogen.cpp:43-74), sum-factorised 3-tap stages
//   k_pinit      P_c(T) = nodal(T)            ("P += nodal", MVH.h:1649)
//   k_prolong    prolongation chains, one launch per dimension (MVH.h:1655-1670, 444-474)
//   k_sf         the level-T cell operator (LocalStiffnessMatrices.cpp:555-582)
//                of dense slabs, factorised over reduced modes (lsg_sf_kernel.cuh)
//   k_cells      the same for sparse slabs, per cell in the Walsh-Hadamard
//                basis where the Q1 element is diagonal
//   k_level      one restriction wavefront: per (case, depth) item the gM
//                bookkeeping + restrictions (MVH.h:1672-1735, 485-530)
//                + ConvertToPrewavelet2 (MVH.h:540-562), sum-factorised 5-tap
//   k_diag       exact Jacobi diagonal (cg_method.h:544-680)
//   CG kernels   CG::solveHomogen vector semantics (cg_method.h:759-886)
#include "lsg_plan.h"
#include "lsg_sf.h"
#include "lsg_coef.cuh"
#include "lsg_internal.h"
#include "../../include/lsg.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <tuple>
#include <string>
#include <type_traits>
#include <vector>

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define CUDA_TRY(expr)                                                                       \
    do {                                                                                     \
        cudaError_t _e = (expr);                                                             \
        if (_e != cudaSuccess)                                                               \
            return fail(LSG_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e));     \
    } while (0)

// ----------------------------------------------------------------------------- device tables
struct DevSlab {
    int64_t off, n, cell_off, ncell, corner_off;
    int32_t dense, pad;
    int32_t T[lsg::kMaxDim];
    int32_t ext[lsg::kMaxDim];     // 2^T_k - 1 (interior points per dim)
    int32_t stride[lsg::kMaxDim];  // slab-position stride of dim k (dense slabs)
};

struct DevPlan {
    int d, nD;
    int64_t n;
    const DevSlab* slabs;
    const int32_t* did;
    const uint8_t* act;
    const int64_t* exa_off;
    const int64_t* exa;
    const uint64_t* cell_key;   // sparse cells
    const int32_t* cell_corner;
    const int64_t* nodal_stage;  // nD*d+1
    const int32_t* nodal_src;
    const int32_t* nodal_code;
    const int64_t* nodal_dom;    // nD*(d+1)
    const int64_t* nodal_scr;    // per depth scratch offset
    const int64_t* conv_stage;
    const int32_t* conv_src;
    const int32_t* conv_code;
    const int64_t* conv_dom;
    const int32_t* prol;
    const int32_t* restr;
    const lsg::PhaseAItem* a_items;
    const lsg::PhaseBItem* b_items;
    const lsg::PhaseBStep* b_steps;
    const int32_t* pts;
    const int32_t* a_chain_off;     // per prolongation chain: range in a_chain_items
    const int32_t* a_chain_items;   // phase-A items, chain by chain, in chain order
    const int64_t* sp_slot_off;     // per phase-B item of a sparse slab: first cell slot (-1: dense)
    const int64_t* sp_inc_base;     // per sparse slab: start of its per-entry ranges in sp_inc_off
    const int64_t* sp_inc_off;      // per sparse-slab entry: range of its (cell, corner) slots in sp_inc
    const int32_t* sp_inc;          // slot ids (cell * 2^d + corner) in cell order
    const int64_t* conv_off;        // per phase-B item: first convert slot (-1: none)
    const int32_t* conv_items_off;  // per depth: range in conv_items
    const int32_t* conv_items;      // items whose restrictions end at the depth, in item order
};

template <typename V>
__device__ __forceinline__ V wcode(int c) {
    // 0: none, 1: 1.0, 2: 0.9, 3: -0.6, 4: 0.1 (nextFiveP weights, indices/index.cc:252-327)
    switch (c) {
    case 1: return V(1.0);
    case 2: return V(0.9);
    case 3: return V(-0.6);
    case 4: return V(0.1);
    default: return V(0.0);
    }
}

// one sum-factorised stencil stage: out[e] = sum_s w_s in[src_s]
template <int NS, typename V, typename VI>
__device__ __forceinline__ void stage_gather(const int32_t* __restrict__ src, const int32_t* __restrict__ code,
                                             int64_t nout, const VI* __restrict__ in, const int64_t* __restrict__ in_map,
                                             V* __restrict__ out) {
    for (int64_t e = threadIdx.x; e < nout; e += blockDim.x) {
        int cd = code[e];
        V acc = V(0);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            int32_t i = src[e * NS + s];
            if (i < 0) break;
            V v = in_map ? V(in[in_map[i]]) : V(in[i]);
            acc += wcode<V>((cd >> (3 * s)) & 7) * v;
        }
        out[e] = acc;
    }
}

// ----------------------------------------------------------------------------- nodal
template <typename V>
__global__ void k_nodal(DevPlan P, const V* __restrict__ x, V* __restrict__ ml, V* __restrict__ scratch) {
    int t = blockIdx.x;
    int d = P.d;
    const DevSlab& s = P.slabs[t];
    V* scr = scratch + P.nodal_scr[t];
    const int64_t* dom = P.nodal_dom + t * (d + 1);
    // stage buffers for domains 1..d-1 are consecutive in scr
    int64_t off_in = 0, off_out = 0;
    for (int j = 0; j < d; ++j) {
        int64_t so = P.nodal_stage[t * d + j];
        int64_t nout = dom[j + 1];
        V* out = (j == d - 1) ? ml + s.off : scr + off_out;
        if (j == 0) stage_gather<3, V, V>(P.nodal_src + so * 3, P.nodal_code + so, nout, x, P.exa + P.exa_off[t], out);
        else stage_gather<3, V, V>(P.nodal_src + so * 3, P.nodal_code + so, nout, scr + off_in, nullptr, out);
        off_in = off_out;
        off_out += (j == d - 1) ? 0 : nout;
        __syncthreads();
    }
}

// ----------------------------------------------------------------------------- P init, prolongation
template <typename V>
__global__ void k_pinit(DevPlan P, const V* __restrict__ ml, V* __restrict__ pc, int32_t item0) {
    const lsg::PhaseBItem it = P.b_items[item0 + blockIdx.x];
    const DevSlab& s = P.slabs[it.t];
    for (int64_t e = threadIdx.x; e < s.n; e += blockDim.x) pc[it.p_off + e] = ml[s.off + e];
}

// One prolongation chain per CTA: the items of one case and dimension k along
// a line of depths T, T + e_k, T + 2 e_k, ... in that order (each item reads
// the previous one's output), so a dimension's whole level loop is one launch.
// Chains of one dimension are independent: they write different slabs.
template <typename V>
__global__ void k_prolong(DevPlan P, V* __restrict__ pc, int32_t chain0) {
    const int32_t c = chain0 + blockIdx.x;
    for (int32_t j = P.a_chain_off[c]; j < P.a_chain_off[c + 1]; ++j) {
        const lsg::PhaseAItem it = P.a_items[P.a_chain_items[j]];
        const int32_t* tab = P.prol + it.tab_off;
        const V* src = pc + it.src_off;
        V* dst = pc + it.dst_off;
        for (int64_t e = threadIdx.x; e < it.n_dst; e += blockDim.x) {
            int32_t a = tab[2 * e], b = tab[2 * e + 1];
            V add;
            if (b == -2) add = src[a];
            else add = V(0.5) * ((b >= 0 ? src[b] : V(0)) + (a >= 0 ? src[a] : V(0)));
            dst[e] = dst[e] + add;
        }
        __syncthreads();
    }
}

// ----------------------------------------------------------------------------- cell operator, lane groups
// A cell's 2^D corner values are spread over a group of G = 2^(D-DL) lanes:
// lane g of the group holds the NL = 2^DL corners whose high bits (dims
// DL..D-1) equal g.  The Walsh-Hadamard butterflies of dims < DL are
// register-local, those of dims >= DL use warp shuffles inside the group.
// lane-group layout: FP32 keeps 2^3 corners per lane (smaller register
// footprint, three CTAs per SM), FP64 2^4 (measured on d = 6 grids)
#ifndef LSG_F32_LOCAL_DIMS
#define LSG_F32_LOCAL_DIMS 3
#endif
template <int D, typename V>
struct CellCfg {
    static constexpr int KDL = std::is_same<V, float>::value ? LSG_F32_LOCAL_DIMS : 4;
    static constexpr int DL = D <= KDL ? D : KDL;
    static constexpr int G = 1 << (D - DL);
    static constexpr int NL = 1 << DL;
};

template <int D, typename V>
__device__ __forceinline__ void wht_group(V* v, int g) {
    constexpr int DL = CellCfg<D, V>::DL, NL = CellCfg<D, V>::NL;
#pragma unroll
    for (int k = 0; k < DL; ++k)
#pragma unroll
        for (int b = 0; b < NL; ++b)
            if (!(b & (1 << k))) {
                V p = v[b], q = v[b | (1 << k)];
                v[b] = p + q;
                v[b | (1 << k)] = p - q;
            }
#pragma unroll
    for (int k = DL; k < D; ++k) {
        int m = 1 << (k - DL);
        V sgn = (g & m) ? V(-1) : V(1);  // low lane: v + p, high lane: p - v
#pragma unroll
        for (int b = 0; b < NL; ++b) {
            V p = __shfl_xor_sync(0xffffffffu, v[b], m);
            v[b] = fma(sgn, v[b], p);
        }
    }
}

// FP32 full-cell transform on packed pairs: value 2q+e of the lane's NL
// corners is component e of v[q]; bit 0 inside pairs, bits 1..DL-1 across
// pairs, dims DL..D-1 across lanes.  Bitwise the same as wht_group<D, float>.
template <int D>
__device__ __forceinline__ void wht_group_f2(float2* v, int g) {
    constexpr int DL = CellCfg<D, float>::DL, NP = CellCfg<D, float>::NL / 2;
    const float2 neg1 = make_float2(-1.f, -1.f);
#pragma unroll
    for (int q = 0; q < NP; ++q) {
        float a = v[q].x, b = v[q].y;
        v[q] = make_float2(a + b, a - b);
    }
#pragma unroll
    for (int k = 1; k < DL; ++k)
#pragma unroll
        for (int q = 0; q < NP; ++q)
            if (!(q & (1 << (k - 1)))) {
                float2 p = v[q], w = v[q | (1 << (k - 1))];
                v[q] = __fadd2_rn(p, w);
                v[q | (1 << (k - 1))] = __ffma2_rn(w, neg1, p);
            }
#pragma unroll
    for (int k = DL; k < D; ++k) {
        int m = 1 << (k - DL);
        float sg = (g & m) ? -1.f : 1.f;
        float2 sgn = make_float2(sg, sg);
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            float2 p;
            p.x = __shfl_xor_sync(0xffffffffu, v[q].x, m);
            p.y = __shfl_xor_sync(0xffffffffu, v[q].y, m);
            v[q] = __ffma2_rn(sgn, v[q], p);
        }
    }
}

// Cell operator of a sparse slab (the cells whose interior corners all exist,
// cells/CellStructure.h:23-61): every cell's 2^d outputs go to its own slots
// (cell * 2^d + corner), and each slab entry then sums the slots of its cells
// in a fixed order (cell, then corner) -- no atomics.
template <int D, typename V>
__device__ void cells_sparse(const DevPlan& P, const DevSlab& s, const V* __restrict__ u, V* __restrict__ slots,
                             const V* __restrict__ ac, const V* lamg) {
    constexpr int DL = CellCfg<D, V>::DL, G = CellCfg<D, V>::G, NL = CellCfg<D, V>::NL;
    constexpr bool PACK = std::is_same<V, float>::value && NL >= 4;
    const int g = threadIdx.x & (G - 1);
    const int64_t group = threadIdx.x / G, ngroups = blockDim.x / G;
    const int64_t rounds = (s.ncell + ngroups - 1) / ngroups;
    for (int64_t r = 0; r < rounds; ++r) {
        int64_t ci = r * ngroups + group;
        bool live = ci < s.ncell;
        const int32_t* cp = P.cell_corner + ((s.corner_off + (live ? ci : 0)) << D) + (g << DL);
        V* out = slots + ((live ? ci : 0) << D) + (g << DL);
        int32_t pos[NL];
#pragma unroll
        for (int b = 0; b < NL; ++b) pos[b] = live ? cp[b] : -1;
        V a = live ? ac[ci] : V(0);
        if constexpr (PACK) {
            constexpr int NP = NL / 2;
            float2 v[NP];
#pragma unroll
            for (int q = 0; q < NP; ++q) {
                v[q].x = pos[2 * q] >= 0 ? u[pos[2 * q]] : 0.f;
                v[q].y = pos[2 * q + 1] >= 0 ? u[pos[2 * q + 1]] : 0.f;
            }
            wht_group_f2<D>(v, g);
            float2 a2 = make_float2((float)a, (float)a);
#pragma unroll
            for (int q = 0; q < NP; ++q)
                v[q] = __fmul2_rn(v[q], __fmul2_rn(a2, make_float2((float)lamg[2 * q], (float)lamg[2 * q + 1])));
            wht_group_f2<D>(v, g);
            if (live)
#pragma unroll
                for (int q = 0; q < NP; ++q) {
                    out[2 * q] = (V)v[q].x;
                    out[2 * q + 1] = (V)v[q].y;
                }
        } else {
            V v[NL];
#pragma unroll
            for (int b = 0; b < NL; ++b) v[b] = pos[b] >= 0 ? u[pos[b]] : V(0);
            wht_group<D, V>(v, g);
#pragma unroll
            for (int b = 0; b < NL; ++b) v[b] *= a * lamg[b];
            wht_group<D, V>(v, g);
            if (live)
#pragma unroll
                for (int b = 0; b < NL; ++b) out[b] = v[b];
        }
    }
}

// ----------------------------------------------------------------------------- phase B, cell operator (sparse slabs)
// z_c(T) = A_T P_c(T) for the (case, depth) items of sparse slabs, one CTA per
// item (dense slabs go to k_sf); u lives in shared memory when N_T fits.
template <int D, typename V>
__global__ void __launch_bounds__(256) k_cells(DevPlan P, const V* __restrict__ pc, V* __restrict__ zb,
                                              const V* __restrict__ acell, const V* __restrict__ lam_all,
                                              const int32_t* __restrict__ order, int32_t ord0, int64_t cap,
                                              V* __restrict__ slot_buf) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NC = 1 << D;
    const int32_t ii = order[ord0 + blockIdx.x];
    const lsg::PhaseBItem it = P.b_items[ii];
    const DevSlab& s = P.slabs[it.t];
    V* lam = reinterpret_cast<V*>(smem_raw);
    for (int b = threadIdx.x; b < NC; b += blockDim.x) lam[b] = lam_all[(int64_t)it.t * NC + b];
    const V* lamg = lam + ((threadIdx.x & (CellCfg<D, V>::G - 1)) << CellCfg<D, V>::DL);
    const V* u = pc + it.p_off;
    if (s.n <= cap) {
        V* us = lam + NC;
        for (int64_t e = threadIdx.x; e < s.n; e += blockDim.x) us[e] = u[e];
        u = us;
    }
    __syncthreads();
    V* slots = slot_buf + P.sp_slot_off[ii];
    cells_sparse<D, V>(P, s, u, slots, acell + s.cell_off, lamg);
    __syncthreads();
    const int64_t* inc_off = P.sp_inc_off + P.sp_inc_base[it.t];
    V* z = zb + it.p_off;
    for (int64_t e = threadIdx.x; e < s.n; e += blockDim.x) {
        V acc = V(0);
        for (int64_t j = inc_off[e]; j < inc_off[e + 1]; ++j) acc += slots[P.sp_inc[j]];
        z[e] = acc;
    }
}

// ----------------------------------------------------------------------------- phase B, wavefront level
// Per (case, depth) item of one restriction wavefront: z = z_c(T) + gM_c(T),
// the restriction steps with the gM swap-add, and ConvertToPrewavelet2 into
// the item's own convert slots (summed into y by k_conv_gather).
// Buffers ping-pong in shared memory when the item's largest vector fits.
template <int D, typename V>
__global__ void __launch_bounds__(512) k_level(DevPlan P, const V* __restrict__ zb, V* __restrict__ gm,
                                               V* __restrict__ scratch, V* __restrict__ conv, int32_t item0,
                                               int64_t buf_elems) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const lsg::PhaseBItem it = P.b_items[item0 + blockIdx.x];
    const DevSlab& s = P.slabs[it.t];
    // largest vector of this item
    int64_t need = s.n;
    for (int32_t si = it.step_begin; si < it.step_end; ++si) need = max(need, P.b_steps[si].n_dst);
    if (it.t_conv >= 0)
        for (int j = 1; j < D; ++j) need = max(need, P.conv_dom[it.t_conv * (D + 1) + j]);
    V *A, *B;
    bool ping = need <= buf_elems;
    int64_t used = 0;
    V* scr = scratch + it.scratch_off;
    if (ping) {
        A = reinterpret_cast<V*>(smem_raw);
        B = A + buf_elems;
    } else {
        A = scr;
        B = scr + s.n;
        used = s.n;
    }
    const V* z0 = zb + it.p_off;
    const V* g0 = gm + it.gm_off;
    for (int64_t e = threadIdx.x; e < s.n; e += blockDim.x) A[e] = it.gm_prev ? z0[e] + g0[e] : z0[e];
    __syncthreads();
    for (int32_t si = it.step_begin; si < it.step_end; ++si) {
        const lsg::PhaseBStep st = P.b_steps[si];
        const int32_t* tab = P.restr + st.tab_off;
        V* g = gm + st.gm_off;
        for (int64_t q = threadIdx.x; q < st.n_dst; q += blockDim.x) {
            int32_t a = tab[3 * q], l = tab[3 * q + 1], r = tab[3 * q + 2];
            V v = A[a];
            if (l >= 0) v = v + V(0.5) * A[l];
            if (r >= 0) v = v + V(0.5) * A[r];
            V tmp = st.gm_prev ? g[q] : V(0);
            g[q] = v;
            B[q] = v + tmp;
        }
        __syncthreads();
        if (ping) { V* t = A; A = B; B = t; }
        else { A = B; used += st.n_dst; B = scr + used; }
    }
    if (it.t_conv >= 0) {
        int tc = it.t_conv;
        const int64_t* dom = P.conv_dom + tc * (D + 1);
        for (int j = 0; j < D; ++j) {
            int64_t so = P.conv_stage[tc * D + j];
            int64_t nout = dom[j + 1];
            if (j == D - 1) {
                const int32_t* src = P.conv_src + so * 5;
                const int32_t* code = P.conv_code + so;
                V* out = conv + P.conv_off[item0 + blockIdx.x];
                for (int64_t e = threadIdx.x; e < nout; e += blockDim.x) {
                    int cd = code[e];
                    V acc = V(0);
#pragma unroll
                    for (int q = 0; q < 5; ++q) {
                        int32_t i = src[e * 5 + q];
                        if (i < 0) break;
                        acc += wcode<V>((cd >> (3 * q)) & 7) * A[i];
                    }
                    out[e] = acc;
                }
            } else {
                stage_gather<5, V, V>(P.conv_src + so * 5, P.conv_code + so, nout, A, nullptr, B);
                __syncthreads();
                if (ping) { V* t = A; A = B; B = t; }
                else { A = B; used += nout; B = scr + used; }
            }
        }
    }
}

// y at every active point: the sum of its convert contributions over the
// items whose restrictions end at its depth, in item order (the reference adds
// the cases' Ax_neu in CasesIterator order, MatrixVectorHomogen.h:740-748).
template <typename V>
__global__ void k_conv_gather(DevPlan P, int64_t na, const V* __restrict__ conv, V* __restrict__ y) {
    int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= na) return;
    const int64_t k = P.exa[g];
    const int t = P.did[k];
    const int64_t e = g - P.exa_off[t];
    V acc = V(0);
    for (int32_t j = P.conv_items_off[t]; j < P.conv_items_off[t + 1]; ++j) acc += conv[P.conv_off[P.conv_items[j]] + e];
    y[k] = acc;
}

}  // namespace
#include "lsg_sf_kernel.cuh"
namespace {

// ----------------------------------------------------------------------------- coefficient, diag
// a(x_c) at the midpoint of every cell of one part of the plan (cells
// [c_lo, c_hi) on slabs [t_lo, t_hi)); the part's family and parameters
__global__ void k_cell_coef(DevPlan P, int64_t c_lo, int64_t c_hi, int t_lo, int t_hi, int family,
                            const double* __restrict__ params, double* __restrict__ a64, float* __restrict__ a32,
                            const int64_t* __restrict__ cell_slab_off) {
    int64_t gi = c_lo + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (gi >= c_hi) return;
    // slab of this cell (cell_slab_off is the prefix of cell counts)
    int lo = t_lo, hi = t_hi;
    while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (cell_slab_off[mid] <= gi) lo = mid;
        else hi = mid;
    }
    const DevSlab& s = P.slabs[lo];
    int64_t ci = gi - s.cell_off;
    uint64_t key = s.dense ? (uint64_t)ci : P.cell_key[s.corner_off + ci];
    double x[lsg::kMaxDim];
    for (int k = 0; k < P.d; ++k) {
        uint64_t cext = (uint64_t)s.ext[k] + 1;
        int64_t m = (int64_t)(key % cext);
        key /= cext;
        double lo_c = ldexp((double)m, -s.T[k]);
        double hi_c = ldexp((double)(m + 1), -s.T[k]);
        x[k] = 0.5 * (lo_c + hi_c);
    }
    double a = lsg_coef_eval_dev(family, params, P.d, x);
    a64[gi] = a;
    a32[gi] = (float)a;
}

// diag_i = v^T A_T v for v = psi_i on level T = Depth(i): sum over the level-T
// cells inside the grid that touch the support of psi_i of
// a_c * sum_k qK_k prod_{j!=k} qM_j (v is a tensor product on every such cell).
template <int D>
__global__ void k_diag(DevPlan P, const double* __restrict__ acell, double* __restrict__ diag, int form) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= P.n) return;
    if (!P.act[k]) { diag[k] = 0.0; return; }
    const DevSlab& s = P.slabs[P.did[k]];
    // 1D weights at the 6 candidate cells of each dim: cell m in {c-3..c+2}
    double wl[D][6], wr[D][6], h[D];
    int64_t mm[D][6];
    int nm[D];
    for (int j = 0; j < D; ++j) {
        int32_t idx = P.pts[k * D + j];
        int t = s.T[j];
        int64_t c = 2 * (int64_t)(idx - (1 << t)) + 1;
        int64_t top = (int64_t)1 << t;
        h[j] = ldexp(1.0, -t);
        bool lok = c - 1 > 0, rok = c + 1 < top;
        double w[7];  // weights at c-3..c+3
        for (int q = 0; q < 7; ++q) w[q] = 0.0;
        w[3] = (t > 1 && (!lok || !rok)) ? 0.9 : 1.0;
        if (lok) { w[2] = -0.6; w[1] = 0.1; }
        if (rok) { w[4] = -0.6; w[5] = 0.1; }
        nm[j] = 0;
        for (int q = 0; q < 6; ++q) {
            int64_t m = c - 3 + q;
            if (m < 0 || m >= top) continue;
            if (w[q] == 0.0 && w[q + 1] == 0.0) continue;
            mm[j][nm[j]] = m;
            wl[j][nm[j]] = w[q];
            wr[j][nm[j]] = w[q + 1];
            nm[j]++;
        }
    }
    double acc = 0.0;
    int ctr[D];
    for (int j = 0; j < D; ++j) ctr[j] = 0;
    for (;;) {
        uint64_t key = 0, cs = 1;
        for (int j = 0; j < D; ++j) {
            key += (uint64_t)mm[j][ctr[j]] * cs;
            cs *= (uint64_t)s.ext[j] + 1;
        }
        int64_t ci = -1;
        if (s.dense) ci = (int64_t)key;
        else {
            const uint64_t* ks = P.cell_key + s.corner_off;
            int64_t lo = 0, hi = s.ncell;
            while (lo < hi) {
                int64_t mid = (lo + hi) / 2;
                if (ks[mid] < key) lo = mid + 1;
                else hi = mid;
            }
            if (lo < s.ncell && ks[lo] == key) ci = lo;
        }
        if (ci >= 0) {
            double qK[D], qM[D];
            for (int j = 0; j < D; ++j) {
                double a = wl[j][ctr[j]], b = wr[j][ctr[j]];
                qK[j] = (a - b) * (a - b) / h[j];
                qM[j] = h[j] * (a * a + a * b + b * b) / 3.0;
            }
            double sum = 0.0;
            if (form == 1) {  // mass: prod_j qM_j
                sum = 1.0;
                for (int j = 0; j < D; ++j) sum *= qM[j];
            } else {
                for (int i = 0; i < D; ++i) {
                    double prod = qK[i];
                    for (int j = 0; j < D; ++j)
                        if (j != i) prod *= qM[j];
                    sum += prod;
                }
            }
            acc += acell[s.cell_off + ci] * sum;
        }
        int j = 0;
        while (j < D && ++ctr[j] == nm[j]) { ctr[j] = 0; ++j; }
        if (j == D) break;
    }
    diag[k] = acc;
}


// ----------------------------------------------------------------------------- learned diagonal
// Features of point k for the diagonal MLP (F = 7d + 5): depths t_j / 8,
// coordinates x_j, next-to-boundary flags, log a(x), sum_j t_j / (8 d), the
// log-coefficient differences log a(x +- h_j e_j) - log a(x), h_j = 2^-t_j,
// whether the same-depth points two level steps left / right exist (nbmask),
// and mean / min / max of log a - log a(x) over the 2^d surrounding cell midpoints.
__global__ void k_features(DevPlan P, int family, const double* __restrict__ params, const uint16_t* __restrict__ nbmask,
                           float* __restrict__ feat) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= P.n) return;
    int d = P.d, F = 7 * d + 5;
    float* f = feat + k * F;
    double x[lsg::kMaxDim], h[lsg::kMaxDim];
    int tsum = 0;
    for (int j = 0; j < d; ++j) {
        int32_t idx = P.pts[k * d + j];
        int t = 31 - __clz(idx);
        int64_t c = 2 * (int64_t)(idx - (1 << t)) + 1;
        h[j] = ldexp(1.0, -t);
        x[j] = (double)c * h[j];
        bool nb = (c - 1 == 0) || (c + 1 == ((int64_t)1 << t));
        f[j] = t / 8.0f;
        f[d + j] = (float)x[j];
        f[2 * d + j] = nb ? 1.f : 0.f;
        tsum += t;
    }
    double la = log(fmax(lsg_coef_eval_dev(family, params, d, x), 1e-300));
    f[3 * d] = (float)la;
    f[3 * d + 1] = tsum / (8.0f * d);
    for (int j = 0; j < d; ++j) {
        double xs = x[j];
        x[j] = xs + h[j];
        f[3 * d + 2 + 2 * j] = (float)(log(fmax(lsg_coef_eval_dev(family, params, d, x), 1e-300)) - la);
        x[j] = xs - h[j];
        f[3 * d + 3 + 2 * j] = (float)(log(fmax(lsg_coef_eval_dev(family, params, d, x), 1e-300)) - la);
        x[j] = xs;
    }
    const uint16_t m = nbmask[k];
    for (int j = 0; j < 2 * d; ++j) f[5 * d + 2 + j] = ((m >> j) & 1) ? 1.f : 0.f;
    // log a at the midpoints of the 2^d level-T cells around the point (the
    // cells that weigh most in its diagonal): mean, min, max relative to log a(x)
    double sum = 0.0, lo = 1e300, hi = -1e300;
    for (int b = 0; b < (1 << d); ++b) {
        double xm[lsg::kMaxDim];
        for (int j = 0; j < d; ++j) xm[j] = x[j] + ((b >> j) & 1 ? 0.5 : -0.5) * h[j];
        double v = log(fmax(lsg_coef_eval_dev(family, params, d, xm), 1e-300)) - la;
        sum += v;
        lo = fmin(lo, v);
        hi = fmax(hi, v);
    }
    f[7 * d + 2] = (float)(sum / (1 << d));
    f[7 * d + 3] = (float)lo;
    f[7 * d + 4] = (float)hi;
}

// Cheap diagonal a(x_k) * psi_k^T K_ref psi_k for a constant coefficient on a
// complete level-T grid: per dimension the 1D sums over the six cells of the
// prewavelet support factorise the tensor sum (exact when a is constant and
// every cell exists).
__global__ void k_base_diag(DevPlan P, int family, const double* __restrict__ params, double* __restrict__ base) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= P.n) return;
    int d = P.d;
    if (!P.act[k]) { base[k] = 0.0; return; }
    double x[lsg::kMaxDim], sK[lsg::kMaxDim], sM[lsg::kMaxDim];
    for (int j = 0; j < d; ++j) {
        int32_t idx = P.pts[k * d + j];
        int t = 31 - __clz(idx);
        int64_t c = 2 * (int64_t)(idx - (1 << t)) + 1, top = (int64_t)1 << t;
        double h = ldexp(1.0, -t);
        x[j] = (double)c * h;
        bool lok = c - 1 > 0, rok = c + 1 < top;
        double w[7] = {0, 0, 0, 0, 0, 0, 0};
        w[3] = (t > 1 && (!lok || !rok)) ? 0.9 : 1.0;
        if (lok) { w[2] = -0.6; w[1] = 0.1; }
        if (rok) { w[4] = -0.6; w[5] = 0.1; }
        double a = 0, b = 0;
        for (int q = 0; q < 6; ++q) {
            int64_t m = c - 3 + q;
            if (m < 0 || m >= top) continue;
            double l = w[q], r = w[q + 1];
            a += (l - r) * (l - r) / h;
            b += h * (l * l + l * r + r * r) / 3.0;
        }
        sK[j] = a;
        sM[j] = b;
    }
    double sum = 0.0;
    for (int i = 0; i < d; ++i) {
        double prod = sK[i];
        for (int j = 0; j < d; ++j)
            if (j != i) prod *= sM[j];
        sum += prod;
    }
    base[k] = lsg_coef_eval_dev(family, params, d, x) * sum;
}

__global__ void k_install_learned(int64_t n, const uint8_t* __restrict__ act, const double* __restrict__ base,
                                  const float* __restrict__ out, double* __restrict__ diag) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    double o = out[k];
    double sp = o > 30.0 ? o : log1p(exp(o));
    diag[k] = act[k] ? base[k] * sp : 0.0;
}

// ----------------------------------------------------------------------------- vector kernels

constexpr int kRedBlocks = 592;  // 4 x 148 SMs
constexpr int kRedThreads = 256;

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) red[w] = v;
    __syncthreads();
    v = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    if (w == 0)
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    return v;
}

// partial dot products (FP64 accumulation), deterministic two-pass
template <typename A, typename B>
__global__ void k_dot_partial(const A* __restrict__ a, const B* __restrict__ b, int64_t n, double* __restrict__ part) {
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc += (double)a[i] * (double)b[i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}
__global__ void k_dot_final(const double* __restrict__ part, int np, double* __restrict__ out) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) acc += part[i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) *out = acc;
}

// scalars: s[0]=delta s[1]=dg s[2]=tau s[3]=delta_new s[4]=beta s[5]=rr s[6]=ff
__global__ void k_tau(double* s) { s[2] = s[0] / s[1]; }
__global__ void k_beta(double* s) { s[4] = s[3] / s[0]; s[0] = s[3]; }

// r += tau g ; x -= tau d   (all entries, ET semantics of cg_method.h:862-863)
template <typename V>
__global__ void k_update_rx(int64_t n, const double* s, V* r, V* x, const V* g, const V* d) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    V tau = (V)s[2];
    r[i] = r[i] + tau * g[i];
    x[i] = x[i] - tau * d[i];
}
// h = r (all) ; h /= z on active entries (apply_inverse, cg_method.h:717-727)
template <typename V>
__global__ void k_precond(int64_t n, const uint8_t* act, const V* r, const V* z, V* h, int all) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (act[i]) h[i] = z ? r[i] / z[i] : r[i];
    else if (all) h[i] = r[i];
}
// d = -h + beta d
template <typename V>
__global__ void k_update_d(int64_t n, const double* s, const V* h, V* d) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    d[i] = V(-1.0) * h[i] + (V)s[4] * d[i];
}
template <typename V>
__global__ void k_sub(int64_t n, const V* f, V* r) {  // r = f - r
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) r[i] = f[i] - r[i];
}
template <typename V>
__global__ void k_neg(int64_t n, const V* h, V* d) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) d[i] = V(-1.0) * h[i];
}
__global__ void k_scale_to_f32(int64_t n, const double* a, double scale, float* b) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)(a[i] * scale);
}
__global__ void k_axpy_f32(int64_t n, double alpha, const float* e, double* x) {  // x += alpha * e
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) x[i] += alpha * (double)e[i];
}
__global__ void k_to_f32(int64_t n, const double* a, float* b) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// ----------------------------------------------------------------------------- device buffer helper
struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~DBuf() { if (p) cudaFree(p); }
    int alloc(size_t b, size_t* total) {
        if (p) { cudaFree(p); p = nullptr; *total -= bytes; }
        bytes = b;
        if (b == 0) return 0;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) return fail(LSG_E_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        *total += b;
        return 0;
    }
    template <typename T>
    int upload(const std::vector<T>& v, size_t* total) {
        int rc = alloc(v.size() * sizeof(T), total);
        if (rc) return rc;
        if (!v.empty()) {
            cudaError_t e = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) return fail(LSG_E_CUDA, std::string("cudaMemcpy: ") + cudaGetErrorString(e));
        }
        return 0;
    }
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

}  // namespace

struct lsg_operator {
    lsg::Plan plan;
    DevPlan dp{};
    int device = 0;
    size_t dev_bytes = 0;
    // tables
    DBuf slabs, did, act, exa_off, exa, cell_key, cell_corner, nodal_stage, nodal_src, nodal_code, nodal_dom, nodal_scr,
        conv_stage, conv_src, conv_code, conv_dom, prol, restr, a_items, b_items, b_steps, pts, cell_slab_off,
        conv_off, conv_items_off, conv_items, sp_slot_off, sp_inc_base, sp_inc_off, sp_inc, a_chain_off, a_chain_items;
    std::vector<int32_t> a_dim_chain_off;  // per dimension: its chains [off[k], off[k+1])

    int64_t conv_total = 0;  // convert slots of one matvec
    int64_t sp_total = 0;    // cell slots of the sparse-slab items of one matvec
    DBuf lam64, lam32;   // Hadamard-basis eigenvalues of the Q1 stiffness (form 0)
    DBuf mu64, mu32;     // ... of the Q1 mass (form 1)
    DBuf one64, one32;   // unit coefficient per cell (constant-coefficient norms)
    bool unit_coef = false;  // matvec with coefficient 1 (set only inside matvec64_unit)
    int32_t form = 0;
    // coefficient (one family and parameter set per part of a concatenated plan)
    bool have_coef = false;
    int32_t family = 0;
    std::vector<uint8_t> part_coef;
    DBuf acell64, acell32, params;
    DBuf feat, mlp_out, base;  // learned-diagonal work buffers
    DBuf nbmask;               // same-depth neighbour flags (features)
    // work buffers per precision
    struct Work {
        DBuf ml, pc, zb, gm, scratch, nscratch, conv, sp;
    } w64, w32;
    DBuf xbuf64, ybuf64;  // host-call staging
    DBuf diag;            // Jacobi diagonal (FP64)
    bool have_diag = false;
    DBuf learned;
    bool have_learned = false;
    int64_t smem_cap64 = 0, smem_cap32 = 0;
    std::vector<int64_t> level_need;  // per phase-B level: largest vector of any item
    lsg_tuning tune{256, 72, 4, 256, 2048, 256};  // launch parameters (lsg_operator_autotune)
    std::shared_ptr<void> basis;      // basis-transform tables (lsg_basis.cu), built on first use
    std::shared_ptr<void> bdrhs;      // boundary right-hand-side tables (lsg_bdrhs.cu), built on first use
    // cell operator launch plan, per precision: the factorised dense-slab
    // operator k_sf (slab plans, item order, launch classes by work space) and
    // k_cells for the items of sparse slabs (order, classes by slab size)
    lsg::SfCoefLayout sf_layout;
    DBuf coll64, coll32, coll_off, coll_slab, slab_T, slab_cell_off;  // collapsed coefficients
    struct SfPrec {
        DBuf plans, order;
        std::vector<int32_t> class_off;    // k_sf launches (work-space classes)
        std::vector<int32_t> class_w;      // dynamic shared memory (bytes) of each launch
        std::vector<uint8_t> ok;  // per slab: the plan fits
        DBuf cstr;                // per (slab, dim): coefficient stride in this precision's order
        DBuf cell_order;
        std::vector<int32_t> cell_class_off;
        std::vector<int64_t> cell_class_n;
    } sf32, sf64;
};

namespace {

// Launch plan of the cell operator.  Dense slabs go to k_sf (planned per
// precision for a work space of tune.cell_space_kb, FP64 with half the
// elements) in work-space classes.  Items of sparse slabs go to k_cells by
// slab size in classes, with shared memory for N_T of the class's largest
// slab.  A new class (launch) starts when the size shrinks by
// tune.class_ratio.
int build_sf_prec(lsg_operator* op, lsg_operator::SfPrec& S, int64_t wcap, int na_max) {
    const lsg::Plan& p = op->plan;
    std::vector<lsg::SfSlab> plans = lsg::sf_plan(p, op->sf_layout, wcap, na_max);
    S.ok.assign(p.nD, 0);
    for (int t = 0; t < p.nD; ++t) {
        S.ok[t] = plans[t].nm >= 0;
        if (p.slabs[t].dense && !S.ok[t]) return fail(LSG_E_INVALID, "no factorised plan fits a dense slab");
    }
    // k_sf: items by work space, largest first, in classes (a new class,
    // i.e. launch, starts when the work space shrinks by tune.class_ratio);
    // each launch has thousands of items, which keeps every SM busy
    std::vector<int32_t> ord, cord;
    for (size_t i = 0; i < p.b_items.size(); ++i) (S.ok[p.b_items[i].t] ? ord : cord).push_back((int32_t)i);
    std::stable_sort(ord.begin(), ord.end(), [&](int32_t a, int32_t b) {
        return plans[p.b_items[a].t].wtotal > plans[p.b_items[b].t].wtotal;
    });
    S.class_off.clear();
    S.class_w.clear();
    {
        const size_t vb = (&S == &op->sf32) ? 4 : 8;
        int64_t bound = -1;
        for (size_t i = 0; i < ord.size(); ++i) {
            const lsg::SfSlab& D = plans[p.b_items[ord[i]].t];
            int64_t w = std::max(D.wtotal, 1);
            int64_t bytes = (int64_t)lsg::sf_smem_bytes(D, vb);
            if (bound < 0 || w * op->tune.class_ratio < bound) {
                S.class_off.push_back((int32_t)i);
                S.class_w.push_back((int32_t)bytes);
                bound = w;
            } else {
                S.class_w.back() = std::max<int32_t>(S.class_w.back(), (int32_t)bytes);
            }
        }
    }
    S.class_off.push_back((int32_t)ord.size());
    std::stable_sort(cord.begin(), cord.end(), [&](int32_t a, int32_t b) {
        return p.slabs[p.b_items[a].t].n > p.slabs[p.b_items[b].t].n;
    });
    S.cell_class_off.clear();
    S.cell_class_n.clear();
    int64_t bound = -1;
    for (size_t i = 0; i < cord.size(); ++i) {
        int64_t n = p.slabs[p.b_items[cord[i]].t].n;
        if (bound < 0 || n * op->tune.class_ratio < bound) {
            S.cell_class_off.push_back((int32_t)i);
            S.cell_class_n.push_back(n);
            bound = n;
        }
    }
    S.cell_class_off.push_back((int32_t)cord.size());
    std::vector<int32_t> cstr((size_t)p.nD * p.d, 0);
    for (int t = 0; t < p.nD; ++t)
        if (S.ok[t]) lsg::sf_cell_strides(p, t, plans[t], cstr.data() + (size_t)t * p.d);
    int rc = S.plans.upload(plans, &op->dev_bytes);
    if (!rc) rc = S.cstr.upload(cstr, &op->dev_bytes);
    if (!rc) rc = S.order.upload(ord, &op->dev_bytes);
    if (!rc) rc = S.cell_order.upload(cord, &op->dev_bytes);
    return rc ? LSG_E_CUDA : 0;
}

// Collapsed coefficients of one part's dense slabs (k_sf), in the order of the
// current FP64 and FP32 plans.
cudaError_t collapse_part(lsg_operator* op, int part) {
    const lsg::Plan& p = op->plan;
    int t_lo = p.inst_t_off[part], t_hi = p.inst_t_off[part + 1];
    int64_t lo = -1, hi = -1;
    for (int t = t_lo; t < t_hi; ++t) {
        int64_t o = op->sf_layout.coef_off[t];
        if (o < 0) continue;
        if (lo < 0) lo = o;
        int64_t c = 1;
        for (int k = 0; k < p.d; ++k)
            if (p.slabs[t].T[k] >= 2) c *= ((int64_t)1 << p.slabs[t].T[k]);
        hi = o + c;
    }
    if (lo >= 0 && hi > lo)
        k_sf_collapse<<<nblk(hi - lo), 256>>>(op->slab_T.as<int32_t>(), p.d, op->slab_cell_off.as<int64_t>(),
                                               op->coll_off.as<int64_t>(), op->coll_slab.as<int32_t>(), lo, hi,
                                               op->acell64.as<double>(), op->sf64.cstr.as<int32_t>(),
                                               op->sf32.cstr.as<int32_t>(), op->coll64.as<double>(),
                                               op->coll32.as<float>());
    return cudaGetLastError();
}

int build_cell_classes(lsg_operator* op) {
    const int64_t w32 = (int64_t)op->tune.cell_space_kb * 1024 / 4, w64 = (int64_t)op->tune.cell_space_kb * 1024 / 8;
    int rc = build_sf_prec(op, op->sf32, w32, 7);
    if (!rc) rc = build_sf_prec(op, op->sf64, w64, 3);
    if (rc) return rc;
    // new plans order the collapsed coefficients differently: redo the parts
    // whose coefficients are set
    for (size_t part = 0; part < op->part_coef.size(); ++part)
        if (op->part_coef[part]) CUDA_TRY(collapse_part(op, (int)part));
    return 0;
}

int upload_plan(lsg_operator* op) {
    const lsg::Plan& p = op->plan;
    size_t* tot = &op->dev_bytes;
    int d = p.d;
    std::vector<DevSlab> ds(p.nD);
    for (int t = 0; t < p.nD; ++t) {
        const lsg::Slab& s = p.slabs[t];
        DevSlab& o = ds[t];
        memset(&o, 0, sizeof o);
        o.off = s.off;
        o.n = s.n;
        o.cell_off = s.cell_off;
        o.ncell = s.ncell;
        o.corner_off = s.corner_off;
        o.dense = s.dense ? 1 : 0;
        int64_t stride = 1;
        for (int k = 0; k < d; ++k) {
            o.T[k] = s.T[k];
            o.ext[k] = (1 << s.T[k]) - 1;
            o.stride[k] = (int32_t)stride;
            stride *= o.ext[k];
        }
    }
    std::vector<int64_t> nscr(p.nD);
    int64_t acc = 0;
    for (int t = 0; t < p.nD; ++t) {
        nscr[t] = acc;
        for (int j = 1; j < d; ++j) acc += p.nodal_dom[t * (d + 1) + j];
    }
    std::vector<int64_t> cso(p.nD + 1);
    for (int t = 0; t < p.nD; ++t) cso[t] = p.slabs[t].cell_off;
    cso[p.nD] = p.C;
    int rc = 0;
    rc |= op->slabs.upload(ds, tot);
    rc |= op->did.upload(p.did, tot);
    rc |= op->act.upload(p.act, tot);
    rc |= op->exa_off.upload(p.exa_off, tot);
    rc |= op->exa.upload(p.exa, tot);
    rc |= op->cell_key.upload(p.cell_key, tot);
    rc |= op->cell_corner.upload(p.cell_corner, tot);
    rc |= op->nodal_stage.upload(p.nodal.stage_off, tot);
    rc |= op->nodal_src.upload(p.nodal.src, tot);
    rc |= op->nodal_code.upload(p.nodal.code, tot);
    rc |= op->nodal_dom.upload(p.nodal_dom, tot);
    rc |= op->nodal_scr.upload(nscr, tot);
    rc |= op->conv_stage.upload(p.convert.stage_off, tot);
    rc |= op->conv_src.upload(p.convert.src, tot);
    rc |= op->conv_code.upload(p.convert.code, tot);
    rc |= op->conv_dom.upload(p.convert_dom, tot);
    rc |= op->prol.upload(p.prol, tot);
    rc |= op->restr.upload(p.restr, tot);
    rc |= op->a_items.upload(p.a_items, tot);
    rc |= op->b_items.upload(p.b_items, tot);
    rc |= op->b_steps.upload(p.b_steps, tot);
    rc |= op->pts.upload(p.pts, tot);
    rc |= op->cell_slab_off.upload(cso, tot);
    {  // private convert slots per item and, per depth, the items that end there
        std::vector<int64_t> coff(std::max<size_t>(p.b_items.size(), 1), -1);
        std::vector<std::vector<int32_t>> per(p.nD);
        int64_t tot_slots = 0;
        for (size_t i = 0; i < p.b_items.size(); ++i) {
            int tc = p.b_items[i].t_conv;
            if (tc < 0) continue;
            coff[i] = tot_slots;
            tot_slots += p.exa_off[tc + 1] - p.exa_off[tc];
            per[tc].push_back((int32_t)i);
        }
        std::vector<int32_t> ioff(p.nD + 1, 0), items;
        for (int t = 0; t < p.nD; ++t) {
            ioff[t] = (int32_t)items.size();
            items.insert(items.end(), per[t].begin(), per[t].end());
        }
        ioff[p.nD] = (int32_t)items.size();
        if (items.empty()) items.push_back(0);
        op->conv_total = tot_slots;
        rc |= op->conv_off.upload(coff, tot);
        rc |= op->conv_items_off.upload(ioff, tot);
        rc |= op->conv_items.upload(items, tot);
    }
    {  // prolongation chains: per dimension, items linked source -> target within a case
        std::map<std::tuple<int, int, int>, int32_t> by_src;  // (case, source depth, dim) -> item
        std::set<std::tuple<int, int, int>> targets;
        for (size_t i = 0; i < p.a_items.size(); ++i) {
            const lsg::PhaseAItem& a = p.a_items[i];
            by_src[std::make_tuple(a.c, a.t_src, a.dim)] = (int32_t)i;
            targets.insert(std::make_tuple(a.c, a.t_dst, a.dim));
        }
        std::vector<int32_t> coff, citems;
        op->a_dim_chain_off.assign(d + 1, 0);
        for (int k = 0; k < d; ++k) {
            op->a_dim_chain_off[k] = (int32_t)coff.size();
            for (size_t i = 0; i < p.a_items.size(); ++i) {  // chain heads: not the target of another item
                const lsg::PhaseAItem& a = p.a_items[i];
                if (a.dim != k || targets.count(std::make_tuple(a.c, a.t_src, a.dim))) continue;
                coff.push_back((int32_t)citems.size());
                for (int32_t cur = (int32_t)i;;) {
                    citems.push_back(cur);
                    auto nx = by_src.find(std::make_tuple(a.c, p.a_items[cur].t_dst, k));
                    if (nx == by_src.end()) break;
                    cur = nx->second;
                }
            }
        }
        op->a_dim_chain_off[d] = (int32_t)coff.size();
        coff.push_back((int32_t)citems.size());
        if (citems.empty()) citems.push_back(0);
        rc |= op->a_chain_off.upload(coff, tot);
        rc |= op->a_chain_items.upload(citems, tot);
    }
    {  // sparse slabs: per item its cell slots; per entry its (cell, corner) slots in cell order
        const int nc = 1 << d;
        std::vector<int64_t> soff(std::max<size_t>(p.b_items.size(), 1), -1), base(p.nD, -1), ioff;
        std::vector<int32_t> inc;
        int64_t slots = 0;
        for (size_t i = 0; i < p.b_items.size(); ++i) {
            const lsg::Slab& sl = p.slabs[p.b_items[i].t];
            if (sl.dense) continue;
            soff[i] = slots;
            slots += sl.ncell * nc;
        }
        for (int t = 0; t < p.nD; ++t) {
            const lsg::Slab& sl = p.slabs[t];
            if (sl.dense) continue;
            base[t] = (int64_t)ioff.size();
            std::vector<std::vector<int32_t>> per(sl.n);
            for (int64_t c = 0; c < sl.ncell; ++c)
                for (int b = 0; b < nc; ++b) {
                    int32_t at = p.cell_corner[(size_t)(sl.corner_off + c) * nc + b];
                    if (at >= 0) per[at].push_back((int32_t)(c * nc + b));
                }
            int64_t run = (int64_t)inc.size();
            for (int64_t e = 0; e < sl.n; ++e) {
                ioff.push_back(run);
                inc.insert(inc.end(), per[e].begin(), per[e].end());
                run = (int64_t)inc.size();
            }
            ioff.push_back(run);
        }
        if (ioff.empty()) ioff.push_back(0);
        if (inc.empty()) inc.push_back(0);
        op->sp_total = slots;
        rc |= op->sp_slot_off.upload(soff, tot);
        rc |= op->sp_inc_base.upload(base, tot);
        rc |= op->sp_inc_off.upload(ioff, tot);
        rc |= op->sp_inc.upload(inc, tot);
    }
    if (rc) return LSG_E_CUDA;
    // Hadamard-basis eigenvalues of the Q1 element per depth, 1/2^d folded in
    int nc = 1 << d;
    std::vector<double> lam(p.nD * (size_t)nc), mu_t(lam.size());
    std::vector<float> lamf(lam.size()), muf_t(lam.size());
    for (int t = 0; t < p.nD; ++t) {
        double h[lsg::kMaxDim];
        for (int k = 0; k < d; ++k) h[k] = std::ldexp(1.0, -p.slabs[t].T[k]);
        for (int sgn = 0; sgn < nc; ++sgn) {
            double l = 0.0;
            for (int i = 0; i < d; ++i) {
                if (!((sgn >> i) & 1)) continue;
                double prod = 2.0 / h[i];
                for (int j = 0; j < d; ++j)
                    if (j != i) prod *= ((sgn >> j) & 1) ? h[j] / 6.0 : h[j] / 2.0;
                l += prod;
            }
            lam[(size_t)t * nc + sgn] = l / nc;
            lamf[(size_t)t * nc + sgn] = (float)(l / nc);
            double mu = 1.0;  // mass: M1 = (h/6)[[2,1],[1,2]] has eigenvalues h/2 (+) and h/6 (-)
            for (int j = 0; j < d; ++j) mu *= ((sgn >> j) & 1) ? h[j] / 6.0 : h[j] / 2.0;
            mu_t[(size_t)t * nc + sgn] = mu / nc;
            muf_t[(size_t)t * nc + sgn] = (float)(mu / nc);
        }
    }
    rc |= op->lam64.upload(lam, tot);
    rc |= op->lam32.upload(lamf, tot);
    rc |= op->mu64.upload(mu_t, tot);
    rc |= op->mu32.upload(muf_t, tot);
    if (rc) return LSG_E_CUDA;
    DevPlan& P = op->dp;
    P.d = d;
    P.nD = p.nD;
    P.n = p.n;
    P.slabs = op->slabs.as<DevSlab>();
    P.did = op->did.as<int32_t>();
    P.act = op->act.as<uint8_t>();
    P.exa_off = op->exa_off.as<int64_t>();
    P.exa = op->exa.as<int64_t>();
    P.cell_key = op->cell_key.as<uint64_t>();
    P.cell_corner = op->cell_corner.as<int32_t>();
    P.nodal_stage = op->nodal_stage.as<int64_t>();
    P.nodal_src = op->nodal_src.as<int32_t>();
    P.nodal_code = op->nodal_code.as<int32_t>();
    P.nodal_dom = op->nodal_dom.as<int64_t>();
    P.nodal_scr = op->nodal_scr.as<int64_t>();
    P.conv_stage = op->conv_stage.as<int64_t>();
    P.conv_src = op->conv_src.as<int32_t>();
    P.conv_code = op->conv_code.as<int32_t>();
    P.conv_dom = op->conv_dom.as<int64_t>();
    P.prol = op->prol.as<int32_t>();
    P.restr = op->restr.as<int32_t>();
    P.a_items = op->a_items.as<lsg::PhaseAItem>();
    P.b_items = op->b_items.as<lsg::PhaseBItem>();
    P.b_steps = op->b_steps.as<lsg::PhaseBStep>();
    P.pts = op->pts.as<int32_t>();
    P.a_chain_off = op->a_chain_off.as<int32_t>();
    P.a_chain_items = op->a_chain_items.as<int32_t>();
    P.sp_slot_off = op->sp_slot_off.as<int64_t>();
    P.sp_inc_base = op->sp_inc_base.as<int64_t>();
    P.sp_inc_off = op->sp_inc_off.as<int64_t>();
    P.sp_inc = op->sp_inc.as<int32_t>();
    P.conv_off = op->conv_off.as<int64_t>();
    P.conv_items_off = op->conv_items_off.as<int32_t>();
    P.conv_items = op->conv_items.as<int32_t>();
    // per-level largest vector of an item (dynamic shared memory of k_level)
    op->level_need.clear();
    for (size_t L = 0; L + 1 < p.b_level_off.size(); ++L) {
        int64_t mx = 0;
        for (int32_t i = p.b_level_off[L]; i < p.b_level_off[L + 1]; ++i) {
            const lsg::PhaseBItem& it = p.b_items[i];
            int64_t need = p.slabs[it.t].n;
            for (int32_t k = it.step_begin; k < it.step_end; ++k) need = std::max(need, p.b_steps[k].n_dst);
            if (it.t_conv >= 0)
                for (int j = 1; j < d; ++j) need = std::max(need, p.convert_dom[it.t_conv * (d + 1) + j]);
            mx = std::max(mx, need);
        }
        op->level_need.push_back(mx);
    }
    // collapsed coefficients of the dense slabs (k_sf): per slab its depths,
    // first cell and collapsed offset; per collapsed cell its slab
    op->sf_layout = lsg::sf_coef_layout(p);
    {
        const int64_t cc = std::max<int64_t>(op->sf_layout.ccount, 1);
        std::vector<int32_t> cslab(cc, 0);
        std::vector<int64_t> coff(p.nD + 1, 0), celloff(p.nD);
        for (int t = 0; t < p.nD; ++t) {
            celloff[t] = p.slabs[t].cell_off;
            coff[t] = op->sf_layout.coef_off[t] < 0 ? 0 : op->sf_layout.coef_off[t];
        }
        for (int t = 0; t < p.nD; ++t) {
            int64_t o = op->sf_layout.coef_off[t];
            if (o < 0) continue;
            int64_t c = 1;
            for (int k = 0; k < d; ++k)
                if (p.slabs[t].T[k] >= 2) c *= ((int64_t)1 << p.slabs[t].T[k]);
            std::fill(cslab.begin() + o, cslab.begin() + o + c, t);
        }
        std::vector<int32_t> sT(p.nD * (size_t)d);
        for (int t = 0; t < p.nD; ++t)
            for (int k = 0; k < d; ++k) sT[(size_t)t * d + k] = p.slabs[t].T[k];
        rc |= op->coll_slab.upload(cslab, tot);
        rc |= op->coll_off.upload(coff, tot);
        rc |= op->slab_T.upload(sT, tot);
        rc |= op->slab_cell_off.upload(celloff, tot);
        rc |= op->coll64.alloc(cc * sizeof(double), tot);
        rc |= op->coll32.alloc(cc * sizeof(float), tot);
        if (rc) return LSG_E_CUDA;
    }
    return build_cell_classes(op);
}

// per-cell coefficient the cell operator multiplies by
template <typename V>
const V* cell_coef(const lsg_operator* op) {
    if (std::is_same<V, double>::value) return (const V*)(op->unit_coef ? op->one64.p : op->acell64.p);
    return (const V*)(op->unit_coef ? op->one32.p : op->acell32.p);
}

template <typename V>
int ensure_work(lsg_operator* op, lsg_operator::Work& w) {
    if (w.ml.p) return 0;
    const lsg::Plan& p = op->plan;
    size_t* tot = &op->dev_bytes;
    int rc = 0;
    rc |= w.ml.alloc(p.M * sizeof(V), tot);
    rc |= w.pc.alloc(p.p_total * sizeof(V), tot);
    rc |= w.zb.alloc(p.p_total * sizeof(V), tot);
    rc |= w.gm.alloc(p.gm_total * sizeof(V), tot);
    rc |= w.scratch.alloc(std::max<int64_t>(p.scratch_total, 1) * sizeof(V), tot);
    rc |= w.nscratch.alloc(std::max<int64_t>(p.nodal_scratch, 1) * sizeof(V), tot);
    rc |= w.conv.alloc(std::max<int64_t>(op->conv_total, 1) * sizeof(V), tot);
    rc |= w.sp.alloc(std::max<int64_t>(op->sp_total, 1) * sizeof(V), tot);
    return rc ? LSG_E_CUDA : 0;
}

// Dynamic shared memory above 48 KB needs an opt-in per kernel and device;
// both precisions are set on the first call for a dimension on a device, so
// that no attribute call happens later (e.g. inside a stream capture).
template <int D>
int set_phaseB_smem() {
    static bool done[256] = {};
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return fail(LSG_E_INVALID, "device ordinal out of range");
    if (done[dev]) return 0;
    CUDA_TRY(cudaFuncSetAttribute(k_cells<D, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_cells<D, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_level<D, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_level<D, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_sf<float, 7>, cudaFuncAttributeMaxDynamicSharedMemorySize, 210 * 1024));
    CUDA_TRY(cudaFuncSetAttribute(k_sf<double, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 210 * 1024));
    done[dev] = true;
    return 0;
}

// Phase B: the cell operator (k_cells per sparse size class, k_sf per
// work-space class), one k_level per restriction wavefront, the gather into y.
template <int D, typename V>
int phaseB_launch(lsg_operator* op, const V* pc, V* zb, V* gm, V* scratch, V* conv, V* sp, V* y, const V* acell,
                  const V* lam, cudaStream_t st, cudaEvent_t ev_cells = nullptr) {
    const lsg::Plan& p = op->plan;
    constexpr bool F32 = std::is_same<V, float>::value;
    const lsg_operator::SfPrec& S = F32 ? op->sf32 : op->sf64;
    const V* coll = F32 ? (const V*)op->coll32.p : (const V*)op->coll64.p;
    // the cell operator: sparse slabs (few, small), then k_sf per work-space class
    const int64_t cap_elems = (200 * 1024) / sizeof(V) - (1 << D);
    for (size_t c = 0; c + 1 < S.cell_class_off.size(); ++c) {
        int32_t b = S.cell_class_off[c], e = S.cell_class_off[c + 1];
        int64_t need = S.cell_class_n[c];
        int64_t alloc = need <= cap_elems ? need : 0;
        size_t smem = (size_t)((1 << D) + alloc) * sizeof(V);
        k_cells<D, V><<<e - b, op->tune.cell_threads, smem, st>>>(op->dp, pc, zb, acell, lam,
                                                                  S.cell_order.as<int32_t>(), b, alloc, sp);
    }
    for (size_t c = 0; c + 1 < S.class_off.size(); ++c) {
        int32_t b = S.class_off[c], e = S.class_off[c + 1];
        size_t smem = (size_t)S.class_w[c];
        if (F32)
            k_sf<float, 7><<<e - b, op->tune.cell_threads, smem, st>>>(
                op->b_items.as<lsg::PhaseBItem>(), S.plans.as<lsg::SfSlab>(), (const float*)pc, (float*)zb,
                (const float*)coll, S.order.as<int32_t>(), b, op->unit_coef ? 1 : 0, op->form);
        else
            k_sf<double, 3><<<e - b, op->tune.cell_threads, smem, st>>>(
                op->b_items.as<lsg::PhaseBItem>(), S.plans.as<lsg::SfSlab>(), (const double*)pc, (double*)zb,
                (const double*)coll, S.order.as<int32_t>(), b, op->unit_coef ? 1 : 0, op->form);
    }
    if (ev_cells) cudaEventRecord(ev_cells, st);
    // restriction wavefronts, then every active entry of y from the convert slots
    const int64_t lvl_cap = std::min<int64_t>(op->tune.level_cap, (110 * 1024) / sizeof(V));
    for (size_t L = 0; L + 1 < p.b_level_off.size(); ++L) {
        int32_t b = p.b_level_off[L], e = p.b_level_off[L + 1];
        if (e <= b) continue;
        int64_t bufn = std::min<int64_t>(op->level_need[L], lvl_cap);
        k_level<D, V><<<e - b, op->tune.level_threads, 2 * bufn * sizeof(V), st>>>(op->dp, zb, gm, scratch, conv, b, bufn);
    }
    int64_t na = p.exa_off[p.nD];
    if (na > 0) k_conv_gather<V><<<nblk(na), 256, 0, st>>>(op->dp, na, conv, y);
    CUDA_TRY(cudaGetLastError());
    return 0;
}

// The matvec: a fixed sequence of launches on one stream.
template <int D, typename V>
int matvec_impl(lsg_operator* op, const V* x, V* y, cudaStream_t st, cudaEvent_t* ev = nullptr) {
    const lsg::Plan& p = op->plan;
    lsg_operator::Work& w = std::is_same<V, double>::value ? op->w64 : op->w32;
    int rc = ensure_work<V>(op, w);
    if (rc) return rc;
    rc = set_phaseB_smem<D>();
    if (rc) return rc;
    const V* acell = cell_coef<V>(op);
    const V* lam = std::is_same<V, double>::value ? (const V*)(op->form ? op->mu64.p : op->lam64.p)
                                                  : (const V*)(op->form ? op->mu32.p : op->lam32.p);
    if (ev) cudaEventRecord(ev[0], st);
    k_nodal<V><<<p.nD, 256, 0, st>>>(op->dp, x, w.ml.as<V>(), w.nscratch.as<V>());
    if (ev) cudaEventRecord(ev[1], st);
    int32_t nb = (int32_t)p.b_items.size();
    if (nb > 0) k_pinit<V><<<nb, 256, 0, st>>>(op->dp, w.ml.as<V>(), w.pc.as<V>(), 0);
    if (ev) cudaEventRecord(ev[2], st);
    for (int k = 0; k < p.d; ++k) {
        int32_t b = op->a_dim_chain_off[k], e = op->a_dim_chain_off[k + 1];
        if (e > b) k_prolong<V><<<e - b, op->tune.prolong_threads, 0, st>>>(op->dp, w.pc.as<V>(), b);
    }
    if (ev) cudaEventRecord(ev[3], st);
    rc = phaseB_launch<D, V>(op, w.pc.as<V>(), w.zb.as<V>(), w.gm.as<V>(), w.scratch.as<V>(), w.conv.as<V>(),
                             w.sp.as<V>(), y, acell, lam, st, ev ? ev[4] : nullptr);
    if (rc) return rc;
    if (ev) cudaEventRecord(ev[5], st);
    CUDA_TRY(cudaGetLastError());
    return 0;
}

template <int D, typename V>
int prepare_impl(lsg_operator* op) {
    lsg_operator::Work& w = std::is_same<V, double>::value ? op->w64 : op->w32;
    int rc = ensure_work<V>(op, w);
    if (rc) return rc;
    return set_phaseB_smem<D>();
}

// allocations and function attributes that must not happen during graph capture
template <typename V>
int prepare(lsg_operator* op) {
    switch (op->plan.d) {
    case 1: return prepare_impl<1, V>(op);
    case 2: return prepare_impl<2, V>(op);
    case 3: return prepare_impl<3, V>(op);
    case 4: return prepare_impl<4, V>(op);
    case 5: return prepare_impl<5, V>(op);
    case 6: return prepare_impl<6, V>(op);
    case 7: return prepare_impl<7, V>(op);
    case 8: return prepare_impl<8, V>(op);
    }
    return fail(LSG_E_INVALID, "unsupported dimension");
}

template <typename V>
int matvec_dispatch(lsg_operator* op, const V* x, V* y, cudaStream_t st, cudaEvent_t* ev = nullptr) {
    switch (op->plan.d) {
    case 1: return matvec_impl<1, V>(op, x, y, st, ev);
    case 2: return matvec_impl<2, V>(op, x, y, st, ev);
    case 3: return matvec_impl<3, V>(op, x, y, st, ev);
    case 4: return matvec_impl<4, V>(op, x, y, st, ev);
    case 5: return matvec_impl<5, V>(op, x, y, st, ev);
    case 6: return matvec_impl<6, V>(op, x, y, st, ev);
    case 7: return matvec_impl<7, V>(op, x, y, st, ev);
    case 8: return matvec_impl<8, V>(op, x, y, st, ev);
    }
    return fail(LSG_E_INVALID, "unsupported dimension");
}

int compute_diag(lsg_operator* op, cudaStream_t st) {
    if (!op->have_coef) return fail(LSG_E_STATE, "no coefficient set");
    if (!op->diag.p) {
        int rc = op->diag.alloc(op->plan.n * sizeof(double), &op->dev_bytes);
        if (rc) return rc;
    }
    unsigned g = nblk(op->plan.n, 128);
    const double* a = op->acell64.as<double>();
    double* dg = op->diag.as<double>();
    switch (op->plan.d) {
    case 1: k_diag<1><<<g, 128, 0, st>>>(op->dp, a, dg, op->form); break;
    case 2: k_diag<2><<<g, 128, 0, st>>>(op->dp, a, dg, op->form); break;
    case 3: k_diag<3><<<g, 128, 0, st>>>(op->dp, a, dg, op->form); break;
    case 4: k_diag<4><<<g, 128, 0, st>>>(op->dp, a, dg, op->form); break;
    case 5: k_diag<5><<<g, 128, 0, st>>>(op->dp, a, dg, op->form); break;
    case 6: k_diag<6><<<g, 128, 0, st>>>(op->dp, a, dg, op->form); break;
    case 7: k_diag<7><<<g, 128, 0, st>>>(op->dp, a, dg, op->form); break;
    case 8: k_diag<8><<<g, 128, 0, st>>>(op->dp, a, dg, op->form); break;
    }
    CUDA_TRY(cudaGetLastError());
    op->have_diag = true;
    return 0;
}

}  // namespace

// forward helpers used by the CG section
static int lsg_internal_matvec64(lsg_operator* op, const double* x, double* y, cudaStream_t st);
static int lsg_internal_matvec32(lsg_operator* op, const float* x, float* y, cudaStream_t st);
static const uint8_t* lsg_internal_active(lsg_operator* op);

// ============================================================================= C-ABI
__global__ void k_fill_one(int64_t n, double* a64, float* a32) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) { a64[i] = 1.0; a32[i] = 1.0f; }
}

namespace lsg_internal {

int create_from_plan(lsg::Plan&& plan, lsg_operator** out) {
    *out = nullptr;
    std::unique_ptr<lsg_operator> op(new lsg_operator());
    op->plan = std::move(plan);
    CUDA_TRY(cudaGetDevice(&op->device));
    op->part_coef.assign(op->plan.inst_n_off.size() - 1, 0);
    int rc = upload_plan(op.get());
    if (rc) return rc;
    *out = op.release();
    return 0;
}

int set_part_coefficient(lsg_operator* op, int part, int32_t family, const double* params, int32_t nparams) {
    if (!op) return fail(LSG_E_INVALID, "null operator");
    const lsg::Plan& p = op->plan;
    int nparts = (int)p.inst_n_off.size() - 1;
    if (part < 0 || part >= nparts) return fail(LSG_E_INVALID, "part index out of range");
    if (family < 0 || family > 4) return fail(LSG_E_INVALID, "unknown coefficient family");
    if (nparams < 0 || nparams > LSG_MAX_COEF_PARAMS || (nparams > 0 && !params))
        return fail(LSG_E_INVALID, "bad coefficient parameters");
    std::vector<double> pv(LSG_MAX_COEF_PARAMS, 0.0);
    for (int i = 0; i < nparams; ++i) pv[i] = params[i];
    size_t* tot = &op->dev_bytes;
    int rc = 0;
    if (!op->params.p) rc |= op->params.alloc((size_t)nparts * LSG_MAX_COEF_PARAMS * sizeof(double), tot);
    if (!op->acell64.p) {
        rc |= op->acell64.alloc(std::max<int64_t>(p.C, 1) * sizeof(double), tot);
        rc |= op->acell32.alloc(std::max<int64_t>(p.C, 1) * sizeof(float), tot);
    }
    if (rc) return LSG_E_CUDA;
    double* pp = op->params.as<double>() + (size_t)part * LSG_MAX_COEF_PARAMS;
    CUDA_TRY(cudaMemcpy(pp, pv.data(), pv.size() * sizeof(double), cudaMemcpyHostToDevice));
    int64_t c_lo = p.inst_c_off[part], c_hi = p.inst_c_off[part + 1];
    if (c_hi > c_lo)
        k_cell_coef<<<nblk(c_hi - c_lo), 256>>>(op->dp, c_lo, c_hi, p.inst_t_off[part], p.inst_t_off[part + 1], family,
                                                pp, op->acell64.as<double>(), op->acell32.as<float>(),
                                                op->cell_slab_off.as<int64_t>());
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(collapse_part(op, part));
    CUDA_TRY(cudaDeviceSynchronize());
    op->part_coef[part] = 1;
    op->have_coef = std::all_of(op->part_coef.begin(), op->part_coef.end(), [](uint8_t v) { return v != 0; });
    op->family = family;
    op->have_diag = false;
    return 0;
}

int matvec64(lsg_operator* op, const double* x, double* y, cudaStream_t st) { return matvec_dispatch<double>(op, x, y, st); }
int matvec32(lsg_operator* op, const float* x, float* y, cudaStream_t st) { return matvec_dispatch<float>(op, x, y, st); }
int prepare_precision(lsg_operator* op, bool fp32) {
    int rc = prepare<double>(op);
    if (!rc && fp32) rc = prepare<float>(op);
    return rc;
}
const uint8_t* active(lsg_operator* op) { return op->act.as<uint8_t>(); }
int jacobi_diag(lsg_operator* op, cudaStream_t st, const double** diag) {
    int rc = op->have_diag ? 0 : compute_diag(op, st);
    *diag = op->diag.as<double>();
    return rc;
}
bool has_coefficient(const lsg_operator* op) { return op->have_coef; }
const lsg::Plan& plan(const lsg_operator* op) { return op->plan; }
size_t device_bytes(const lsg_operator* op) { return op->dev_bytes; }
int64_t matvec_launch_count(const lsg_operator* op, bool f32) {
    const lsg::Plan& p = op->plan;
    const lsg_operator::SfPrec& S = f32 ? op->sf32 : op->sf64;
    int64_t prol = 0;
    for (int k = 0; k < p.d; ++k) prol += op->a_dim_chain_off[k + 1] > op->a_dim_chain_off[k];
    int64_t lv = 0;
    for (size_t L = 0; L + 1 < p.b_level_off.size(); ++L) lv += p.b_level_off[L + 1] > p.b_level_off[L];
    // nodal, P init, prolongation, cell operator (k_sf classes, k_cells classes), wavefronts, gather
    return 2 + prol + (int64_t)S.class_off.size() - 1 + (int64_t)S.cell_class_off.size() - 1 + lv +
           (p.exa_off[p.nD] > 0 ? 1 : 0);
}
int fail_msg(int code, const char* msg) { return fail(code, msg); }

// y = A x with coefficient 1 in the given form (Poisson / HelmHoltz of the
// norms), leaving the operator's own coefficient and form in place
int matvec64_unit(lsg_operator* op, int form, const double* x, double* y, cudaStream_t st) {
    const int64_t C = std::max<int64_t>(op->plan.C, 1);
    if (!op->one64.p) {
        if (op->one64.alloc(C * sizeof(double), &op->dev_bytes) || op->one32.alloc(C * sizeof(float), &op->dev_bytes))
            return LSG_E_CUDA;
        k_fill_one<<<nblk(C), 256, 0, st>>>(C, op->one64.as<double>(), op->one32.as<float>());
    }
    int rc = prepare<double>(op);
    if (rc) return rc;
    const int32_t f0 = op->form;
    op->form = form;
    op->unit_coef = true;
    rc = matvec_dispatch<double>(op, x, y, st);
    op->unit_coef = false;
    op->form = f0;
    return rc;
}
std::shared_ptr<void>& basis_slot(lsg_operator* op) { return op->basis; }
std::shared_ptr<void>& bdrhs_slot(lsg_operator* op) { return op->bdrhs; }
int autotune(lsg_operator* op, int32_t precision, int32_t reps) {
    return lsg_operator_autotune(op, precision, reps, nullptr, nullptr, nullptr);
}

}  // namespace lsg_internal

extern "C" {

const char* lsg_last_error(void) { return g_err.c_str(); }

int lsg_operator_create(int32_t d, const int32_t* points, const uint8_t* active, int64_t n, lsg_operator** out) {
    if (!out || !points || !active) return fail(LSG_E_INVALID, "null argument");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return fail(LSG_E_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
    lsg::Plan plan;
    if (!lsg::build_plan(d, n, points, active, plan)) return fail(LSG_E_INVALID, plan.error);
    return lsg_internal::create_from_plan(std::move(plan), out);
}

void lsg_operator_destroy(lsg_operator* op) { delete op; }

int lsg_operator_info(const lsg_operator* op, lsg_info* info) {
    if (!op || !info) return fail(LSG_E_INVALID, "null argument");
    const lsg::Plan& p = op->plan;
    memset(info, 0, sizeof *info);
    info->d = p.d;
    info->n_points = p.n;
    info->n_active = p.exa_off[p.nD];
    info->n_depths = p.nD;
    info->n_slab_entries = p.M;
    info->n_cells = p.C;
    int64_t cse = 0, cc = 0;
    for (int c = 0; c < p.ncase; ++c)
        for (int t : p.sorted[c]) { cse += p.slabs[t].n; cc += p.slabs[t].ncell; }
    info->case_slab_entries = cse;
    info->case_cells = cc;
    info->device_bytes = (int64_t)op->dev_bytes;
    info->plan_seconds = p.plan_seconds;
    // algorithmic bytes of one FP64 matvec: x in, y out, nodal slabs, per-case
    // P/gM/z slab traffic (3 passes), per-cell coefficient, corner tables of
    // sparse slabs (read once per case item)
    double s = 8.0;
    double bytes = s * 2.0 * p.n + s * p.M + s * 3.0 * cse + s * cc;
    int64_t sparse_cells = 0;
    for (int c = 0; c < p.ncase; ++c)
        for (int t : p.sorted[c])
            if (!p.slabs[t].dense) sparse_cells += p.slabs[t].ncell;
    bytes += 4.0 * (double)(1 << p.d) * sparse_cells;
    info->matvec_bytes_fp64 = bytes;
    info->matvec_flops = (double)cc * ((double)(2 * p.d + 2) * (1 << p.d));
    return 0;
}

int lsg_operator_set_coefficient(lsg_operator* op, int32_t family, const double* params, int32_t nparams) {
    if (!op) return fail(LSG_E_INVALID, "null operator");
    int nparts = (int)op->plan.inst_n_off.size() - 1;
    for (int b = 0; b < nparts; ++b) {
        int rc = lsg_internal::set_part_coefficient(op, b, family, params, nparams);
        if (rc) return rc;
    }
    return 0;
}

int lsg_matvec_device(lsg_operator* op, const void* x, void* y, int32_t precision, void* stream) {
    if (!op || !x || !y) return fail(LSG_E_INVALID, "null argument");
    if (!op->have_coef) return fail(LSG_E_STATE, "no coefficient set");
    cudaStream_t st = (cudaStream_t)stream;
    if (precision == LSG_FP64) return matvec_dispatch<double>(op, (const double*)x, (double*)y, st);
    if (precision == LSG_FP32) return matvec_dispatch<float>(op, (const float*)x, (float*)y, st);
    return fail(LSG_E_INVALID, "precision must be LSG_FP64 or LSG_FP32");
}

// Kernel launches of one matvec in the given precision.
static int64_t matvec_launches(const lsg_operator* op, bool f32) { return lsg_internal::matvec_launch_count(op, f32); }

// Algorithmic bytes per phase of one matvec (value size sv): every array the
// phase must touch, counted once per item that touches it.

static void phase_bytes(const lsg_operator* op, double sv, double* b) {
    const lsg::Plan& p = op->plan;
    int d = p.d;
    double nodal = sv * (double)p.exa_off[p.nD] + sv * (double)p.M;  // x gathered, nodal slabs written
    for (size_t i = 0; i < p.nodal.code.size(); ++i) nodal += 4.0 * (1 + p.nodal.nsrc);  // stage tables
    double pinit = 0, prol = 0, cell = 0, wave = 0;
    for (const auto& it : p.b_items) pinit += 2.0 * sv * p.slabs[it.t].n;
    for (const auto& a : p.a_items) prol += a.n_dst * (3.0 * sv + 8.0) + sv * p.slabs[a.t_src].n;
    const lsg::SfCoefLayout& L = op->sf_layout;
    for (const auto& it : p.b_items) {
        const lsg::Slab& s = p.slabs[it.t];
        // cell operator: slab read, slab written, coefficients (collapsed for k_sf)
        cell += 2.0 * sv * s.n;
        if (s.dense && L.coef_off[it.t] >= 0) {
            double c = 1;
            for (int k = 0; k < d; ++k)
                if (s.T[k] >= 2) c *= (double)((int64_t)1 << s.T[k]);
            cell += sv * c;
        } else {
            cell += sv * s.ncell + 4.0 * (1 << d) * s.ncell;  // per-cell coefficient, corner table
        }
        // wavefronts: z (+ gM) read, restriction tables and vectors, convert stages and slots
        wave += sv * s.n * (it.gm_prev ? 2.0 : 1.0);
        for (int32_t k = it.step_begin; k < it.step_end; ++k) {
            const lsg::PhaseBStep& st = p.b_steps[k];
            wave += st.n_dst * (12.0 + sv * (st.gm_prev ? 3.0 : 2.0)) + sv * st.n_src;
        }
        if (it.t_conv >= 0) {
            const int64_t* dom = &p.convert_dom[it.t_conv * (d + 1)];
            for (int j = 1; j <= d; ++j) wave += dom[j] * (24.0 + sv);
            wave += 2.0 * sv * dom[d];                          // slots written, gathered
        }
    }
    wave += sv * (double)p.exa_off[p.nD];                      // y
    b[0] = nodal;
    b[1] = pinit;
    b[2] = prol;
    b[3] = cell;
    b[4] = wave;
    b[5] = nodal + pinit + prol + cell + wave;
}

// Floating-point operations of the cell operator as the kernels issue them:
// k_sf per chunk (gather, mid sweeps, the fused a-b step per pencil plane,
// transposed sweeps, scatter), k_cells per cell (two Hadamard transforms and
// the scaling of 2^d corner values).
static double cell_op_flops(const lsg_operator* op, bool f32) {
    const lsg::Plan& p = op->plan;
    const lsg_operator::SfPrec& S = f32 ? op->sf32 : op->sf64;
    const std::vector<lsg::SfSlab> plans = lsg::sf_plan(p, op->sf_layout, (int64_t)op->tune.cell_space_kb * 1024 / (f32 ? 4 : 8),
                                                        f32 ? 7 : 3);
    double fl = 0.0;
    for (const auto& it : p.b_items) {
        if (S.ok[it.t]) {
            const lsg::SfSlab& D = plans[it.t];
            double ncomb = 1;
            for (int i = 0; i < D.nq; ++i) ncomb *= 2;
            double per = 2.0 * D.slice * ncomb;  // gather + scatter
            for (int k = 0; k < D.nm; ++k) per += D.stage[k + 1] + 1.5 * D.stage[k + 1];  // sweeps, both ways
            const double na = D.a.n, nb = D.b.n, ma = D.a.T < 0 ? 1 : 2 * na;
            double row = 2 * (na - 1) + 3 * na;           // E_a and E_a^T of one row
            double plane = nb * row + (nb - 1) * 9 * ma + 2 * 3 * ma;  // interior and boundary b cells
            per += D.npl * plane;
            fl += per * D.nchunk;
        } else {
            const int d = p.d, nc = 1 << d;
            fl += (double)p.slabs[it.t].ncell * ((2.0 * d + 1.0) * nc);
        }
    }
    return fl;
}

int lsg_matvec_profile(lsg_operator* op, const void* x, void* y, int32_t precision, int32_t iters, double* phase_ms,
                       double* bytes, double* flops) {
    if (!op || !x || !y || !phase_ms || iters < 1) return fail(LSG_E_INVALID, "bad argument");
    if (!op->have_coef) return fail(LSG_E_STATE, "no coefficient set");
    cudaEvent_t ev[6];
    for (auto& e : ev) cudaEventCreate(&e);
    double acc[6] = {0, 0, 0, 0, 0, 0};
    int rc = 0;
    for (int i = 0; i < iters && !rc; ++i) {
        rc = precision == LSG_FP64 ? matvec_dispatch<double>(op, (const double*)x, (double*)y, nullptr, ev)
                                   : matvec_dispatch<float>(op, (const float*)x, (float*)y, nullptr, ev);
        if (rc) break;
        cudaEventSynchronize(ev[5]);
        float ms;
        for (int k = 0; k < 5; ++k) {
            cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
            acc[k] += ms;
        }
        cudaEventElapsedTime(&ms, ev[0], ev[5]);
        acc[5] += ms;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (rc) return rc;
    for (int k = 0; k < 6; ++k) phase_ms[k] = acc[k] / iters;
    const bool f32 = precision != LSG_FP64;
    if (bytes) phase_bytes(op, f32 ? 4.0 : 8.0, bytes);
    if (flops) *flops = cell_op_flops(op, f32);
    return 0;
}

int lsg_matvec(lsg_operator* op, const double* x, double* y) {
    if (!op || !x || !y) return fail(LSG_E_INVALID, "null argument");
    size_t b = op->plan.n * sizeof(double);
    int rc = 0;
    if (!op->xbuf64.p) rc |= op->xbuf64.alloc(b, &op->dev_bytes);
    if (!op->ybuf64.p) rc |= op->ybuf64.alloc(b, &op->dev_bytes);
    if (rc) return LSG_E_CUDA;
    CUDA_TRY(cudaMemcpy(op->xbuf64.p, x, b, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(op->ybuf64.p, y, b, cudaMemcpyHostToDevice));  // hanging entries stay as given
    rc = lsg_matvec_device(op, op->xbuf64.p, op->ybuf64.p, LSG_FP64, nullptr);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpy(y, op->ybuf64.p, b, cudaMemcpyDeviceToHost));
    return 0;
}

int lsg_diag_device(lsg_operator* op, double* diag, void* stream) {
    if (!op || !diag) return fail(LSG_E_INVALID, "null argument");
    int rc = compute_diag(op, (cudaStream_t)stream);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(diag, op->diag.p, op->plan.n * sizeof(double), cudaMemcpyDeviceToDevice,
                             (cudaStream_t)stream));
    return 0;
}

int lsg_diag(lsg_operator* op, double* diag) {
    if (!op || !diag) return fail(LSG_E_INVALID, "null argument");
    int rc = compute_diag(op, nullptr);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpy(diag, op->diag.p, op->plan.n * sizeof(double), cudaMemcpyDeviceToHost));
    return 0;
}

int lsg_set_learned_diag(lsg_operator* op, const double* diag) {
    if (!op || !diag) return fail(LSG_E_INVALID, "null argument");
    if (!op->learned.p) {
        int rc = op->learned.alloc(op->plan.n * sizeof(double), &op->dev_bytes);
        if (rc) return rc;
    }
    CUDA_TRY(cudaMemcpy(op->learned.p, diag, op->plan.n * sizeof(double), cudaMemcpyHostToDevice));
    op->have_learned = true;
    return 0;
}

struct lsg_plan {
    lsg::Plan plan;
};

int lsg_plan_create(int32_t d, const int32_t* points, const uint8_t* active, int64_t n, lsg_plan** out) {
    if (!out || !points || !active) return fail(LSG_E_INVALID, "null argument");
    *out = nullptr;
    std::unique_ptr<lsg_plan> p(new lsg_plan());
    if (!lsg::build_plan(d, n, points, active, p->plan)) return fail(LSG_E_INVALID, p->plan.error);
    *out = p.release();
    return 0;
}
void lsg_plan_destroy(lsg_plan* p) { delete p; }

int lsg_plan_info(const lsg_plan* p, lsg_info* info) {
    if (!p || !info) return fail(LSG_E_INVALID, "null argument");
    lsg_operator tmp;  // info only needs the plan
    tmp.plan = p->plan;
    return lsg_operator_info(&tmp, info);
}
int lsg_plan_export_depths(const lsg_plan* p, int32_t* depths) {
    if (!p || !depths) return fail(LSG_E_INVALID, "null argument");
    memcpy(depths, p->plan.D.data(), p->plan.D.size() * sizeof(int32_t));
    return 0;
}
int lsg_plan_export_sorted_depths(const lsg_plan* p, int32_t c, int32_t* ids, int32_t* count) {
    if (!p || !ids || !count) return fail(LSG_E_INVALID, "null argument");
    if (c < 0 || c >= p->plan.ncase) return fail(LSG_E_INVALID, "case out of range");
    const auto& v = p->plan.sorted[c];
    memcpy(ids, v.data(), v.size() * sizeof(int32_t));
    *count = (int32_t)v.size();
    return 0;
}
int lsg_plan_export_cell_counts(const lsg_plan* p, int64_t* counts) {
    if (!p || !counts) return fail(LSG_E_INVALID, "null argument");
    for (int t = 0; t < p->plan.nD; ++t) counts[t] = p->plan.slabs[t].ncell;
    return 0;
}
int lsg_plan_check_slab_operator(const lsg_plan* p, int32_t t, int32_t form, int64_t wcap, int32_t na_max,
                                 const double* acell, const double* u, double* z_cells, double* z_sf, int32_t* info) {
    if (!p || !acell || !u || !z_cells || !z_sf) return fail(LSG_E_INVALID, "null argument");
    const lsg::Plan& P = p->plan;
    if (t < 0 || t >= P.nD) return fail(LSG_E_INVALID, "depth id out of range");
    if (!P.slabs[t].dense) return fail(LSG_E_INVALID, "the factorised operator covers dense slabs only");
    if (form != LSG_FORM_STIFFNESS && form != LSG_FORM_MASS) return fail(LSG_E_INVALID, "unknown operator form");
    lsg::cells_apply_host(P, t, form, acell, u, z_cells);
    lsg::SfCoefLayout L = lsg::sf_coef_layout(P);
    std::vector<lsg::SfSlab> sf = lsg::sf_plan(P, L, wcap, na_max);
    const lsg::SfSlab& D = sf[t];
    if (D.nm < 0) return fail(LSG_E_INVALID, "the slab's two innermost dimensions do not fit the work space");
    int64_t cc = 1;
    for (int k = 0; k < P.d; ++k)
        if (P.slabs[t].T[k] >= 2) cc *= ((int64_t)1 << P.slabs[t].T[k]);
    std::vector<double> coef(cc);
    lsg::sf_collapse_host(P, t, D, acell, coef.data());
    lsg::sf_apply_host(D, form, coef.data(), u, z_sf);
    if (info) {
        int ncol = 0;
        for (int k = 0; k < P.d; ++k) ncol += P.slabs[t].T[k] == 1;
        info[0] = D.nm;
        info[1] = D.nq;
        info[2] = D.nchunk;
        info[3] = D.a.T < 0 ? 0 : D.a.n;
        info[4] = D.b.T < 0 ? 0 : D.b.n;
        info[5] = ncol;
    }
    return 0;
}
int lsg_plan_export_slab(const lsg_plan* p, int32_t t, int64_t* idx, int64_t* count) {
    if (!p || !count) return fail(LSG_E_INVALID, "null argument");
    if (t < 0 || t >= p->plan.nD) return fail(LSG_E_INVALID, "depth id out of range");
    const lsg::Slab& s = p->plan.slabs[t];
    *count = s.n;
    if (idx) memcpy(idx, p->plan.slab_pt.data() + s.off, s.n * sizeof(int64_t));
    return 0;
}
int lsg_plan_export_cells(const lsg_plan* p, int32_t t, int64_t* corners, int64_t* count) {
    if (!p || !count) return fail(LSG_E_INVALID, "null argument");
    const lsg::Plan& P = p->plan;
    if (t < 0 || t >= P.nD) return fail(LSG_E_INVALID, "depth id out of range");
    const lsg::Slab& s = P.slabs[t];
    *count = s.ncell;
    if (!corners) return 0;
    int d = P.d, nc = 1 << d;
    int64_t ext[lsg::kMaxDim], stride[lsg::kMaxDim];
    int64_t st = 1;
    for (int k = 0; k < d; ++k) { ext[k] = ((int64_t)1 << s.T[k]) - 1; stride[k] = st; st *= ext[k]; }
    for (int64_t ci = 0; ci < s.ncell; ++ci) {
        for (int b = 0; b < nc; ++b) {
            int64_t pos;
            if (!s.dense) pos = P.cell_corner[(s.corner_off + ci) * nc + b];
            else {
                int64_t r = ci;
                pos = 0;
                for (int k = 0; k < d && pos >= 0; ++k) {
                    int64_t m = r % (ext[k] + 1);
                    r /= (ext[k] + 1);
                    int64_t c = m + ((b >> k) & 1);
                    if (c == 0 || c == ext[k] + 1) pos = -1;
                    else pos += (c - 1) * stride[k];
                }
            }
            corners[ci * nc + b] = pos < 0 ? -1 : P.slab_pt[s.off + pos];
        }
    }
    return 0;
}

static int64_t plan_lookup(const lsg::Plan& P, const int32_t* idx) {
    // a point of depth <= T lies in slab T; look it up in the slab of its own depth
    int d = P.d;
    int32_t T[lsg::kMaxDim];
    for (int k = 0; k < d; ++k) {
        if (idx[k] < 2) return -1;
        T[k] = lsg::depth1(idx[k]);
    }
    int t = -1;
    for (int u = 0; u < P.nD && t < 0; ++u) {
        bool eq = true;
        for (int k = 0; k < d; ++k) eq &= P.D[u * d + k] == T[k];
        if (eq) t = u;
    }
    if (t < 0) return -1;
    const lsg::Slab& s = P.slabs[t];
    uint64_t key = 0, st = 1;
    for (int k = 0; k < d; ++k) {
        int64_t c = 2 * (int64_t)(idx[k] - (1 << T[k])) + 1;
        key += (uint64_t)(c - 1) * st;
        st *= ((uint64_t)1 << T[k]) - 1;
    }
    const uint64_t* ks = P.slab_key.data() + s.off;
    const uint64_t* it = std::lower_bound(ks, ks + s.n, key);
    if (it == ks + s.n || *it != key) return -1;
    return P.slab_pt[s.off + (it - ks)];
}

int lsg_plan_export_neighbors(const lsg_plan* p, int64_t* nbr) {
    if (!p || !nbr) return fail(LSG_E_INVALID, "null argument");
    const lsg::Plan& P = p->plan;
    int d = P.d;
    for (int64_t k = 0; k < P.n; ++k) {
        int32_t J[lsg::kMaxDim];
        for (int j = 0; j < d; ++j) {
            for (int side = 0; side < 2; ++side) {
                memcpy(J, &P.pts[k * d], d * sizeof(int32_t));
                int32_t i = J[j];
                J[j] = side ? (i >> (__builtin_ctz(~(unsigned)i) + 1)) : (i >> (__builtin_ctz((unsigned)i) + 1));
                nbr[(k * d + j) * 2 + side] = plan_lookup(P, J);
            }
        }
    }
    return 0;
}

int lsg_plan_export_stencil(const lsg_plan* p, int64_t k, int64_t* idx, double* w, int32_t* count) {
    if (!p || !idx || !w || !count) return fail(LSG_E_INVALID, "null argument");
    const lsg::Plan& P = p->plan;
    if (k < 0 || k >= P.n) return fail(LSG_E_INVALID, "point out of range");
    int d = P.d;
    int32_t j1[lsg::kMaxDim][5];
    double w1[lsg::kMaxDim][5];
    int n1[lsg::kMaxDim];
    for (int j = 0; j < d; ++j) {
        int32_t i = P.pts[k * d + j];
        int t = lsg::depth1(i);
        int32_t l = i >> (__builtin_ctz((unsigned)i) + 1), r = i >> (__builtin_ctz(~(unsigned)i) + 1);
        bool lok = l > 1, rok = r > 1;
        int n = 0;
        j1[j][n] = i; w1[j][n++] = (t > 1 && (!lok || !rok)) ? 0.9 : 1.0;
        if (lok) { j1[j][n] = l; w1[j][n++] = -0.6; }
        if (rok) { j1[j][n] = r; w1[j][n++] = -0.6; }
        // next left/right on level t of the neighbour (index.h:834-866)
        if (lok) { int32_t x = l << 1; for (int q = 1; q < t - lsg::depth1(l); ++q) x = (x << 1) + 1; j1[j][n] = x; w1[j][n++] = 0.1; }
        if (rok) { int32_t x = (r << 1) + 1; for (int q = 1; q < t - lsg::depth1(r); ++q) x <<= 1; j1[j][n] = x; w1[j][n++] = 0.1; }
        n1[j] = n;
    }
    int pos[lsg::kMaxDim] = {0};
    int cnt = 0;
    for (;;) {
        int32_t J[lsg::kMaxDim];
        double val = 1.0;
        for (int j = 0; j < d; ++j) {
            J[j] = j1[j][pos[j]];
            double wj = w1[j][pos[j]];
            if (wj != 1.0) val = wj * val;  // the reference scales val in dimension order
        }
        idx[cnt] = plan_lookup(P, J);
        w[cnt] = val;
        ++cnt;
        int j = 0;
        while (j < d && ++pos[j] == n1[j]) { pos[j] = 0; ++j; }
        if (j == d) break;
    }
    *count = cnt;
    return 0;
}

}  // extern "C"

// ============================================================================= CG
namespace {

struct Pinned {
    double* h = nullptr;
    Pinned() { cudaMallocHost(&h, 16 * sizeof(double)); }
    ~Pinned() { if (h) cudaFreeHost(h); }
};

struct Solver {
    lsg_operator* op;
    int64_t n;
    size_t bytes = 0;
    DBuf r, g, d, h, part, s, ones;
    DBuf r32, g32, d32, h32, e32, z32;
    Pinned pin;
};

constexpr int kInnerStallWindow = 400;  // iterations without a 10 % residual gain

// Inner reduction of one refinement step, given the factor `need` (< 1) by
// which the residual still has to shrink: when this step can reach the target
// (need within 10x of itol) aim at `margin` x need -- 0.5 lands below the
// target with margin and costs little when need is large, and a step after
// one that fell short aims at 0.1 -- otherwise reduce by itol.
inline double inner_step_tol(double itol, double need, double margin) {
    double t = margin * need;
    return t >= 0.1 * itol ? std::min(0.5, std::max(t, 0.1 * itol)) : itol;
}

int solver_init(Solver& S, bool fp32, cudaStream_t st) {
    int64_t n = S.n;
    size_t* t = &S.bytes;
    int rc = 0;
    rc |= S.r.alloc(n * 8, t);
    rc |= S.g.alloc(n * 8, t);
    rc |= S.d.alloc(n * 8, t);
    rc |= S.h.alloc(n * 8, t);
    rc |= S.part.alloc(kRedBlocks * 8, t);
    rc |= S.s.alloc(16 * 8, t);
    if (fp32) {
        rc |= S.r32.alloc(n * 4, t);
        rc |= S.g32.alloc(n * 4, t);
        rc |= S.d32.alloc(n * 4, t);
        rc |= S.h32.alloc(n * 4, t);
        rc |= S.e32.alloc(n * 4, t);
        rc |= S.z32.alloc(n * 4, t);
    }
    if (rc) return LSG_E_CUDA;
    // every vector starts at zero (fresh VectorSparseG), hanging entries
    // included; zeroed on the solver's own stream, which does not wait for
    // work on the legacy default stream
    for (DBuf* b : {&S.r, &S.g, &S.d, &S.h, &S.s, &S.r32, &S.g32, &S.d32, &S.h32, &S.e32, &S.z32})
        if (b->p) CUDA_TRY(cudaMemsetAsync(b->p, 0, b->bytes, st));
    return 0;
}

// One CG iteration (CG::solveHomogen loop body, cg_method.h:852-879) with
// beta/d-update of the previous iteration moved to the front; the scalars
// live on the device so the body can be captured as a CUDA graph.
// s[0]=delta s[1]=dg s[2]=tau s[3]=delta_new s[4]=beta s[5]=rr
template <typename V>
int cg_body(Solver& S, V* x, V* r, V* g, V* d, V* h, const V* z, bool want_rr, cudaStream_t st) {
    int64_t n = S.n;
    double* s = S.s.as<double>();
    double* part = S.part.as<double>();
    k_beta<<<1, 1, 0, st>>>(s);
    k_update_d<V><<<nblk(n), 256, 0, st>>>(n, s, h, d);
    int rc = std::is_same<V, double>::value
                 ? lsg_internal_matvec64(S.op, (const double*)d, (double*)g, st)
                 : lsg_internal_matvec32(S.op, (const float*)d, (float*)g, st);
    if (rc) return rc;
    k_dot_partial<V, V><<<kRedBlocks, kRedThreads, 0, st>>>(d, g, n, part);
    k_dot_final<<<1, 1024, 0, st>>>(part, kRedBlocks, s + 1);
    k_tau<<<1, 1, 0, st>>>(s);
    k_update_rx<V><<<nblk(n), 256, 0, st>>>(n, s, r, x, g, d);
    k_precond<V><<<nblk(n), 256, 0, st>>>(n, lsg_internal_active(S.op), r, z, h, 1);
    k_dot_partial<V, V><<<kRedBlocks, kRedThreads, 0, st>>>(r, h, n, part);
    k_dot_final<<<1, 1024, 0, st>>>(part, kRedBlocks, s + 3);
    if (want_rr) {
        k_dot_partial<V, V><<<kRedBlocks, kRedThreads, 0, st>>>(r, r, n, part);
        k_dot_final<<<1, 1024, 0, st>>>(part, kRedBlocks, s + 5);
    }
    cudaMemcpyAsync(S.pin.h, s, 8 * sizeof(double), cudaMemcpyDeviceToHost, st);
    CUDA_TRY(cudaGetLastError());
    return 0;
}

// Runs CG on (x, r, ...) until the criterion holds.  r must hold f - A x and
// h, d, s[0], s[3] the start state.  Returns iterations in *its.
template <typename V>
int cg_loop(Solver& S, V* x, V* r, V* g, V* d, V* h, const V* z, double eps, int crit, double rr_stop, int maxit,
            bool use_graph, cudaStream_t st, int* its, double* last_rr, int64_t* launches, int stall_window = 0) {
    cudaGraphExec_t exec = nullptr;
    bool want_rr = crit == 1;
    int it = 0;
    int rc = 0;
    if (use_graph) {
        cudaGraph_t graph;
        CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        rc = cg_body<V>(S, x, r, g, d, h, z, want_rr, st);
        cudaError_t e = cudaStreamEndCapture(st, &graph);
        if (rc) return rc;
        if (e != cudaSuccess) return fail(LSG_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return fail(LSG_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    // loop condition of the first iteration (delta > eps, or the residual test)
    CUDA_TRY(cudaMemcpyAsync(S.pin.h, S.s.as<double>(), 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if ((crit == 0 && !(S.pin.h[0] > eps)) || (crit == 1 && S.pin.h[5] <= rr_stop)) maxit = 0;
    // stall_window > 0 (inner FP32 solves of the refinement): stop once the
    // recursive residual has not dropped below 0.9 x its best value for that
    // many iterations -- FP32 cannot reduce it further, the outer FP64
    // residual takes over.  The window is long because the 2-norm of a PCG
    // residual is not monotone: it can sit above its best for a hundred
    // iterations while the error still falls.
    double best = S.pin.h[5];
    int best_it = 0;
    for (int i = 1; i <= maxit; ++i) {
        if (use_graph) {
            cudaError_t e = cudaGraphLaunch(exec, st);
            if (e != cudaSuccess) { rc = fail(LSG_E_CUDA, cudaGetErrorString(e)); break; }
        } else {
            rc = cg_body<V>(S, x, r, g, d, h, z, want_rr, st);
            if (rc) break;
        }
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) { rc = fail(LSG_E_CUDA, cudaGetErrorString(e)); break; }
        it = i;
        double dn = S.pin.h[3];
        if (want_rr) *last_rr = S.pin.h[5];
        if (!std::isfinite(dn)) break;
        // reference: break when delta' < eps^2, and the loop runs while delta > eps
        // (cg_method.h:852,871) -- so it ends as soon as delta' <= eps as well
        if (crit == 0 && (dn < eps * eps || dn <= eps)) break;
        if (crit == 1 && S.pin.h[5] <= rr_stop) break;
        if (stall_window > 0) {
            if (S.pin.h[5] < 0.81 * best) { best = S.pin.h[5]; best_it = i; }
            else if (i - best_it >= stall_window) break;
        }
    }
    if (exec) cudaGraphExecDestroy(exec);
    *its = it;
    *launches += (int64_t)it * (matvec_launches(S.op, std::is_same<V, float>::value) + 9 + (want_rr ? 2 : 0));
    return rc;
}

template <typename V>
int cg_start(Solver& S, const V* f, V* x, V* r, V* d, V* h, const V* z, cudaStream_t st, bool x_zero = false) {
    int64_t n = S.n;
    double* s = S.s.as<double>();
    CUDA_TRY(cudaMemsetAsync(r, 0, n * sizeof(V), st));
    // A x of an all-zero x is exactly zero: skip the product
    int rc = x_zero ? 0
                    : std::is_same<V, double>::value ? lsg_internal_matvec64(S.op, (const double*)x, (double*)r, st)
                                                     : lsg_internal_matvec32(S.op, (const float*)x, (float*)r, st);
    if (rc) return rc;
    k_sub<V><<<nblk(n), 256, 0, st>>>(n, f, r);
    CUDA_TRY(cudaMemsetAsync(h, 0, n * sizeof(V), st));
    k_precond<V><<<nblk(n), 256, 0, st>>>(n, lsg_internal_active(S.op), r, z, h, 0);
    CUDA_TRY(cudaMemsetAsync(d, 0, n * sizeof(V), st));
    k_dot_partial<V, V><<<kRedBlocks, kRedThreads, 0, st>>>(r, h, n, S.part.as<double>());
    k_dot_final<<<1, 1024, 0, st>>>(S.part.as<double>(), kRedBlocks, s + 0);
    CUDA_TRY(cudaMemcpyAsync(s + 3, s + 0, sizeof(double), cudaMemcpyDeviceToDevice, st));
    k_dot_partial<V, V><<<kRedBlocks, kRedThreads, 0, st>>>(r, r, n, S.part.as<double>());
    k_dot_final<<<1, 1024, 0, st>>>(S.part.as<double>(), kRedBlocks, s + 5);
    CUDA_TRY(cudaGetLastError());
    return 0;
}

double host_dot(Solver& S, const double* a, const double* b, cudaStream_t st) {
    k_dot_partial<double, double><<<kRedBlocks, kRedThreads, 0, st>>>(a, b, S.n, S.part.as<double>());
    k_dot_final<<<1, 1024, 0, st>>>(S.part.as<double>(), kRedBlocks, S.s.as<double>() + 8);
    cudaMemcpyAsync(S.pin.h + 8, S.s.as<double>() + 8, sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    return S.pin.h[8];
}

int solve_device(lsg_operator* op, const double* f, double* x, const lsg_solver_opts* o, lsg_solve_report* rep,
                 cudaStream_t user_st) {
    if (!op || !f || !x || !o) return fail(LSG_E_INVALID, "null argument");
    if (!op->have_coef) return fail(LSG_E_STATE, "no coefficient set");
    cudaStream_t st;
    CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    cudaEvent_t ev0, ev1, evu;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    cudaEventCreate(&evu);
    cudaEventRecord(evu, user_st);
    cudaStreamWaitEvent(st, evu, 0);
    Solver S;
    S.op = op;
    S.n = op->plan.n;
    int64_t n = S.n;
    lsg_solve_report R;
    memset(&R, 0, sizeof R);
    int rc = solver_init(S, o->precision == LSG_FP32, st);
    if (!rc) rc = prepare<double>(op);
    if (!rc && o->precision == LSG_FP32) rc = prepare<float>(op);
    const double* zdiag = nullptr;
    if (!rc && o->precond == 0) { rc = compute_diag(op, st); zdiag = op->diag.as<double>(); }
    if (!rc && o->precond == 2) {
        if (!op->have_learned) rc = fail(LSG_E_STATE, "no learned diagonal installed");
        zdiag = op->learned.as<double>();
    }
    int maxit = o->max_iter > 0 ? o->max_iter : 500;
    double eps = o->eps;
    cudaEventRecord(ev0, st);
    double ff = rc ? 0.0 : host_dot(S, f, f, st);
    const bool x_zero = !rc && host_dot(S, x, x, st) == 0.0;  // zero initial guess (the common case)
    double final_rr = -1.0;  // FP64 residual of the final x when the refinement measured it
    if (!rc && o->precision == LSG_FP64) {
        DBuf x0;  // initial guess, kept for the fallback of a learned diagonal
        if (!rc && o->precond == 2) {
            size_t dummy = 0;
            rc = x0.alloc(n * sizeof(double), &dummy);
            if (!rc) CUDA_TRY(cudaMemcpyAsync(x0.p, x, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
        }
        if (!rc) rc = cg_start<double>(S, f, x, S.r.as<double>(), S.d.as<double>(), S.h.as<double>(), zdiag, st, x_zero);
        int its = 0;
        double rr = 0.0;
        if (!rc)
            rc = cg_loop<double>(S, x, S.r.as<double>(), S.g.as<double>(), S.d.as<double>(), S.h.as<double>(), zdiag, eps,
                                 o->criterion, eps * eps * ff, maxit, o->use_graph != 0, st, &its, &rr,
                                 &R.kernel_launches);
        R.iterations = its;
        R.outer_iterations = 1;
        // learned diagonal that stalled (not converged, or non-finite): continue
        // from the current iterate with the exact Jacobi diagonal
        bool stalled = !rc && o->precond == 2 &&
                       (o->criterion == 1 ? !(rr <= eps * eps * ff) : (its >= maxit || !std::isfinite(S.pin.h[3])));
        if (stalled) {
            R.fell_back = 1;
            // restart from the initial guess if the iterate was spoiled by non-finite values
            if (!std::isfinite(S.pin.h[3]) || !std::isfinite(rr))
                CUDA_TRY(cudaMemcpyAsync(x, x0.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
            rc = compute_diag(op, st);
            const double* zj = op->diag.as<double>();
            if (!rc) rc = cg_start<double>(S, f, x, S.r.as<double>(), S.d.as<double>(), S.h.as<double>(), zj, st);
            if (!rc)
                rc = cg_loop<double>(S, x, S.r.as<double>(), S.g.as<double>(), S.d.as<double>(), S.h.as<double>(), zj,
                                     eps, o->criterion, eps * eps * ff, maxit, o->use_graph != 0, st, &its, &rr,
                                     &R.kernel_launches);
            R.iterations += its;
        }
    } else if (!rc) {
        // FP32 inner CG inside FP64 iterative refinement
        int inner = o->inner_iter > 0 ? o->inner_iter : 1000;
        double itol = o->inner_tol > 0 ? o->inner_tol : 1e-5;
        float* z32 = nullptr;
        if (zdiag) {
            k_to_f32<<<nblk(n), 256, 0, st>>>(n, zdiag, S.z32.as<float>());
            z32 = S.z32.as<float>();
        }
        double* r = S.r.as<double>();
        int total = 0, outer = 0;
        double rr_prev = -1.0;
        int slow_steps = 0;
        for (outer = 0; outer < maxit && total < maxit; ++outer) {
            CUDA_TRY(cudaMemsetAsync(r, 0, n * 8, st));
            rc = (outer == 0 && x_zero) ? 0 : lsg_internal_matvec64(op, x, r, st);
            if (rc) break;
            k_sub<double><<<nblk(n), 256, 0, st>>>(n, f, r);
            double rr = host_dot(S, r, r, st);
            if (!std::isfinite(rr)) { rc = fail(LSG_E_NOCONV, "non-finite residual"); break; }
            if (rr <= eps * eps * ff) { final_rr = rr; break; }  // x is final: this is its residual
            // a refinement step that did not halve the residual with the learned
            // diagonal: switch to the exact Jacobi diagonal
            if (o->precond == 2 && !R.fell_back && rr_prev > 0 && rr > 0.25 * rr_prev) {
                R.fell_back = 1;
                rc = compute_diag(op, st);
                if (rc) break;
                k_to_f32<<<nblk(n), 256, 0, st>>>(n, op->diag.as<double>(), S.z32.as<float>());
                z32 = S.z32.as<float>();
            }
            // refinement that stopped making progress (six steps in a row that did not
            // halve the residual): give up
            if (rr_prev > 0 && rr > 0.25 * rr_prev) {
                if (++slow_steps >= 6) { rc = fail(LSG_E_NOCONV, "iterative refinement stagnated"); break; }
            } else {
                slow_steps = 0;
            }
            rr_prev = rr;
            double nr = std::sqrt(rr);
            float* r32 = S.r32.as<float>();
            float* e32 = S.e32.as<float>();
            k_scale_to_f32<<<nblk(n), 256, 0, st>>>(n, r, 1.0 / nr, r32);
            CUDA_TRY(cudaMemsetAsync(e32, 0, n * 4, st));
            // inner start: r32 already = rhs - A*0
            float* h32 = S.h32.as<float>();
            float* d32 = S.d32.as<float>();
            CUDA_TRY(cudaMemsetAsync(h32, 0, n * 4, st));
            k_precond<float><<<nblk(n), 256, 0, st>>>(n, lsg_internal_active(op), r32, z32, h32, 0);
            CUDA_TRY(cudaMemsetAsync(d32, 0, n * 4, st));
            double* s = S.s.as<double>();
            k_dot_partial<float, float><<<kRedBlocks, kRedThreads, 0, st>>>(r32, h32, n, S.part.as<double>());
            k_dot_final<<<1, 1024, 0, st>>>(S.part.as<double>(), kRedBlocks, s + 0);
            cudaMemcpyAsync(s + 3, s + 0, 8, cudaMemcpyDeviceToDevice, st);
            k_dot_partial<float, float><<<kRedBlocks, kRedThreads, 0, st>>>(r32, r32, n, S.part.as<double>());
            k_dot_final<<<1, 1024, 0, st>>>(S.part.as<double>(), kRedBlocks, s + 5);
            int its = 0;
            double lrr = 0.0;
            const double istep = inner_step_tol(itol, std::sqrt(eps * eps * ff / rr), slow_steps ? 0.1 : 0.5);
            rc = cg_loop<float>(S, e32, r32, S.g32.as<float>(), d32, h32, z32, 0.0, 1, istep * istep, inner,
                                o->use_graph != 0, st, &its, &lrr, &R.kernel_launches, kInnerStallWindow);
            R.kernel_launches += matvec_launches(op, true) + 12;
            if (rc) break;
            total += its;
            if (!std::isfinite(lrr) || !std::isfinite(S.pin.h[3])) {
                // the correction is unusable: drop it; with a learned diagonal switch to Jacobi
                if (o->precond == 2 && !R.fell_back) {
                    R.fell_back = 1;
                    rc = compute_diag(op, st);
                    if (rc) break;
                    k_to_f32<<<nblk(n), 256, 0, st>>>(n, op->diag.as<double>(), S.z32.as<float>());
                    z32 = S.z32.as<float>();
                    rr_prev = -1.0;
                    continue;
                }
                rc = fail(LSG_E_NOCONV, "non-finite inner residual");
                break;
            }
            k_axpy_f32<<<nblk(n), 256, 0, st>>>(n, nr, e32, x);
        }
        R.iterations = total;
        R.outer_iterations = outer;
    }
    cudaEventRecord(ev1, st);
    if (!rc) {
        // true relative residual in FP64 (the refinement's last residual when it
        // was taken of the final x)
        double rr = final_rr;
        if (rr < 0.0) {
            double* r = S.r.as<double>();
            cudaMemsetAsync(r, 0, n * 8, st);
            rc = lsg_internal_matvec64(op, x, r, st);
            if (!rc) {
                k_sub<double><<<nblk(n), 256, 0, st>>>(n, f, r);
                rr = host_dot(S, r, r, st);
            }
        }
        if (!rc) R.rel_residual = ff > 0 ? std::sqrt(rr / ff) : std::sqrt(rr);
    }
    cudaStreamSynchronize(st);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    R.seconds = ms * 1e-3;
    double target = o->criterion == 1 ? eps : 1e300;
    R.converged = (!rc && R.rel_residual <= target * 1.0000001) ? 1 : 0;
    if (o->criterion == 0 && !rc) R.converged = 1;
    cudaEventRecord(evu, st);
    cudaStreamWaitEvent(user_st, evu, 0);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    cudaEventDestroy(evu);
    cudaStreamDestroy(st);
    if (rep) *rep = R;
    return rc;
}

}  // namespace

extern "C" {

int lsg_cg_solve_device(lsg_operator* op, const double* f, double* x, const lsg_solver_opts* opts,
                        lsg_solve_report* rep, void* stream) {
    return solve_device(op, f, x, opts, rep, (cudaStream_t)stream);
}

int lsg_cg_solve(lsg_operator* op, const double* f, double* x, const lsg_solver_opts* opts, lsg_solve_report* rep) {
    if (!op || !f || !x || !opts) return fail(LSG_E_INVALID, "null argument");
    size_t b = op->plan.n * sizeof(double);
    DBuf fd, xd;
    size_t dummy = 0;
    if (fd.alloc(b, &dummy) || xd.alloc(b, &dummy)) return LSG_E_CUDA;
    CUDA_TRY(cudaMemcpy(fd.p, f, b, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(xd.p, x, b, cudaMemcpyHostToDevice));
    int rc = solve_device(op, fd.as<double>(), xd.as<double>(), opts, rep, nullptr);
    CUDA_TRY(cudaDeviceSynchronize());
    if (rc) return rc;
    CUDA_TRY(cudaMemcpy(x, xd.p, b, cudaMemcpyDeviceToHost));
    return 0;
}

}  // extern "C"

static int lsg_internal_matvec64(lsg_operator* op, const double* x, double* y, cudaStream_t st) {
    return matvec_dispatch<double>(op, x, y, st);
}
static int lsg_internal_matvec32(lsg_operator* op, const float* x, float* y, cudaStream_t st) {
    return matvec_dispatch<float>(op, x, y, st);
}
static const uint8_t* lsg_internal_active(lsg_operator* op) { return op->act.as<uint8_t>(); }

// ============================================================================= launch parameters, autotuner
namespace {

__global__ void k_pattern(int64_t n, double* x64, float* x32) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = (double)((i * 2654435761ull) % 1000003ull) / 1000003.0 - 0.5;
    if (x64) x64[i] = v;
    if (x32) x32[i] = (float)v;
}

bool tuning_valid(const lsg_tuning& t) {
    auto warps = [](int v, int lo, int hi) { return v >= lo && v <= hi && v % 32 == 0; };
    return warps(t.cell_threads, 64, 256) && t.cell_space_kb >= 16 && t.cell_space_kb <= 200 && t.class_ratio >= 2 &&
           t.class_ratio <= 1024 && warps(t.level_threads, 32, 512) && t.level_cap >= 256 && t.level_cap <= 65536 &&
           warps(t.prolong_threads, 32, 1024);
}

}  // namespace

extern "C" int lsg_operator_set_form(lsg_operator* op, int32_t form) {
    if (!op) return fail(LSG_E_INVALID, "null operator");
    if (form != LSG_FORM_STIFFNESS && form != LSG_FORM_MASS) return fail(LSG_E_INVALID, "unknown operator form");
    if (form != op->form) op->have_diag = false;
    op->form = form;
    return 0;
}

extern "C" int lsg_operator_get_tuning(const lsg_operator* op, lsg_tuning* t) {
    if (!op || !t) return fail(LSG_E_INVALID, "null argument");
    *t = op->tune;
    return 0;
}

extern "C" int lsg_operator_set_tuning(lsg_operator* op, const lsg_tuning* t) {
    if (!op || !t) return fail(LSG_E_INVALID, "null argument");
    if (!tuning_valid(*t)) return fail(LSG_E_INVALID, "launch parameters out of range");
    op->tune = *t;
    return build_cell_classes(op);
}

extern "C" int lsg_operator_autotune(lsg_operator* op, int32_t precision, int32_t reps, lsg_tuning* best,
                                     double* best_ms, double* default_ms) {
    if (!op) return fail(LSG_E_INVALID, "null operator");
    if (!op->have_coef) return fail(LSG_E_STATE, "no coefficient set");
    if (precision != LSG_FP64 && precision != LSG_FP32) return fail(LSG_E_INVALID, "bad precision");
    if (reps < 1) reps = 3;
    const bool f32 = precision == LSG_FP32;
    int rc = f32 ? prepare<float>(op) : prepare<double>(op);
    if (rc) return rc;
    int64_t n = op->plan.n;
    DBuf x, y;
    size_t dummy = 0, vs = f32 ? 4 : 8;
    if (x.alloc(n * vs, &dummy) || y.alloc(n * vs, &dummy)) return LSG_E_CUDA;
    k_pattern<<<nblk(n), 256>>>(n, f32 ? nullptr : x.as<double>(), f32 ? x.as<float>() : nullptr);
    CUDA_TRY(cudaMemset(y.p, 0, n * vs));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int err = 0;
    auto run = [&]() {
        return f32 ? matvec_dispatch<float>(op, x.as<float>(), y.as<float>(), 0)
                   : matvec_dispatch<double>(op, x.as<double>(), y.as<double>(), 0);
    };
    auto time_cfg = [&](const lsg_tuning& t) -> double {
        op->tune = t;
        if (build_cell_classes(op) || run()) { err = 1; return 1e30; }
        double bestt = 1e30;
        for (int r = 0; r < reps; ++r) {
            cudaEventRecord(e0, 0);
            if (run()) { err = 1; return 1e30; }
            cudaEventRecord(e1, 0);
            if (cudaEventSynchronize(e1) != cudaSuccess) { err = 1; return 1e30; }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            bestt = std::min(bestt, (double)ms);
        }
        return bestt;
    };
    const lsg_tuning start = op->tune;
    lsg_tuning cur = start;
    double cur_ms = time_cfg(cur), def_ms = cur_ms;
    const std::vector<std::pair<int32_t lsg_tuning::*, std::vector<int32_t>>> space = {
        {&lsg_tuning::cell_space_kb, {48, 72, 100}},  {&lsg_tuning::cell_threads, {128, 256}},
        {&lsg_tuning::class_ratio, {2, 4, 16}},       {&lsg_tuning::level_threads, {64, 128, 256, 512}},
        {&lsg_tuning::level_cap, {2048, 4096, 8192, 12288}}, {&lsg_tuning::prolong_threads, {128, 256, 512}}};
    for (int pass = 0; pass < 2 && !err; ++pass) {
        bool moved = false;
        for (const auto& dim : space) {
            for (int32_t v : dim.second) {
                if (cur.*(dim.first) == v) continue;
                lsg_tuning t = cur;
                t.*(dim.first) = v;
                double ms = time_cfg(t);
                if (err) break;
                if (ms < 0.99 * cur_ms) { cur = t; cur_ms = ms; moved = true; }
            }
            if (err) break;
        }
        if (!moved) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    op->tune = err ? start : cur;
    rc = build_cell_classes(op);
    if (err) return fail(LSG_E_CUDA, std::string("autotune: ") + (g_err.empty() ? "launch failed" : g_err));
    if (rc) return rc;
    if (best) *best = cur;
    if (best_ms) *best_ms = cur_ms;
    if (default_ms) *default_ms = def_ms;
    return 0;
}

// ============================================================================= allocation-free matvec
// Some callers cannot allocate device memory when they need a product: host
// applications whose own allocator owns every byte of the device and forbids
// foreign allocations, and latency-critical loops that cannot afford the
// implicit synchronisation of cudaMalloc/cudaFree.  For them
// lsg_matvec_device_noalloc takes its work space from one fixed array that is
// part of the library image on every GPU that loads it.
#define LSG_NOALLOC_SCRATCH_BYTES ((size_t)32 << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[LSG_NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_noalloc_mu;
void* g_noalloc_addr[256] = {nullptr};  // device address of g_noalloc_scratch, per device

// The array's host-side name is not a device address: resolve it once per
// device, with that device current.
int noalloc_address(unsigned char** out) {
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return fail(LSG_E_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(LSG_E_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
        g_noalloc_addr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_noalloc_addr[dev]);
    return 0;
}

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

template <int D, typename V>
int matvec_noalloc_impl(lsg_operator* op, const V* x, V* y, cudaStream_t st, unsigned char* base) {
    const lsg::Plan& p = op->plan;
    size_t b_ml = align256(p.M * sizeof(V)), b_pc = align256(p.p_total * sizeof(V));
    size_t b_zb = b_pc;
    size_t b_gm = align256(p.gm_total * sizeof(V));
    size_t b_sc = align256(std::max<int64_t>(p.scratch_total, 1) * sizeof(V));
    size_t b_ns = align256(std::max<int64_t>(p.nodal_scratch, 1) * sizeof(V));
    size_t b_cv = align256(std::max<int64_t>(op->conv_total, 1) * sizeof(V));
    size_t b_sp = align256(std::max<int64_t>(op->sp_total, 1) * sizeof(V));
    size_t need = b_ml + b_pc + b_zb + b_gm + b_sc + b_ns + b_cv + b_sp;
    if (need > LSG_NOALLOC_SCRATCH_BYTES)
        return fail(LSG_E_INVALID, "lsg_matvec_device_noalloc: this grid needs " + std::to_string(need) +
                                       " bytes of work space, the fixed array holds " +
                                       std::to_string(LSG_NOALLOC_SCRATCH_BYTES) +
                                       "; use lsg_matvec_device for larger grids");
    V* ml = reinterpret_cast<V*>(base);
    V* pc = reinterpret_cast<V*>(base + b_ml);
    V* zb = reinterpret_cast<V*>(base + b_ml + b_pc);
    V* gm = reinterpret_cast<V*>(base + b_ml + b_pc + b_zb);
    V* scratch = reinterpret_cast<V*>(base + b_ml + b_pc + b_zb + b_gm);
    V* nscratch = reinterpret_cast<V*>(base + b_ml + b_pc + b_zb + b_gm + b_sc);
    V* conv = reinterpret_cast<V*>(base + b_ml + b_pc + b_zb + b_gm + b_sc + b_ns);
    V* sp = reinterpret_cast<V*>(base + b_ml + b_pc + b_zb + b_gm + b_sc + b_ns + b_cv);
    int rc = set_phaseB_smem<D>();
    if (rc) return rc;
    const V* acell = cell_coef<V>(op);
    const V* lam = std::is_same<V, double>::value ? (const V*)(op->form ? op->mu64.p : op->lam64.p)
                                                  : (const V*)(op->form ? op->mu32.p : op->lam32.p);
    // Every region is written before it is read within one call (nodal slabs by
    // k_nodal, P by k_pinit, gM only where an earlier item of the same call
    // wrote it, item scratch, convert and cell slots by their own item), so
    // nothing needs clearing; every active entry of y is written by the final gather.
    k_nodal<V><<<p.nD, 256, 0, st>>>(op->dp, x, ml, nscratch);
    int32_t nb = (int32_t)p.b_items.size();
    if (nb > 0) k_pinit<V><<<nb, 256, 0, st>>>(op->dp, ml, pc, 0);
    for (int k = 0; k < p.d; ++k) {
        int32_t b = op->a_dim_chain_off[k], e = op->a_dim_chain_off[k + 1];
        if (e > b) k_prolong<V><<<e - b, op->tune.prolong_threads, 0, st>>>(op->dp, pc, b);
    }
    rc = phaseB_launch<D, V>(op, pc, zb, gm, scratch, conv, sp, y, acell, lam, st);
    if (rc) return rc;
    CUDA_TRY(cudaGetLastError());
    return 0;
}

template <typename V>
int matvec_noalloc_dispatch(lsg_operator* op, const V* x, V* y, cudaStream_t st, unsigned char* base) {
    switch (op->plan.d) {
    case 1: return matvec_noalloc_impl<1, V>(op, x, y, st, base);
    case 2: return matvec_noalloc_impl<2, V>(op, x, y, st, base);
    case 3: return matvec_noalloc_impl<3, V>(op, x, y, st, base);
    case 4: return matvec_noalloc_impl<4, V>(op, x, y, st, base);
    case 5: return matvec_noalloc_impl<5, V>(op, x, y, st, base);
    case 6: return matvec_noalloc_impl<6, V>(op, x, y, st, base);
    case 7: return matvec_noalloc_impl<7, V>(op, x, y, st, base);
    case 8: return matvec_noalloc_impl<8, V>(op, x, y, st, base);
    }
    return fail(LSG_E_INVALID, "unsupported dimension");
}

}  // namespace

extern "C" int lsg_matvec_device_noalloc(lsg_operator* op, const void* x, void* y, int32_t precision, void* stream) {
    if (!op || !x || !y) return fail(LSG_E_INVALID, "null argument");
    if (!op->have_coef) return fail(LSG_E_STATE, "no coefficient set");
    if (precision != LSG_FP64 && precision != LSG_FP32)
        return fail(LSG_E_INVALID, "precision must be LSG_FP64 or LSG_FP32");
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev != op->device) return fail(LSG_E_INVALID, "the operator lives on another device than the current one");
    unsigned char* base = nullptr;
    int rc = noalloc_address(&base);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (precision == LSG_FP64) return matvec_noalloc_dispatch<double>(op, (const double*)x, (double*)y, st, base);
    return matvec_noalloc_dispatch<float>(op, (const float*)x, (float*)y, st, base);
}

// ============================================================================= learned diagonal C-ABI
struct lsg_mlp;
extern "C" int lsg_mlp_forward(lsg_mlp* m, const float* X, int64_t rows, float* out, void* stream);

extern "C" int lsg_operator_features(lsg_operator* op, float* feat, void* stream) {
    if (!op || !feat) return fail(LSG_E_INVALID, "null argument");
    if (!op->have_coef) return fail(LSG_E_STATE, "no coefficient set");
    if (!op->nbmask.p) {  // same-depth neighbour flags, built on first use
        std::vector<uint16_t> m = lsg::same_depth_neighbor_mask(op->plan);
        if (op->nbmask.upload(m, &op->dev_bytes)) return LSG_E_CUDA;
    }
    k_features<<<nblk(op->plan.n, 128), 128, 0, (cudaStream_t)stream>>>(op->dp, op->family, op->params.as<double>(),
                                                                        op->nbmask.as<uint16_t>(), feat);
    CUDA_TRY(cudaGetLastError());
    return 0;
}

extern "C" int lsg_operator_base_diag(lsg_operator* op, double* base, void* stream) {
    if (!op || !base) return fail(LSG_E_INVALID, "null argument");
    if (!op->have_coef) return fail(LSG_E_STATE, "no coefficient set");
    k_base_diag<<<nblk(op->plan.n, 128), 128, 0, (cudaStream_t)stream>>>(op->dp, op->family, op->params.as<double>(), base);
    CUDA_TRY(cudaGetLastError());
    return 0;
}

extern "C" int lsg_operator_install_learned(lsg_operator* op, lsg_mlp* m, void* stream) {
    if (!op || !m) return fail(LSG_E_INVALID, "null argument");
    if (!op->have_coef) return fail(LSG_E_STATE, "no coefficient set");
    int64_t n = op->plan.n;
    int F = 7 * op->plan.d + 5;
    size_t* tot = &op->dev_bytes;
    int rc = 0;
    if (!op->feat.p) rc |= op->feat.alloc((size_t)n * F * sizeof(float), tot);
    if (!op->mlp_out.p) rc |= op->mlp_out.alloc((size_t)n * sizeof(float), tot);
    if (!op->base.p) rc |= op->base.alloc((size_t)n * sizeof(double), tot);
    if (!op->learned.p) rc |= op->learned.alloc((size_t)n * sizeof(double), tot);
    if (rc) return LSG_E_CUDA;
    rc = lsg_operator_features(op, op->feat.as<float>(), stream);
    if (!rc) rc = lsg_operator_base_diag(op, op->base.as<double>(), stream);
    if (!rc) rc = lsg_mlp_forward(m, op->feat.as<float>(), n, op->mlp_out.as<float>(), stream);
    if (rc) return rc;
    k_install_learned<<<nblk(n), 256, 0, (cudaStream_t)stream>>>(n, op->act.as<uint8_t>(), op->base.as<double>(),
                                                                 op->mlp_out.as<float>(), op->learned.as<double>());
    CUDA_TRY(cudaGetLastError());
    op->have_learned = true;
    return 0;
}
