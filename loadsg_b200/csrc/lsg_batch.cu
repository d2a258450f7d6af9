// Batched operators and CG solves: many grids of uneven size (any mix of
// dimensions), each with its own coefficient and right-hand side.
//
// Grids of one dimension are concatenated into one plan (lsg::concat_plans),
// so one matvec of the group is the same short sequence of launches as for a
// single grid, each launch covering the level's items of every grid.  The
// batch vectors are the groups' vectors side by side; per-grid quantities
// (dot products, CG scalars, convergence) are reduced over fixed chunks of
// at most kChunk entries that never straddle two grids, so every reduction
// is deterministic and a grid's CG arithmetic is the single-grid CG's
// (CG::solveHomogen, applications/cg_method.h:759-886) with per-grid scalars.
// One batched CG iteration is captured as a CUDA graph and replayed; the host
// reads only the number of grids still iterating.  Grids that converge stop
// changing (step sizes forced to zero) while the others continue.
#include "lsg_internal.h"
#include "../../include/lsg.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace {

using lsg_internal::fail_msg;

#define BT_TRY(expr)                                                                          \
    do {                                                                                      \
        cudaError_t _e = (expr);                                                              \
        if (_e != cudaSuccess)                                                                \
            return fail_msg(LSG_E_CUDA, (std::string(#expr) + ": " + cudaGetErrorString(_e)).c_str()); \
    } while (0)

constexpr int64_t kChunk = 8192;  // entries per reduction chunk (one CTA)
constexpr int kThreads = 256;

struct Chunk {
    int64_t lo, hi;
    int32_t inst, pad;
};

struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
    ~Buf() { if (p) cudaFree(p); }
    int alloc(size_t b) {
        if (p) { cudaFree(p); p = nullptr; }
        bytes = b;
        if (!b) return 0;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) return fail_msg(LSG_E_CUDA, (std::string("cudaMalloc: ") + cudaGetErrorString(e)).c_str());
        return 0;
    }
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

// ----------------------------------------------------------------------------- kernels
__device__ __forceinline__ double bsum(double v, double* red) {
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

// Per-grid scalars, structure of arrays of `count` entries each.
struct Scal {
    double *delta, *dg, *tau, *dnew, *beta, *rr, *stop, *scale, *best;
    int32_t *conv, *its, *bad, *best_it;
    int32_t* pending;
};

// part[c] = sum over chunk c of a*b (and of a2*b2 when a2 is given)
template <typename A, typename B>
__global__ void kb_dot(const Chunk* __restrict__ ch, const A* __restrict__ a, const B* __restrict__ b,
                       double* __restrict__ part) {
    __shared__ double red[32];
    const Chunk c = ch[blockIdx.x];
    double acc = 0.0;
    for (int64_t i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) acc += (double)a[i] * (double)b[i];
    acc = bsum(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// out[i] = sum of part over grid i's chunks [cb[i], ce[i])  (one CTA per grid)
__global__ void kb_final(const int32_t* __restrict__ cb, const int32_t* __restrict__ ce, const double* __restrict__ part,
                         int stride, double* __restrict__ out) {
    __shared__ double red[32];
    int i = blockIdx.x;
    double acc = 0.0;
    for (int k = cb[i] + threadIdx.x; k < ce[i]; k += blockDim.x) acc += part[(int64_t)k * stride];
    acc = bsum(acc, red);
    if (threadIdx.x == 0) out[i] = acc;
}

// beta = delta_new / delta, delta = delta_new (k_beta of the single-grid CG)
__global__ void kb_beta(int count, Scal s) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    if (s.conv[i]) { s.beta[i] = 0.0; return; }
    s.beta[i] = s.delta[i] != 0.0 ? s.dnew[i] / s.delta[i] : 0.0;
    s.delta[i] = s.dnew[i];
}

// tau = delta / (d^T A d)
__global__ void kb_tau(int count, Scal s) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    s.tau[i] = (s.conv[i] || s.dg[i] == 0.0) ? 0.0 : s.delta[i] / s.dg[i];
}

template <typename V>
__global__ void kb_update_d(const Chunk* __restrict__ ch, const double* __restrict__ beta, const V* __restrict__ h,
                            V* __restrict__ d) {
    const Chunk c = ch[blockIdx.x];
    V b = (V)beta[c.inst];
    for (int64_t i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) d[i] = V(-1.0) * h[i] + b * d[i];
}

// r += tau g; x -= tau d; h = r / z (active) or r; partial sums of r.h and r.r
template <typename V>
__global__ void kb_update_rxh(const Chunk* __restrict__ ch, const double* __restrict__ tau, V* __restrict__ r,
                              V* __restrict__ x, const V* __restrict__ g, const V* __restrict__ d, V* __restrict__ h,
                              const V* __restrict__ z, const uint8_t* __restrict__ act, double* __restrict__ part) {
    __shared__ double red[32];
    const Chunk c = ch[blockIdx.x];
    V t = (V)tau[c.inst];
    double a1 = 0.0, a2 = 0.0;
    for (int64_t i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
        V ri = r[i] + t * g[i];
        r[i] = ri;
        x[i] = x[i] - t * d[i];
        V hi = (act[i] && z) ? ri / z[i] : ri;
        h[i] = hi;
        a1 += (double)ri * (double)hi;
        a2 += (double)ri * (double)ri;
    }
    a1 = bsum(a1, red);
    a2 = bsum(a2, red);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = a1;
        part[2 * blockIdx.x + 1] = a2;
    }
}

// per grid: delta_new, rr from the chunk partials; convergence test; iteration count
// stall > 0 (inner FP32 solves of the refinement): a grid whose residual has
// not dropped below 0.9 x its best for `stall` iterations stops iterating
__global__ void kb_check(const int32_t* __restrict__ cb, const int32_t* __restrict__ ce, const double* __restrict__ part,
                         Scal s, int crit, double eps, int count_its, int stall) {
    __shared__ double red[32];
    int i = blockIdx.x;
    double a1 = 0.0, a2 = 0.0;
    for (int k = cb[i] + threadIdx.x; k < ce[i]; k += blockDim.x) {
        a1 += part[2 * (int64_t)k];
        a2 += part[2 * (int64_t)k + 1];
    }
    a1 = bsum(a1, red);
    a2 = bsum(a2, red);
    if (threadIdx.x != 0) return;
    bool was = s.conv[i] != 0;
    if (was) return;
    s.dnew[i] = a1;
    s.rr[i] = a2;
    if (count_its) s.its[i] += 1;
    bool done;
    if (!isfinite(a1) || !isfinite(a2)) { s.bad[i] = 1; done = true; }
    else if (crit == 0) done = a1 < eps * eps || a1 <= eps;  // cg_method.h:852,871
    else done = a2 <= s.stop[i];
    if (!count_its) { s.best[i] = a2; s.best_it[i] = s.its[i]; }
    else if (stall > 0 && !done) {
        if (a2 < 0.81 * s.best[i]) { s.best[i] = a2; s.best_it[i] = s.its[i]; }
        else if (s.its[i] - s.best_it[i] >= stall) done = true;
    }
    if (done) s.conv[i] = 1;
    else atomicAdd(s.pending, 1);
}

template <typename V>
__global__ void kb_precond_start(int64_t n, const uint8_t* __restrict__ act, const V* __restrict__ r,
                                 const V* __restrict__ z, V* __restrict__ h) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n && act[i]) h[i] = z ? r[i] / z[i] : r[i];
}

template <typename V>
__global__ void kb_sub(int64_t n, const V* __restrict__ f, V* __restrict__ r) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) r[i] = f[i] - r[i];
}

// delta = delta_new after the start test (grids already converged keep theirs)
__global__ void kb_set_delta(int count, Scal s) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count && !s.conv[i]) s.delta[i] = s.dnew[i];
}

// interleaved chunk partials of r.h and r.r (the layout kb_check reads)
template <typename V>
__global__ void kb_dot2(const Chunk* __restrict__ ch, const V* __restrict__ r, const V* __restrict__ h,
                        double* __restrict__ part) {
    __shared__ double red[32];
    const Chunk c = ch[blockIdx.x];
    double a1 = 0.0, a2 = 0.0;
    for (int64_t i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
        a1 += (double)r[i] * (double)h[i];
        a2 += (double)r[i] * (double)r[i];
    }
    a1 = bsum(a1, red);
    a2 = bsum(a2, red);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = a1;
        part[2 * blockIdx.x + 1] = a2;
    }
}

// stop thresholds: eps^2 * ff for the relative-residual criterion
__global__ void kb_stop(int count, Scal s, const double* __restrict__ ff, double eps2) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) s.stop[i] = eps2 * ff[i];
}

// IR: outer convergence on the FP64 residual, per-grid scale 1/||r|| (0 when done)
// the inner stop for grids still refining: when this step can reach the
// target (the missing factor within 10x of itol) aim at 0.5 x that factor,
// or 0.1 x after a step that did not halve the residual, otherwise reduce by
// itol (the single-grid refinement's rule); rr_prev[i] keeps the last residual
__global__ void kb_outer(int count, Scal s, const double* __restrict__ rr64, const double* __restrict__ ff, double eps2,
                         double itol, int32_t* __restrict__ outer_conv, int32_t* __restrict__ outer_its,
                         double* __restrict__ rr_prev) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    double rr = rr64[i];
    bool done = outer_conv[i] || rr <= eps2 * ff[i] || !isfinite(rr);
    if (!isfinite(rr)) s.bad[i] = 1;
    if (done) { outer_conv[i] = 1; s.scale[i] = 0.0; }
    else {
        s.scale[i] = 1.0 / sqrt(rr);
        outer_its[i] += 1;
        const double margin = rr_prev[i] > 0.0 && rr > 0.25 * rr_prev[i] ? 0.1 : 0.5;
        rr_prev[i] = rr;
        double t = margin * sqrt(eps2 * ff[i] / rr);
        t = t >= 0.1 * itol ? fmin(0.5, fmax(t, 0.1 * itol)) : itol;
        s.stop[i] = t * t;
    }
    s.conv[i] = done ? 1 : 0;  // inner CG runs only on grids still refining
    if (!done) atomicAdd(s.pending, 1);
}

__global__ void kb_scale_f32(const Chunk* __restrict__ ch, const double* __restrict__ scale, const double* __restrict__ r,
                             float* __restrict__ r32) {
    const Chunk c = ch[blockIdx.x];
    double sc = scale[c.inst];
    for (int64_t i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) r32[i] = (float)(r[i] * sc);
}

__global__ void kb_axpy_f32(const Chunk* __restrict__ ch, const double* __restrict__ scale, const float* __restrict__ e,
                            double* __restrict__ x) {
    const Chunk c = ch[blockIdx.x];
    double sc = scale[c.inst];
    if (sc == 0.0) return;
    double a = 1.0 / sc;
    for (int64_t i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) x[i] += a * (double)e[i];
}

__global__ void kb_to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

inline unsigned nb(int64_t n, int t = kThreads) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// ============================================================================= batch object
struct lsg_batch {
    int count = 0;
    int64_t n = 0;
    std::vector<int64_t> off, len;  // per grid (input order)
    struct Group {
        lsg_operator* op = nullptr;
        int64_t off = 0, n = 0;
        std::vector<int> members;  // grid indices, part order
    };
    std::vector<Group> groups;
    std::vector<int> grid_group, grid_part;
    int nchunks = 0;
    Buf chunks, cb, ce, act;
    ~lsg_batch() {
        for (Group& g : groups)
            if (g.op) lsg_operator_destroy(g.op);
    }
};

namespace {

template <typename V>
int batch_matvec(lsg_batch* b, const V* x, V* y, cudaStream_t st) {
    for (auto& g : b->groups) {
        int rc = std::is_same<V, double>::value
                     ? lsg_internal::matvec64(g.op, (const double*)(x + g.off), (double*)(y + g.off), st)
                     : lsg_internal::matvec32(g.op, (const float*)(x + g.off), (float*)(y + g.off), st);
        if (rc) return rc;
    }
    return 0;
}

int64_t batch_matvec_launches(const lsg_batch* b, bool f32) {
    int64_t l = 0;
    for (auto& g : b->groups) l += lsg_internal::matvec_launch_count(g.op, f32);
    return l;
}

struct BSolver {
    lsg_batch* B;
    int count;
    int64_t n;
    int stall = 0;  // stall window of the current loop (0: off)
    Buf r, g, d, h, z, part, sc, flags, ff, rr64;
    Buf r32, g32, d32, h32, e32, z32;
    Buf outer_conv, outer_its, rr_prev;
    int32_t* pend_h = nullptr;
    Scal S{};
    ~BSolver() { if (pend_h) cudaFreeHost(pend_h); }
    int init(bool fp32, cudaStream_t st) {
        int rc = 0;
        rc |= r.alloc(n * 8);
        rc |= g.alloc(n * 8);
        rc |= d.alloc(n * 8);
        rc |= h.alloc(n * 8);
        rc |= part.alloc((size_t)B->nchunks * 2 * 8);
        rc |= sc.alloc((size_t)count * 9 * 8);
        rc |= flags.alloc(((size_t)count * 4 + 1) * 4);
        rc |= ff.alloc((size_t)count * 8);
        rc |= rr64.alloc((size_t)count * 8);
        rc |= outer_conv.alloc((size_t)count * 4);
        rc |= outer_its.alloc((size_t)count * 4);
        rc |= rr_prev.alloc((size_t)count * 8);
        if (fp32) {
            rc |= r32.alloc(n * 4);
            rc |= g32.alloc(n * 4);
            rc |= d32.alloc(n * 4);
            rc |= h32.alloc(n * 4);
            rc |= e32.alloc(n * 4);
        }
        if (rc) return LSG_E_CUDA;
        if (cudaMallocHost(&pend_h, sizeof(int32_t)) != cudaSuccess) return fail_msg(LSG_E_CUDA, "cudaMallocHost");
        double* s = sc.as<double>();
        S.delta = s;
        S.dg = s + count;
        S.tau = s + 2 * count;
        S.dnew = s + 3 * count;
        S.beta = s + 4 * count;
        S.rr = s + 5 * count;
        S.stop = s + 6 * count;
        S.scale = s + 7 * count;
        S.best = s + 8 * count;
        int32_t* f = flags.as<int32_t>();
        S.conv = f;
        S.its = f + count;
        S.bad = f + 2 * count;
        S.best_it = f + 3 * count;
        S.pending = f + 4 * count;
        for (Buf* bf :
             {&r, &g, &d, &h, &sc, &flags, &outer_conv, &outer_its, &rr_prev, &r32, &g32, &d32, &h32, &e32})
            if (bf->p) BT_TRY(cudaMemsetAsync(bf->p, 0, bf->bytes, st));  // on the solver's stream
        return 0;
    }
    const Chunk* ch() const { return B->chunks.as<Chunk>(); }
    const int32_t* cb() const { return B->cb.as<int32_t>(); }
    const int32_t* ce() const { return B->ce.as<int32_t>(); }
    const uint8_t* act() const { return B->act.as<uint8_t>(); }

    // per-grid sums of a.b into out[count]
    template <typename A, typename Bt>
    void dot(const A* a, const Bt* b, double* out, cudaStream_t st) {
        kb_dot<A, Bt><<<B->nchunks, kThreads, 0, st>>>(ch(), a, b, part.as<double>());
        kb_final<<<count, kThreads, 0, st>>>(cb(), ce(), part.as<double>(), 1, out);
    }

    // CG start: r holds rhs - A x; h = precond(r) on active entries (0 elsewhere),
    // d = 0, delta = delta_new = r.h, rr = r.r, then the loop-entry test
    // (cg_method.h:820-851 and the while condition)
    template <typename V>
    int start(V* rv, V* dv, V* hv, const V* zv, int crit, double eps, cudaStream_t st) {
        BT_TRY(cudaMemsetAsync(hv, 0, n * sizeof(V), st));
        kb_precond_start<V><<<nb(n), kThreads, 0, st>>>(n, act(), rv, zv, hv);
        BT_TRY(cudaMemsetAsync(dv, 0, n * sizeof(V), st));
        kb_dot2<V><<<B->nchunks, kThreads, 0, st>>>(ch(), rv, hv, part.as<double>());
        BT_TRY(cudaMemsetAsync(S.pending, 0, 4, st));
        kb_check<<<count, kThreads, 0, st>>>(cb(), ce(), part.as<double>(), S, crit, eps, 0, 0);
        kb_set_delta<<<nb(count), kThreads, 0, st>>>(count, S);
        BT_TRY(cudaGetLastError());
        return 0;
    }

    template <typename V>
    int body(V* x, V* rv, V* gv, V* dv, V* hv, const V* zv, int crit, double eps, cudaStream_t st) {
        kb_beta<<<nb(count), kThreads, 0, st>>>(count, S);
        kb_update_d<V><<<B->nchunks, kThreads, 0, st>>>(ch(), S.beta, hv, dv);
        int rc = batch_matvec<V>(B, dv, gv, st);
        if (rc) return rc;
        dot<V, V>(dv, gv, S.dg, st);
        kb_tau<<<nb(count), kThreads, 0, st>>>(count, S);
        kb_update_rxh<V><<<B->nchunks, kThreads, 0, st>>>(ch(), S.tau, rv, x, gv, dv, hv, zv, act(), part.as<double>());
        BT_TRY(cudaMemsetAsync(S.pending, 0, 4, st));
        kb_check<<<count, kThreads, 0, st>>>(cb(), ce(), part.as<double>(), S, crit, eps, 1, stall);
        BT_TRY(cudaMemcpyAsync(pend_h, S.pending, 4, cudaMemcpyDeviceToHost, st));
        BT_TRY(cudaGetLastError());
        return 0;
    }

    // loop until every grid has converged or maxit iterations; returns iterations run
    template <typename V>
    int loop(V* x, V* rv, V* gv, V* dv, V* hv, const V* zv, int crit, double eps, int maxit, bool use_graph,
             cudaStream_t st, int* ran, int64_t* launches) {
        cudaGraphExec_t exec = nullptr;
        if (use_graph) {
            cudaGraph_t graph;
            BT_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            int rc = body<V>(x, rv, gv, dv, hv, zv, crit, eps, st);
            cudaError_t e = cudaStreamEndCapture(st, &graph);
            if (rc) return rc;
            if (e != cudaSuccess) return fail_msg(LSG_E_CUDA, cudaGetErrorString(e));
            e = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) return fail_msg(LSG_E_CUDA, cudaGetErrorString(e));
        }
        int rc = 0, it = 0;
        BT_TRY(cudaMemcpyAsync(pend_h, S.pending, 4, cudaMemcpyDeviceToHost, st));
        BT_TRY(cudaStreamSynchronize(st));
        for (int i = 1; i <= maxit && *pend_h > 0; ++i) {
            if (exec) {
                cudaError_t e = cudaGraphLaunch(exec, st);
                if (e != cudaSuccess) { rc = fail_msg(LSG_E_CUDA, cudaGetErrorString(e)); break; }
            } else {
                rc = body<V>(x, rv, gv, dv, hv, zv, crit, eps, st);
                if (rc) break;
            }
            cudaError_t e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) { rc = fail_msg(LSG_E_CUDA, cudaGetErrorString(e)); break; }
            it = i;
        }
        if (exec) cudaGraphExecDestroy(exec);
        *ran = it;
        *launches += (int64_t)it * (batch_matvec_launches(B, std::is_same<V, float>::value) + 8);
        return rc;
    }
};


int batch_solve(lsg_batch* b, const double* f, double* x, const lsg_solver_opts* o, lsg_solve_report* reps,
                lsg_solve_report* total, cudaStream_t user_st) {
    if (!b || !f || !x || !o) return fail_msg(LSG_E_INVALID, "null argument");
    if (o->precond != 0 && o->precond != 1)
        return fail_msg(LSG_E_INVALID, "batched solves take precond 0 (Jacobi) or 1 (none)");
    if (o->precision != LSG_FP64 && o->precision != LSG_FP32) return fail_msg(LSG_E_INVALID, "bad precision");
    const bool fp32 = o->precision == LSG_FP32;
    for (auto& g : b->groups) {
        if (!lsg_internal::has_coefficient(g.op)) return fail_msg(LSG_E_STATE, "a grid of the batch has no coefficient");
        int rc = lsg_internal::prepare_precision(g.op, fp32);
        if (rc) return rc;
    }
    const int count = b->count;
    const int64_t n = b->n;
    cudaStream_t st;
    BT_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        cudaEvent_t e0, e1, eu;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            cudaEventDestroy(eu);
            cudaStreamDestroy(s);
        }
    } guard{st, nullptr, nullptr, nullptr};
    cudaEventCreate(&guard.e0);
    cudaEventCreate(&guard.e1);
    cudaEventCreate(&guard.eu);
    cudaEventRecord(guard.eu, user_st);
    cudaStreamWaitEvent(st, guard.eu, 0);
    BSolver S;
    S.B = b;
    S.count = count;
    S.n = n;
    int rc = S.init(fp32, st);
    if (rc) return rc;
    // diagonal of every grid, side by side in batch order
    const double* z = nullptr;
    if (o->precond == 0) {
        rc = S.z.alloc(n * 8);
        if (rc) return rc;
        for (auto& g : b->groups) {
            const double* dg = nullptr;
            rc = lsg_internal::jacobi_diag(g.op, st, &dg);
            if (rc) return rc;
            BT_TRY(cudaMemcpyAsync(S.z.as<double>() + g.off, dg, g.n * 8, cudaMemcpyDeviceToDevice, st));
        }
        z = S.z.as<double>();
    }
    const int maxit = o->max_iter > 0 ? o->max_iter : 500;
    const double eps = o->eps;
    const int crit = o->criterion;
    const bool graph = o->use_graph != 0;
    int64_t launches = 0;
    int rounds = 0, outer_rounds = 0;
    double* r = S.r.as<double>();
    cudaEventRecord(guard.e0, st);
    S.dot<double, double>(f, f, S.ff.as<double>(), st);
    kb_stop<<<nb(count), kThreads, 0, st>>>(count, S.S, S.ff.as<double>(), eps * eps);
    if (!fp32) {
        BT_TRY(cudaMemsetAsync(r, 0, n * 8, st));
        rc = batch_matvec<double>(b, x, r, st);
        if (rc) return rc;
        kb_sub<double><<<nb(n), kThreads, 0, st>>>(n, f, r);
        rc = S.start<double>(r, S.d.as<double>(), S.h.as<double>(), z, crit, eps, st);
        if (!rc)
            rc = S.loop<double>(x, r, S.g.as<double>(), S.d.as<double>(), S.h.as<double>(), z, crit, eps, maxit, graph, st,
                                &rounds, &launches);
        launches += batch_matvec_launches(b, false) + 12;
        outer_rounds = 1;
    } else {
        const int inner = o->inner_iter > 0 ? o->inner_iter : 1000;
        const double itol = o->inner_tol > 0 ? o->inner_tol : 1e-5;
        float* z32 = nullptr;
        if (z) {
            rc = S.z32.alloc(n * 4);
            if (rc) return rc;
            kb_to_f32<<<nb(n), kThreads, 0, st>>>(n, z, S.z32.as<float>());
            z32 = S.z32.as<float>();
        }
        // bounded like the single-grid refinement: at most 4 max_iter inner iterations
        for (int outer = 0; outer < maxit && rounds < 4 * maxit; ++outer) {
            BT_TRY(cudaMemsetAsync(r, 0, n * 8, st));
            rc = batch_matvec<double>(b, x, r, st);
            if (rc) break;
            kb_sub<double><<<nb(n), kThreads, 0, st>>>(n, f, r);
            S.dot<double, double>(r, r, S.rr64.as<double>(), st);
            BT_TRY(cudaMemsetAsync(S.S.pending, 0, 4, st));
            kb_outer<<<nb(count), kThreads, 0, st>>>(count, S.S, S.rr64.as<double>(), S.ff.as<double>(), eps * eps,
                                                     itol, S.outer_conv.as<int32_t>(), S.outer_its.as<int32_t>(),
                                                     S.rr_prev.as<double>());
            BT_TRY(cudaMemcpyAsync(S.pend_h, S.S.pending, 4, cudaMemcpyDeviceToHost, st));
            BT_TRY(cudaStreamSynchronize(st));
            launches += batch_matvec_launches(b, false) + 6;
            if (*S.pend_h == 0) break;
            ++outer_rounds;
            kb_scale_f32<<<b->nchunks, kThreads, 0, st>>>(S.ch(), S.S.scale, r, S.r32.as<float>());
            BT_TRY(cudaMemsetAsync(S.e32.p, 0, n * 4, st));
            rc = S.start<float>(S.r32.as<float>(), S.d32.as<float>(), S.h32.as<float>(), z32, 1, itol, st);
            if (rc) break;
            int ran = 0;
            S.stall = 400;  // long: PCG residual 2-norms are not monotone
            rc = S.loop<float>(S.e32.as<float>(), S.r32.as<float>(), S.g32.as<float>(), S.d32.as<float>(),
                               S.h32.as<float>(), z32, 1, itol, inner, graph, st, &ran, &launches);
            S.stall = 0;
            if (rc) break;
            rounds += ran;
            kb_axpy_f32<<<b->nchunks, kThreads, 0, st>>>(S.ch(), S.S.scale, S.e32.as<float>(), x);
            launches += 12;
        }
    }
    cudaEventRecord(guard.e1, st);
    if (rc) return rc;
    // true relative residuals in FP64
    BT_TRY(cudaMemsetAsync(r, 0, n * 8, st));
    rc = batch_matvec<double>(b, x, r, st);
    if (rc) return rc;
    kb_sub<double><<<nb(n), kThreads, 0, st>>>(n, f, r);
    S.dot<double, double>(r, r, S.rr64.as<double>(), st);
    std::vector<double> rr(count), ff(count);
    std::vector<int32_t> its(count), bad(count), oits(count);
    BT_TRY(cudaMemcpyAsync(rr.data(), S.rr64.p, count * 8, cudaMemcpyDeviceToHost, st));
    BT_TRY(cudaMemcpyAsync(ff.data(), S.ff.p, count * 8, cudaMemcpyDeviceToHost, st));
    BT_TRY(cudaMemcpyAsync(its.data(), S.S.its, count * 4, cudaMemcpyDeviceToHost, st));
    BT_TRY(cudaMemcpyAsync(bad.data(), S.S.bad, count * 4, cudaMemcpyDeviceToHost, st));
    BT_TRY(cudaMemcpyAsync(oits.data(), S.outer_its.p, count * 4, cudaMemcpyDeviceToHost, st));
    BT_TRY(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, guard.e0, guard.e1);
    lsg_solve_report T;
    memset(&T, 0, sizeof T);
    T.converged = 1;
    T.iterations = rounds;
    T.outer_iterations = outer_rounds;
    T.seconds = ms * 1e-3;
    T.kernel_launches = launches;
    for (int i = 0; i < count; ++i) {
        lsg_solve_report R;
        memset(&R, 0, sizeof R);
        R.iterations = its[i];
        R.outer_iterations = fp32 ? oits[i] : 1;
        R.rel_residual = ff[i] > 0 ? std::sqrt(rr[i] / ff[i]) : std::sqrt(rr[i]);
        R.seconds = T.seconds;
        R.kernel_launches = launches;
        R.converged = !bad[i] && (crit != 1 || R.rel_residual <= eps * 1.0000001);
        if (reps) reps[i] = R;
        T.converged &= R.converged;
        T.rel_residual = std::max(T.rel_residual, R.rel_residual);
    }
    if (total) *total = T;
    cudaEventRecord(guard.eu, st);
    cudaStreamWaitEvent(user_st, guard.eu, 0);
    for (int i = 0; i < count; ++i)
        if (bad[i]) return fail_msg(LSG_E_NOCONV, "non-finite residual in a grid of the batch");
    return 0;
}

}  // namespace

extern "C" {

int lsg_batch_create(int32_t count, const int32_t* dims, const int32_t* const* points, const uint8_t* const* active,
                     const int64_t* n, lsg_batch** out) {
    if (!out || count < 1 || !dims || !points || !active || !n) return fail_msg(LSG_E_INVALID, "null or empty batch");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail_msg(LSG_E_CUDA, "no CUDA device");
    std::unique_ptr<lsg_batch> b(new lsg_batch());
    b->count = count;
    std::vector<lsg::Plan> plans(count);
    for (int i = 0; i < count; ++i)
        if (!points[i] || !active[i]) return fail_msg(LSG_E_INVALID, "null grid in batch");
    // the grids' plans are independent host work: one grid per thread
    std::vector<uint8_t> ok(count, 0);
#pragma omp parallel for schedule(dynamic, 1) if (count > 1)
    for (int i = 0; i < count; ++i) ok[i] = lsg::build_plan(dims[i], n[i], points[i], active[i], plans[i]) ? 1 : 0;
    for (int i = 0; i < count; ++i)
        if (!ok[i]) return fail_msg(LSG_E_INVALID, ("grid " + std::to_string(i) + ": " + plans[i].error).c_str());
    b->grid_group.assign(count, -1);
    b->grid_part.assign(count, -1);
    b->off.assign(count, 0);
    b->len.assign(count, 0);
    for (int d = 1; d <= lsg::kMaxDim; ++d) {
        std::vector<const lsg::Plan*> parts;
        lsg_batch::Group g;
        for (int i = 0; i < count; ++i)
            if (dims[i] == d) {
                b->grid_group[i] = (int)b->groups.size();
                b->grid_part[i] = (int)parts.size();
                parts.push_back(&plans[i]);
                g.members.push_back(i);
            }
        if (parts.empty()) continue;
        lsg::Plan merged;
        if (!lsg::concat_plans(parts, merged)) return fail_msg(LSG_E_INVALID, merged.error.c_str());
        g.off = b->n;
        g.n = merged.n;
        for (size_t k = 0; k < g.members.size(); ++k) {
            int i = g.members[k];
            b->off[i] = g.off + merged.inst_n_off[k];
            b->len[i] = merged.inst_n_off[k + 1] - merged.inst_n_off[k];
        }
        b->n += merged.n;
        int rc = lsg_internal::create_from_plan(std::move(merged), &g.op);
        if (rc) return rc;
        b->groups.push_back(std::move(g));
    }
    for (auto& pl : plans) pl = lsg::Plan();
    // reduction chunks in batch order, grid by grid
    std::vector<Chunk> ch;
    std::vector<int32_t> cbv(count), cev(count);
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int c) { return b->off[a] < b->off[c]; });
    for (int i : order) {
        cbv[i] = (int32_t)ch.size();
        for (int64_t lo = b->off[i]; lo < b->off[i] + b->len[i]; lo += kChunk)
            ch.push_back(Chunk{lo, std::min(lo + kChunk, b->off[i] + b->len[i]), i, 0});
        cev[i] = (int32_t)ch.size();
    }
    b->nchunks = (int)ch.size();
    std::vector<uint8_t> actv((size_t)b->n);
    for (auto& g : b->groups) {
        const lsg::Plan& p = lsg_internal::plan(g.op);
        std::copy(p.act.begin(), p.act.end(), actv.begin() + g.off);
    }
    int rc = 0;
    rc |= b->chunks.alloc(ch.size() * sizeof(Chunk));
    rc |= b->cb.alloc(count * 4);
    rc |= b->ce.alloc(count * 4);
    rc |= b->act.alloc(actv.size());
    if (rc) return LSG_E_CUDA;
    BT_TRY(cudaMemcpy(b->chunks.p, ch.data(), ch.size() * sizeof(Chunk), cudaMemcpyHostToDevice));
    BT_TRY(cudaMemcpy(b->cb.p, cbv.data(), count * 4, cudaMemcpyHostToDevice));
    BT_TRY(cudaMemcpy(b->ce.p, cev.data(), count * 4, cudaMemcpyHostToDevice));
    BT_TRY(cudaMemcpy(b->act.p, actv.data(), actv.size(), cudaMemcpyHostToDevice));
    *out = b.release();
    return 0;
}

void lsg_batch_destroy(lsg_batch* b) { delete b; }

int64_t lsg_batch_size(const lsg_batch* b) { return b ? b->n : 0; }

int lsg_batch_offsets(const lsg_batch* b, int64_t* offsets) {
    if (!b || !offsets) return fail_msg(LSG_E_INVALID, "null argument");
    for (int i = 0; i < b->count; ++i) offsets[i] = b->off[i];
    offsets[b->count] = b->n;
    return 0;
}

int lsg_batch_set_coefficient(lsg_batch* b, int32_t grid, int32_t family, const double* params, int32_t nparams) {
    if (!b) return fail_msg(LSG_E_INVALID, "null batch");
    if (grid < 0 || grid >= b->count) return fail_msg(LSG_E_INVALID, "grid index out of range");
    return lsg_internal::set_part_coefficient(b->groups[b->grid_group[grid]].op, b->grid_part[grid], family, params,
                                              nparams);
}

int lsg_batch_matvec_device(lsg_batch* b, const void* x, void* y, int32_t precision, void* stream) {
    if (!b || !x || !y) return fail_msg(LSG_E_INVALID, "null argument");
    for (auto& g : b->groups)
        if (!lsg_internal::has_coefficient(g.op)) return fail_msg(LSG_E_STATE, "a grid of the batch has no coefficient");
    cudaStream_t st = (cudaStream_t)stream;
    if (precision == LSG_FP64) return batch_matvec<double>(b, (const double*)x, (double*)y, st);
    if (precision == LSG_FP32) return batch_matvec<float>(b, (const float*)x, (float*)y, st);
    return fail_msg(LSG_E_INVALID, "precision must be LSG_FP64 or LSG_FP32");
}

int lsg_batch_autotune(lsg_batch* b, int32_t precision, int32_t reps) {
    if (!b) return fail_msg(LSG_E_INVALID, "null batch");
    for (auto& g : b->groups) {
        int rc = lsg_internal::autotune(g.op, precision, reps);
        if (rc) return rc;
    }
    return 0;
}

int lsg_batch_cg_solve_device(lsg_batch* b, const double* f, double* x, const lsg_solver_opts* opts,
                              lsg_solve_report* reports, lsg_solve_report* total, void* stream) {
    return batch_solve(b, f, x, opts, reports, total, (cudaStream_t)stream);
}

int lsg_batch_cg_solve(lsg_batch* b, const double* f, double* x, const lsg_solver_opts* opts, lsg_solve_report* reports,
                       lsg_solve_report* total) {
    if (!b || !f || !x) return fail_msg(LSG_E_INVALID, "null argument");
    double *fd = nullptr, *xd = nullptr;
    size_t bytes = (size_t)b->n * 8;
    BT_TRY(cudaMalloc(&fd, bytes));
    if (cudaMalloc(&xd, bytes) != cudaSuccess) {
        cudaFree(fd);
        return fail_msg(LSG_E_CUDA, "cudaMalloc");
    }
    int rc = 0;
    if (cudaMemcpy(fd, f, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(xd, x, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = fail_msg(LSG_E_CUDA, "cudaMemcpy");
    if (!rc) rc = batch_solve(b, fd, xd, opts, reports, total, 0);
    if ((!rc || rc == LSG_E_NOCONV) && cudaMemcpy(x, xd, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = fail_msg(LSG_E_CUDA, "cudaMemcpy");
    cudaFree(fd);
    cudaFree(xd);
    return rc;
}

}  // extern "C"
