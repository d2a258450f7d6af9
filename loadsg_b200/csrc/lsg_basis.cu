// Prewavelet basis transforms on the device (BasisTransformations.cpp, paths
// relative to LoAdSG's library/source/):
//
//   calcNodalByPrew (:670-706)  u = values at every grid point of the
//       prewavelet expansion prew: for every depth T the level-T nodal values
//       of the depth-T prewavelets (5^d stencil of every point of depth T,
//       CalcHierbyPrew :321-353) are hierarchized inside the level-T slab and
//       summed as hierarchical surpluses; one dehierarchization of the sum
//       (CalcNodalBasis :174-198) gives u.  All slabs are independent, so each
//       step is one launch over all of them.
//   calcPrewByNodal (:486-545)  the inverse: the depths are visited from the
//       finest backwards; per depth the banded pole systems of its connected
//       components are solved on the current nodal values (SolvePrewavelet
//       :468-484, GetPrewaveletCoefficients :100-172), the surplus of the new
//       coefficients is subtracted and the nodal values are recomputed.
//
// The integer structure (components, boxes, poles, LU factors of the pole
// matrices) comes from lsg::build_basis_plan on the host; the kernels here do
// the value work: one thread per pole for the banded solves, grid-stride
// sweeps for the stencil stages and the (de)hierarchization levels.
#include "lsg_internal.h"
#include "../../include/lsg.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <string>
#include <vector>

namespace {

using lsg_internal::fail_msg;

#define BS_TRY(expr)                                                                                    \
    do {                                                                                                \
        cudaError_t _e = (expr);                                                                        \
        if (_e != cudaSuccess)                                                                          \
            return fail_msg(LSG_E_CUDA, (std::string(#expr) + ": " + cudaGetErrorString(_e)).c_str());  \
    } while (0)

struct DevArr {
    void* p = nullptr;
    size_t bytes = 0;
    ~DevArr() { if (p) cudaFree(p); }
    int alloc(size_t b) {
        bytes = b;
        if (!b) return 0;
        return cudaMalloc(&p, b) == cudaSuccess ? 0 : fail_msg(LSG_E_CUDA, "cudaMalloc (basis tables)");
    }
    template <typename T>
    int upload(const std::vector<T>& v) {
        int rc = alloc(v.size() * sizeof(T));
        if (rc || v.empty()) return rc;
        return cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess
                   ? 0 : fail_msg(LSG_E_CUDA, "cudaMemcpy (basis tables)");
    }
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

struct BasisState {
    lsg::BasisPlan bp;
    int d = 0, nD = 0;
    int64_t n = 0, M = 0;
    std::vector<int64_t> slab_off, slab_n, scr_off, ex_off_h;  // host copies
    std::vector<int32_t> T;                          // nD*d
    DevArr ex_sorted, stage_src, stage_code, slab_pt, slab_nb, slab_dep, pt_nb, lvl_pts, pole_pos, lu;
    DevArr ml, scratch, hier, uw, pscr, act;
};

inline unsigned nblk(int64_t n, int t = 256) {
    int64_t b = (n + t - 1) / t;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 16));
}

__device__ __forceinline__ double wcode(int c) {
    // 5-point prewavelet stencil weights (indices/index.cc:180-250)
    switch (c) {
    case 1: return 1.0;
    case 2: return 0.9;
    case 3: return -0.6;
    case 4: return 0.1;
    default: return 0.0;
    }
}

// one sum-factorised stencil stage: out[e] = sum_s w_s in[src_s]; stage 0 reads
// prew through the depth's point list
__global__ void k_stage(int64_t nout, const int32_t* __restrict__ src, const int32_t* __restrict__ code,
                        const double* __restrict__ in, const int64_t* __restrict__ in_map, double* __restrict__ out) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nout; e += (int64_t)gridDim.x * blockDim.x) {
        int cd = code[e];
        double acc = 0.0;
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            int32_t i = src[e * 3 + s];
            if (i < 0) break;
            double v = in_map ? in[in_map[i]] : in[i];
            acc += wcode((cd >> (3 * s)) & 7) * v;
        }
        out[e] = acc;
    }
}

// v[e] = v[e] - 0.5 (v[left] + v[right]) for slab entries whose point has depth t in dim k
// (CalcHierarchicalBasis, BasisTransformations.cpp:13-38)
__global__ void k_slab_hier(int64_t lo, int64_t hi, int d, int k, int t, const uint8_t* __restrict__ dep,
                            const int32_t* __restrict__ nb, double* __restrict__ v) {
    for (int64_t e = lo + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < hi; e += (int64_t)gridDim.x * blockDim.x) {
        if (dep[e * d + k] != t) continue;
        int32_t l = nb[(e * d + k) * 2], r = nb[(e * d + k) * 2 + 1];
        v[e] = v[e] - 0.5 * ((l >= 0 ? v[l] : 0.0) + (r >= 0 ? v[r] : 0.0));
    }
}

// hier[point of slab entry] += sign * v[entry]
__global__ void k_slab_acc(int64_t lo, int64_t hi, const int32_t* __restrict__ slab_pt, const double* __restrict__ v,
                           double sign, double* __restrict__ hier) {
    for (int64_t e = lo + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < hi; e += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&hier[slab_pt[e]], sign * v[e]);
}

// one (de)hierarchization level of the whole grid: u[p] += sign 0.5 (u[left] + u[right])
// for the points of depth t in dim k (CalcNodalBasis :174-198 with sign +1,
// CalcHierarchicalBasis :390-409 with sign -1)
__global__ void k_pt_level(const int32_t* __restrict__ pts, int64_t np, int d, int k, const int32_t* __restrict__ nb,
                           double sign, double* __restrict__ u) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t p = pts[i];
        int32_t l = nb[((int64_t)p * d + k) * 2], r = nb[((int64_t)p * d + k) * 2 + 1];
        double s = 0.5 * ((l >= 0 ? u[l] : 0.0) + (r >= 0 ? u[r] : 0.0));
        u[p] = sign > 0 ? u[p] + s : u[p] - s;
    }
}

// banded pole solves of one (depth, component, dimension): one thread per pole
// (GetPrewaveletCoefficients with PrewaveletMatrixHomogen::solve,
// sgoperation/matrix.cpp:152-168 and matrix_operations.cc:64-86)
__global__ void k_pole(int64_t npoles, int size, const int32_t* __restrict__ pos, const double* __restrict__ lu,
                       double* __restrict__ scr, double* __restrict__ u, double* __restrict__ prew) {
    int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= npoles) return;
    const int32_t* ps = pos + q * size;
    double* y = scr + q * size;
    for (int i = 0; i < size; ++i) y[i] = ps[i] >= 0 ? u[ps[i] >> 2] : 0.0;
    if (size < 2) {
        y[0] = y[0] / lu[2];
    } else {
        for (int k = 0; k < size - 1; ++k) {
            y[k + 1] = y[k + 1] - lu[5 * k] * y[k];
            if (k + 2 < size) y[k + 2] = y[k + 2] - lu[5 * k + 1] * y[k];
        }
        for (int k = size - 1; k >= 0; --k) {
            double c = y[k];
            if (k + 1 < size) c = c - lu[5 * k + 3] * y[k + 1];
            if (k + 2 < size) c = c - lu[5 * k + 4] * y[k + 2];
            y[k] = c / lu[5 * k + 2];
        }
    }
    for (int i = 0; i < size; ++i) {  // assignments touch active points only
        int32_t p = ps[i];
        if (p < 0 || !(p & 2)) continue;
        u[p >> 2] = y[i];
        if (p & 1) prew[p >> 2] = y[i];
    }
}

// dst[i] = src[i] at active points; elsewhere 0 (zero_else) or unchanged
__global__ void k_masked_copy(int64_t n, const uint8_t* __restrict__ act, const double* __restrict__ src,
                              double* __restrict__ dst, int zero_else) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (act[i]) dst[i] = src[i];
        else if (zero_else) dst[i] = 0.0;
    }
}

int ensure_basis(lsg_operator* op, BasisState** out) {
    auto& slot = lsg_internal::basis_slot(op);
    if (slot) { *out = static_cast<BasisState*>(slot.get()); return 0; }
    const lsg::Plan& p = lsg_internal::plan(op);
    if (p.inst_n_off.size() != 2) return fail_msg(LSG_E_INVALID, "basis transforms take a single-grid operator");
    auto st = std::make_shared<BasisState>();
    std::string err;
    if (!lsg::build_basis_plan(p, st->bp, err)) return fail_msg(LSG_E_INVALID, err.c_str());
    BasisState& S = *st;
    const lsg::BasisPlan& b = S.bp;
    S.d = p.d;
    S.nD = p.nD;
    S.n = p.n;
    S.M = p.M;
    S.T.assign(p.D.begin(), p.D.end());
    S.ex_off_h.assign(p.ex_off.begin(), p.ex_off.end());
    S.slab_off.resize(p.nD);
    S.slab_n.resize(p.nD);
    S.scr_off.resize(p.nD);
    int64_t scr = 0, scr_max = 0;
    for (int t = 0; t < p.nD; ++t) {
        S.slab_off[t] = p.slabs[t].off;
        S.slab_n[t] = p.slabs[t].n;
        S.scr_off[t] = scr;
        int64_t need = 0;
        for (int j = 1; j < p.d; ++j) need += b.nodal_dom[t * (p.d + 1) + j];
        scr += need;
        scr_max = std::max(scr_max, need);
    }
    std::vector<int32_t> spt(p.slab_pt.begin(), p.slab_pt.end());
    int rc = 0;
    rc |= S.ex_sorted.upload(b.ex_sorted);
    rc |= S.stage_src.upload(b.nodal.src);
    rc |= S.stage_code.upload(b.nodal.code);
    rc |= S.slab_pt.upload(spt);
    rc |= S.slab_nb.upload(b.slab_nb);
    rc |= S.slab_dep.upload(b.slab_dep);
    rc |= S.pt_nb.upload(b.pt_nb);
    rc |= S.lvl_pts.upload(b.lvl_pts);
    rc |= S.pole_pos.upload(b.pole_pos);
    rc |= S.lu.upload(b.lu);
    rc |= S.act.upload(p.act);
    rc |= S.ml.alloc(std::max<int64_t>(p.M, 1) * 8);
    rc |= S.scratch.alloc(std::max<int64_t>(scr, 1) * 8);
    rc |= S.hier.alloc(p.n * 8);
    rc |= S.uw.alloc(p.n * 8);
    rc |= S.pscr.alloc(std::max<int64_t>(b.max_pole_elems, 1) * 8);
    if (rc) return LSG_E_CUDA;
    slot = st;
    *out = st.get();
    return 0;
}

// level-T nodal values of the depth-t prewavelets of prew into ml (slab t)
void nodal_depth(BasisState& S, int t, const double* prew, cudaStream_t st) {
    const lsg::BasisPlan& b = S.bp;
    const int d = S.d;
    double* scr = S.scratch.as<double>() + S.scr_off[t];
    int64_t off_in = 0, off_out = 0;
    for (int j = 0; j < d; ++j) {
        int64_t so = b.nodal.stage_off[t * d + j];
        int64_t nout = b.nodal_dom[t * (d + 1) + j + 1];
        double* outp = (j == d - 1) ? S.ml.as<double>() + S.slab_off[t] : scr + off_out;
        if (nout > 0) {
            if (j == 0)
                k_stage<<<nblk(nout), 256, 0, st>>>(nout, S.stage_src.as<int32_t>() + so * 3, S.stage_code.as<int32_t>() + so,
                                                    prew, S.ex_sorted.as<int64_t>() + S.ex_off_h[t], outp);
            else
                k_stage<<<nblk(nout), 256, 0, st>>>(nout, S.stage_src.as<int32_t>() + so * 3, S.stage_code.as<int32_t>() + so,
                                                    scr + off_in, nullptr, outp);
        }
        off_in = off_out;
        if (j < d - 1) off_out += nout;
    }
}

// hierarchize slab entries [lo, hi) in every dim; levels from the finest down
void slab_hierarchize(BasisState& S, int64_t lo, int64_t hi, const int32_t* maxT, cudaStream_t st) {
    for (int k = 0; k < S.d; ++k)
        for (int t = maxT[k]; t >= 1; --t)
            k_slab_hier<<<nblk(hi - lo), 256, 0, st>>>(lo, hi, S.d, k, t, S.slab_dep.as<uint8_t>(), S.slab_nb.as<int32_t>(),
                                                       S.ml.as<double>());
}

void grid_sweep(BasisState& S, double* u, bool hierarchize, cudaStream_t st) {
    const lsg::BasisPlan& b = S.bp;
    const int L = b.maxdep + 1;
    for (int k = 0; k < S.d; ++k)
        for (int i = 1; i <= b.maxdep; ++i) {
            int t = hierarchize ? b.maxdep + 1 - i : i;
            int64_t lo = b.lvl_off[k * L + t], hi = b.lvl_off[k * L + t + 1];
            if (hi > lo)
                k_pt_level<<<nblk(hi - lo), 256, 0, st>>>(S.lvl_pts.as<int32_t>() + lo, hi - lo, S.d, k,
                                                          S.pt_nb.as<int32_t>(), hierarchize ? -1.0 : 1.0, u);
        }
}

int nodal_by_prew(lsg_operator* op, const double* prew, double* u, cudaStream_t st) {
    BasisState* Sp = nullptr;
    int rc = ensure_basis(op, &Sp);
    if (rc) return rc;
    BasisState& S = *Sp;
    std::vector<int32_t> maxT(S.d, 0);
    for (int t = 0; t < S.nD; ++t) {
        nodal_depth(S, t, prew, st);
        for (int k = 0; k < S.d; ++k) maxT[k] = std::max(maxT[k], S.T[t * S.d + k]);
    }
    slab_hierarchize(S, 0, S.M, maxT.data(), st);
    BS_TRY(cudaMemsetAsync(u, 0, S.n * 8, st));
    if (S.M > 0) k_slab_acc<<<nblk(S.M), 256, 0, st>>>(0, S.M, S.slab_pt.as<int32_t>(), S.ml.as<double>(), 1.0, u);
    // u = hier at active points (0 at hanging points), then dehierarchize
    k_masked_copy<<<nblk(S.n), 256, 0, st>>>(S.n, S.act.as<uint8_t>(), u, u, 1);
    grid_sweep(S, u, false, st);
    BS_TRY(cudaGetLastError());
    return 0;
}

int prew_by_nodal(lsg_operator* op, double* prew, const double* u, cudaStream_t st) {
    BasisState* Sp = nullptr;
    int rc = ensure_basis(op, &Sp);
    if (rc) return rc;
    BasisState& S = *Sp;
    const lsg::BasisPlan& b = S.bp;
    double* uw = S.uw.as<double>();
    double* hier = S.hier.as<double>();
    BS_TRY(cudaMemsetAsync(prew, 0, S.n * 8, st));
    BS_TRY(cudaMemcpyAsync(uw, u, S.n * 8, cudaMemcpyDeviceToDevice, st));
    k_masked_copy<<<nblk(S.n), 256, 0, st>>>(S.n, S.act.as<uint8_t>(), u, hier, 1);
    grid_sweep(S, hier, true, st);
    const size_t nsteps = b.step_t.size();
    for (size_t s = 0; s < nsteps; ++s) {
        const int t = b.step_t[s];
        for (int32_t gi = b.step_group[s]; gi < b.step_group[s + 1]; ++gi) {
            const lsg::PoleGroup& g = b.groups[gi];
            k_pole<<<(unsigned)((g.npoles + 127) / 128), 128, 0, st>>>(g.npoles, g.size, S.pole_pos.as<int32_t>() + g.pos_off,
                                                                       S.lu.as<double>() + g.lu_off, S.pscr.as<double>(), uw,
                                                                       prew);
        }
        if (s + 1 == nsteps) break;  // the remaining updates only feed later depths
        nodal_depth(S, t, prew, st);
        const int64_t lo = S.slab_off[t], hi = lo + S.slab_n[t];
        slab_hierarchize(S, lo, hi, &S.T[t * S.d], st);
        k_slab_acc<<<nblk(hi - lo), 256, 0, st>>>(lo, hi, S.slab_pt.as<int32_t>(), S.ml.as<double>(), -1.0, hier);
        k_masked_copy<<<nblk(S.n), 256, 0, st>>>(S.n, S.act.as<uint8_t>(), hier, uw, 0);
        grid_sweep(S, uw, false, st);
    }
    BS_TRY(cudaGetLastError());
    return 0;
}

// partial sums of a[i] b[i] over active points, one per CTA (summed on the host in order)
__global__ void k_dot_active(int64_t n, const uint8_t* __restrict__ act, const double* __restrict__ a,
                             const double* __restrict__ b, double* __restrict__ part) {
    __shared__ double red[32];
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (act[i]) acc += a[i] * b[i];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (threadIdx.x == 0) part[blockIdx.x] = acc;
    }
}

// H1::getValue / L2::getValue (applications/H1_Norm.cpp): v = calcPrewByNodal(u),
// sqrt(sum over active points of v (A v)) with A the coefficient-1 stiffness
// (Poisson) or mass (HelmHoltz) operator
int norm_value(lsg_operator* op, const double* u_host, int form, double* value) {
    if (!op || !u_host || !value) return fail_msg(LSG_E_INVALID, "null argument");
    BasisState* Sp = nullptr;
    int rc = ensure_basis(op, &Sp);
    if (rc) return rc;
    const int64_t n = Sp->n;
    constexpr int kParts = 592;
    double *u = nullptr, *v = nullptr, *Av = nullptr, *part = nullptr;
    BS_TRY(cudaMalloc(&u, n * 8 * 3 + kParts * 8));
    v = u + n;
    Av = v + n;
    part = Av + n;
    std::vector<double> hp(kParts);
    if (cudaMemcpy(u, u_host, n * 8, cudaMemcpyHostToDevice) != cudaSuccess) rc = fail_msg(LSG_E_CUDA, "cudaMemcpy");
    if (!rc) rc = prew_by_nodal(op, v, u, 0);
    if (!rc && cudaMemset(Av, 0, n * 8) != cudaSuccess) rc = fail_msg(LSG_E_CUDA, "cudaMemset");
    if (!rc) rc = lsg_internal::matvec64_unit(op, form, v, Av, 0);
    if (!rc) {
        k_dot_active<<<kParts, 256>>>(n, Sp->act.as<uint8_t>(), v, Av, part);
        if (cudaMemcpy(hp.data(), part, kParts * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = fail_msg(LSG_E_CUDA, "cudaMemcpy");
    }
    cudaFree(u);
    if (rc) return rc;
    double sum = 0.0;
    for (double x : hp) sum += x;
    *value = std::sqrt(sum);
    return 0;
}

int host_call(lsg_operator* op, const double* in, double* out, bool to_nodal) {
    if (!op || !in || !out) return fail_msg(LSG_E_INVALID, "null argument");
    const int64_t n = lsg_internal::plan(op).n;
    double *din = nullptr, *dout = nullptr;
    BS_TRY(cudaMalloc(&din, n * 8));
    if (cudaMalloc(&dout, n * 8) != cudaSuccess) { cudaFree(din); return fail_msg(LSG_E_CUDA, "cudaMalloc"); }
    int rc = cudaMemcpy(din, in, n * 8, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : fail_msg(LSG_E_CUDA, "cudaMemcpy");
    if (!rc) rc = to_nodal ? nodal_by_prew(op, din, dout, 0) : prew_by_nodal(op, dout, din, 0);
    if (!rc && cudaMemcpy(out, dout, n * 8, cudaMemcpyDeviceToHost) != cudaSuccess) rc = fail_msg(LSG_E_CUDA, "cudaMemcpy");
    cudaFree(din);
    cudaFree(dout);
    return rc;
}

}  // namespace

namespace lsg_internal {
int prew_by_nodal_dev(lsg_operator* op, double* prew, const double* u, cudaStream_t st) {
    return prew_by_nodal(op, prew, u, st);
}
}  // namespace lsg_internal

extern "C" {

int lsg_calc_nodal_by_prew_device(lsg_operator* op, const double* prew, double* u, void* stream) {
    if (!op || !prew || !u) return fail_msg(LSG_E_INVALID, "null argument");
    return nodal_by_prew(op, prew, u, (cudaStream_t)stream);
}

int lsg_calc_prew_by_nodal_device(lsg_operator* op, double* prew, const double* u, void* stream) {
    if (!op || !prew || !u) return fail_msg(LSG_E_INVALID, "null argument");
    return prew_by_nodal(op, prew, u, (cudaStream_t)stream);
}

int lsg_calc_nodal_by_prew(lsg_operator* op, const double* prew, double* u) { return host_call(op, prew, u, true); }

int lsg_calc_prew_by_nodal(lsg_operator* op, double* prew, const double* u) { return host_call(op, u, prew, false); }

int lsg_h1_norm(lsg_operator* op, const double* u, double* value) { return norm_value(op, u, 0, value); }

int lsg_l2_norm(lsg_operator* op, const double* u, double* value) { return norm_value(op, u, 1, value); }

}  // extern "C"
