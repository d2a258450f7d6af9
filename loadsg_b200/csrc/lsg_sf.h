// Factorised level-T cell operator of a dense slab (the k_sf kernel in
// lsg_device.cu and its host emulation in lsg_sf.cpp).
//
// The reference applies, per cell of depth T+1, the stored 2^d x 2^d local
// matrix a_c * K_ref (LocalStiffnessMatrices.cpp:555-582; the entries come from
// the StencilTemplate::integration plugin, Stencil.h:740).  With the
// coefficient constant on a cell, K_ref = sum_i K1_i (x) M1_(j != i) is
// diagonal in the tensor basis of the 1D modes "+" = u_L + u_R and
// "-" = u_L - u_R, so on a dense slab
//
//   z = E^T diag(a_c * Lambda) E u,   E = E_(d-1) (x) ... (x) E_0,
//
// where E_k maps the n_k = 2^T_k - 1 interior nodes of dimension k to the 2 n_k
// "reduced modes" of its n_k + 1 cells:
//   r = 0          BL: boundary cell 0, value u_1 (its only interior corner)
//   r = 2i - 1     P : interior cell i, u_i + u_(i+1)          (i = 1 .. n-1)
//   r = 2i         M : interior cell i, u_i - u_(i+1)
//   r = 2n - 1     BR: boundary cell n, value u_n
// A boundary cell has one interior corner, so its "+" and "-" modes carry the
// same value and are merged (B type).  Per dimension and mode type the 1D
// stiffness / mass factors (the 1/2 of the Hadamard normalisation included)
// are
//   P: kappa 0,   mu h/4      M: kappa 1/h, mu h/12      B: kappa 1/h, mu h/3
// and a mode's eigenvalue is Lambda = S (stiffness) or M (mass) of the pair
// (S, M) built dimension by dimension as (S, M) <- (S mu + M kappa, M mu)
// from (0, 1).  A dimension with one interior node (n = 1) has two B modes of
// the same node whose factors are equal: it collapses into its coefficient,
// a~ = a(cell 0) + a(cell 1), and enters (S, M) as a constant.
//
// Per (case, slab) item one CTA applies the operator:
//   * some non-collapsed dimensions may be "chunked": their reduced modes are
//     taken one tuple at a time (the slice of u for a tuple is a signed sum of
//     at most 2^nq strided blocks of u), which bounds the shared-memory work
//     space; the planner picks the fitting set of the lowest estimated cost;
//   * the remaining "mid" dimensions are swept through shared memory, one
//     dimension per stage, ping-ponging between two regions;
//   * the two innermost remaining dimensions (a, held in registers, and b,
//     streamed) are transformed, scaled and transformed back in one pass; when
//     a chunk has few planes, each plane's b cells are split into nseg
//     segments on as many threads, and the row shared by two segments is the
//     sum of their two partial rows, added in segment order after a barrier.
// Stage layouts keep the slab's dimension order without the chunked
// dimensions (a fastest); slice position e maps to u by inserting each chunked
// dimension (fast division by the slice extent below it).  No atomics: every
// output is written by one thread per stage, and the chunk loop adds into z in
// a fixed order.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "lsg_plan.h"

#ifdef __CUDACC__
#define LSG_SF_HD __host__ __device__
#else
#define LSG_SF_HD
#endif

namespace lsg {

// Unsigned division by a constant: q / d = (umulhi(q, m) + q) >> s for
// q < 2^31 (m = floor(2^32 (2^s - d) / d) + 1, s = ceil(log2 d)).
struct SfDiv {
    uint32_t d = 1, m = 1, s = 0;
};
SfDiv sf_div(uint32_t d);

struct SfDim {
    int32_t n = 1;        // interior nodes (1 for a virtual dimension)
    int32_t pstride = 0;  // slab-position stride
    int32_t cstride = 0;  // stride in the slab's collapsed-coefficient array (plan order)
    int32_t T = 0;        // depth (h = 2^-T); a virtual dimension has T = -1
    SfDiv div2n;          // division by 2n (decode of reduced-mode indices)
};

struct SfSlab {
    int32_t nm = 0, nq = 0;   // mid dimensions, chunked dimensions
    SfDim a, b;               // a: registers (n <= the precision's limit) or virtual; b: streamed
    SfDim mid[kMaxDim];       // inner to outer
    SfDim q[kMaxDim];         // chunked, inner to outer
    SfDiv qB[kMaxDim];        // per chunked dim: slice extent below it (slice -> u position)
    int32_t qmult[kMaxDim];   // per chunked dim: qB.d * (n - 1)
    int64_t coef_off = 0;     // offset of the slab's collapsed coefficients
    double S0 = 0.0, M0 = 1.0;  // (S, M) of the collapsed dimensions
    double unit_sum = 1.0;      // collapsed coefficient of a = 1 (2^#collapsed)
    int32_t slice = 0;        // nodes of one chunk slice = n_a n_b prod_mid n
    int32_t nchunk = 1;       // prod over chunked dimensions of 2n
    int32_t npl = 1;          // pencil planes of the fused step = prod_mid 2n
    int32_t stage[kMaxDim + 1] = {};  // stage sizes (elements): stage k has mid dims < k transformed
    SfDiv inner[kMaxDim];     // division by the inner size I_k of mid sweep k
    int32_t hi_off = 0;       // offset of the second ping-pong region (= stage[nm])
    int32_t wtotal = 0;       // work-space elements: stage[0] (nm = 0), else stage[nm] + stage[nm-1]
    int32_t na_max = 0;       // largest a extent this plan was made for
    int32_t nseg = 1;         // b segments per plane in the fused step (power of two; FP64 kernel)
};

// Dynamic shared memory of the k_sf CTA of one slab: the work space, then two
// buffers (this chunk's and the next one's) of the chunk's 2^nq signed blocks:
// int64 offsets of both buffers, then signs of the value size of both.
inline LSG_SF_HD size_t sf_comb_offset(const SfSlab& D, size_t value_bytes) {
    return ((size_t)(D.wtotal > 0 ? D.wtotal : 1) * value_bytes + 15) & ~(size_t)15;
}
inline LSG_SF_HD size_t sf_smem_bytes(const SfSlab& D, size_t value_bytes) {
    return sf_comb_offset(D, value_bytes) + 2 * ((size_t)1 << D.nq) * (8 + value_bytes);
}

// Collapsed-coefficient layout of every dense slab: for slab t, the cells of its
// non-collapsed dimensions (extents n_k + 1) from coef_off[t]; ccount = total.
// Sparse slabs get no entries.  The order of the dimensions inside a slab's
// block is its plan's (sf_plan): the mid dimensions fastest (inner to outer),
// then a, b and the chunked dimensions, so that the threads of a warp, which
// take consecutive mid modes in the fused step, read neighbouring coefficients.
// The FP32 and FP64 plans differ, and so do their coefficient arrays' orders.
struct SfCoefLayout {
    std::vector<int64_t> coef_off;  // per slab
    int64_t ccount = 0;
};
SfCoefLayout sf_coef_layout(const Plan& p);

// Plans every dense slab for a work space of at most wcap elements and an a
// extent of at most na_max (3 or 7); sparse slabs get nm = nq = -1.
std::vector<SfSlab> sf_plan(const Plan& p, const SfCoefLayout& L, int64_t wcap, int na_max);

// Host emulation (tests): collapsed coefficients of one slab from per-cell
// coefficients (slab cell order), and the factorised apply z = A_T u.
// Coefficient stride of every slab dimension k in plan D's order (0 for a
// collapsed dimension): by_dim[0 .. d-1].
void sf_cell_strides(const Plan& p, int t, const SfSlab& D, int32_t* by_dim);
void sf_collapse_host(const Plan& p, int t, const SfSlab& D, const double* acell_slab, double* coef);
void sf_apply_host(const SfSlab& D, int form, const double* coef, const double* u, double* z);
// Direct cell-by-cell apply of the same operator (corner pairs of every cell
// with both corners in the slab), the reference's LocalStiffnessMatrices form.
void cells_apply_host(const Plan& p, int t, int form, const double* acell_slab, const double* u, double* z);

}  // namespace lsg
