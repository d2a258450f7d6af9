// Host-side planner: flattens a LoAdSG grid (points in storage order + active
// flags) once into per-depth structure-of-arrays tables and a static launch
// schedule for the prewavelet matvec.  Everything here is integer work and is
// bit-exact against the reference's own lookups (tests/test_plan_tables.py).
//
// Reference anchors (paths relative to library/source/):
//   depth list              iterator/depthIterator.h:14-50
//   per-case depth order    iterator/depthIterator.cpp:7-45 (sortDepths)
//   case order              tests/old_versions/MatrixVectorMultiplicationPrewavelets.h:23-50
//   multilevel store (I,T)  sgrid/multilevelSparseGrid.cpp:9-34
//   cells of depth T+1      cells/CellStructure.h:23-61
//   prewavelet stencil      indices/index.cc:252-327 (nextFiveP)
//   prolongation            MatrixVectorMultiplication/MatrixVectorHomogen.h:444-474
//   restriction             MatrixVectorMultiplication/MatrixVectorHomogen.h:485-530
//   convert to prewavelets  MatrixVectorMultiplication/MatrixVectorHomogen.h:540-562
//   case function           MatrixVectorMultiplication/MatrixVectorHomogen.h:1618-1738
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace lsg {

constexpr int kMaxDim = 8;

// A "slab" is the level-T full grid restricted to the grid points of depth <= T
// (the reference's multilevel entries (I,T)).  Slab entries are ordered by
// their linear index in the level-T interior grid (dim 0 fastest), so a slab
// that is the complete level-T grid ("dense") needs no position lookups.
struct Slab {
    int32_t T[kMaxDim];
    int64_t off = 0;    // offset of the slab in the flat multilevel layout
    int64_t n = 0;      // N_T
    bool dense = false; // every interior point of the level-T grid is present
    int64_t cell_off = 0, ncell = 0;   // cells of depth T+1 inside the grid
    int64_t corner_off = -1;           // corner table (sparse slabs only)
};

// Gather tables of one sum-factorised tensor stencil stage: out[e] =
// sum_s w(code_s) * in[src_s], with NSRC sources per output.
struct StageSet {
    int nsrc = 0;
    std::vector<int64_t> stage_off;  // per (depth, stage) offset into src/code arrays; size nD*d+1
    std::vector<int32_t> src;        // nsrc per output, -1 = none
    std::vector<int32_t> code;       // 3 bits per source: 0 none, 1: 1.0, 2: 0.9, 3: -0.6, 4: 0.1
};

struct PhaseAItem {      // P_c(T+e_k) += prolong_k P_c(T)
    int32_t c, t_src, t_dst, dim;
    int64_t src_off, dst_off, n_dst;   // data offsets (case-local arrays already resolved)
    int64_t tab_off;                   // 2 int32 per destination entry
};

struct PhaseBStep {      // one restriction step inside a phase-B item
    int32_t t_dst;       // depth id of Tc (valid)
    int32_t dim;
    int64_t tab_off;     // 3 int32 per destination entry (self, left, right)
    int64_t n_src, n_dst;
    int64_t gm_off;      // gM_c(Tc) offset
    int32_t gm_prev;     // 1 if gM_c(Tc) was written by an earlier item
};

struct PhaseBItem {
    int32_t c, t;            // case, depth id of T
    int64_t p_off;           // P_c(T)
    int64_t gm_off;          // gM_c(T)
    int32_t gm_prev;         // 1 if gM_c(T) holds data from earlier items
    int32_t step_begin, step_end;
    int32_t t_conv;          // depth id of the final Tc (convert) or -1
    int64_t scratch_off;     // per-item scratch (two slab-sized buffers + convert stages)
};

struct Plan {
    int d = 0;
    int64_t n = 0;
    std::vector<int32_t> pts;   // n*d
    std::vector<uint8_t> act;   // n
    // depth list
    int nD = 0;
    std::vector<int32_t> D;      // nD*d
    std::vector<int32_t> did;    // per point
    std::vector<int32_t> maxdep; // d
    std::vector<int64_t> ex_off, ex;         // exact-depth points, storage order
    std::vector<int64_t> exa_off, exa;       // active exact-depth points, storage order
    // slabs
    std::vector<Slab> slabs;                 // nD
    int64_t M = 0;                           // total slab entries
    std::vector<int64_t> slab_pt;            // M: storage index
    std::vector<uint64_t> slab_key;          // M: linear index in level-T interior grid
    // cells
    int64_t C = 0;
    std::vector<uint64_t> cell_key;          // C: linear index of min corner in level-T cell grid
    std::vector<int32_t> cell_corner;        // sparse slabs: 2^d slab positions or -1
    // tensor stencil transforms
    StageSet nodal;    // per depth: x (storage) -> slab T (3 sources)
    StageSet convert;  // per depth: slab T -> active exact-depth points (5 sources)
    std::vector<int64_t> nodal_dom, convert_dom; // per (depth, stage j=0..d) domain sizes, nD*(d+1)
    // prolongation tables for (T, k) with T+e_k in D: index nD*d, -1 if absent
    std::vector<int64_t> prol_tab;           // per (t, k) offset into prol
    std::vector<int32_t> prol;               // 2 per destination entry
    // restriction tables keyed by (src depth, dst depth, dim)
    std::vector<int32_t> restr;              // 3 per destination entry
    // per-case schedule
    int ncase = 0;
    std::vector<std::vector<int32_t>> sorted;  // per case: depth ids in sortDepths order
    std::vector<int64_t> p_case_off, gm_case_off; // per case base offsets
    int64_t p_total = 0, gm_total = 0;
    std::vector<int64_t> p_slab_off;   // ncase*nD, -1 if slab not used
    std::vector<int64_t> gm_slab_off;  // ncase*nD, -1 if not used
    std::vector<PhaseAItem> a_items;
    std::vector<int32_t> a_level_off;  // levels of phase A
    std::vector<PhaseBItem> b_items;
    std::vector<PhaseBStep> b_steps;
    std::vector<int32_t> b_level_off;  // levels of phase B (descending restriction sum)
    int64_t scratch_total = 0;         // max over levels of per-level scratch
    int64_t nodal_scratch = 0;
    int64_t max_slab = 0;              // max N_T
    // instances of a concatenated plan (concat_plans); one instance otherwise
    std::vector<int64_t> inst_n_off;   // point offsets, size instances+1
    std::vector<int32_t> inst_t_off;   // depth-id offsets
    std::vector<int64_t> inst_c_off;   // cell offsets
    std::vector<int32_t> slab_inst;    // instance of every slab (depth id)
    // statistics
    double plan_seconds = 0.0;
    std::string error;
};

// Tables of the prewavelet basis transforms (BasisTransformations.cpp):
// calcNodalByPrew evaluates a prewavelet expansion at every grid point,
// calcPrewByNodal inverts it.  Built on first use of a transform.
struct PoleGroup {        // one (depth, component, dimension) of calcPrewByNodal
    int32_t t, dim, size;  // depth id, dimension, pole length
    int32_t pad;
    int64_t npoles;
    int64_t pos_off;       // npoles * size entries: 4 * storage index + 2 * active + (depth == T), or -1
    int64_t lu_off;        // 5 * size doubles: L[k+1][k], L[k+2][k], R[k][k], R[k][k+1], R[k][k+2]
};

struct BasisPlan {
    std::vector<int32_t> order;       // depth ids coarse to fine (ListOfDepthOrderedSubgrids)
    // prewavelet -> level-T nodal values over every point of depth T (hanging included)
    StageSet nodal;
    std::vector<int64_t> nodal_dom;   // nD*(d+1)
    std::vector<int64_t> ex_sorted;   // per depth, its points sorted by level-T key (offsets: Plan::ex_off)
    // hierarchization inside slab T: per slab entry and dim, the slab entries at
    // the entry's own level left/right in that dim (global slab positions, -1 none)
    std::vector<int32_t> slab_nb;     // M*d*2
    std::vector<uint8_t> slab_dep;    // M*d: depth of the entry's point per dim
    // full-grid (de)hierarchization: per point and dim, storage indices of the
    // left/right neighbours at the point's own level (-1: boundary or absent)
    std::vector<int32_t> pt_nb;       // n*d*2
    int maxdep = 0;
    std::vector<int64_t> lvl_off;     // (dim * (maxdep+1) + depth) -> range in lvl_pts (active points)
    std::vector<int32_t> lvl_pts;
    // calcPrewByNodal: pole groups in processing order, grouped per depth
    std::vector<PoleGroup> groups;
    std::vector<int32_t> step_t;      // depth id of each step (reverse subgrid order)
    std::vector<int32_t> step_group;  // groups of step s: [step_group[s], step_group[s+1])
    std::vector<int32_t> pole_pos;
    std::vector<double> lu;
    int64_t max_pole_elems = 0;       // largest npoles*size of a group
    double seconds = 0.0;
};

bool build_basis_plan(const Plan& p, BasisPlan& b, std::string& error);

// Per point, bit 2j / 2j+1: the point of the same depth two level-T steps to the
// left / right in dim j exists (a feature of the learned diagonal: where it is
// missing, part of the prewavelet's support has no cells).
std::vector<uint16_t> same_depth_neighbor_mask(const Plan& p);

// Builds the plan; returns false and sets plan.error on invalid input.
bool build_plan(int d, int64_t n, const int32_t* points, const uint8_t* active, Plan& plan);

// Concatenates plans of the same dimension into one plan whose launches cover
// every part: all offsets are shifted, and the level schedules of phases A and
// B are merged by level index.  The parts are independent grids, so only each
// part's own level order has to be kept; a merged level runs the level-L items
// of all parts side by side.  The per-item arithmetic is unchanged, so a
// part's result equals the result of its own plan bit for bit.
bool concat_plans(const std::vector<const Plan*>& parts, Plan& out);

// Helpers shared with the tests / C-ABI.
int depth1(int32_t i);
// sortDepths order of one case (bit k of c = restriction in dim k).
std::vector<int32_t> sorted_depths(const Plan& p, int c);

}  // namespace lsg
