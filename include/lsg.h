/*
 * lsg.h -- C-ABI of the B200 prewavelet matvec / CG library (liblsg.so).
 *
 * Plain pointers and sizes only.  Every function returns 0 on success and a
 * negative LSG_E* code on failure; lsg_last_error() gives the message of the
 * calling thread's last failure.  Nothing here calls exit() (the reference
 * does, e.g. LocalStiffnessMatrices.cpp:267-268).
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to LoAdSG's library/source/).
 *
 * An operator (or batch) keeps work buffers, its coefficient and its form in
 * its own state, so calls on one operator must come from one host thread at
 * a time (like the reference's MatrixVectorHomogen); different operators are
 * independent.
 */
#ifndef LSG_H
#define LSG_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LSG_OK 0
#define LSG_E_INVALID -1   /* bad argument or grid */
#define LSG_E_CUDA -2      /* CUDA runtime failure (device missing, out of memory, ...) */
#define LSG_E_STATE -3     /* call order (e.g. no coefficient set) */
#define LSG_E_NOCONV -4    /* solver did not reach the tolerance */

#define LSG_FP64 0
#define LSG_FP32 1

/* Coefficient families of -div(a grad u); a is sampled at each cell midpoint.
 * Parameter layouts (p = params):
 *   LSG_COEF_CONST     a = p[0]
 *   LSG_COEF_SINPROD   a = p[0] + p[1] prod_i sin(pi p[2+i] x_i)
 *   LSG_COEF_EXPSIN    a = exp(sum_{k=1..d} p[k-1] sin(k pi x_{k-1}))
 *   LSG_COEF_LOGNORMAL a = exp(sum_{j<J} p[1+j] prod_i sin(pi p[1+J+j*d+i] x_i)), J = p[0]
 *   LSG_COEF_SIN2PI    a = p[0] + p[1] sin(2 pi x_0) cos(2 pi x_1)              */
#define LSG_COEF_CONST 0
#define LSG_COEF_SINPROD 1
#define LSG_COEF_EXPSIN 2
#define LSG_COEF_LOGNORMAL 3
#define LSG_COEF_SIN2PI 4

/* Bilinear form of the local matrices (lsg_operator_set_form): the plugin's
 * a(x_c) times the exact Q1 stiffness (StencilTemplate::integration of a
 * diffusion plugin, stencils/Stencil.h:740) or times the exact Q1 mass
 * (HelmHoltz::integration, stencils/Stencil.h:900-919, for a = 1). */
#define LSG_FORM_STIFFNESS 0
#define LSG_FORM_MASS 1

typedef struct lsg_operator lsg_operator;

typedef struct {
    int32_t d;
    int64_t n_points;     /* N (active + hanging) */
    int64_t n_active;
    int32_t n_depths;     /* |D| */
    int64_t n_slab_entries;  /* sum_T N_T (multilevel entries) */
    int64_t n_cells;      /* sum_T C_T */
    int64_t case_slab_entries;   /* sum_c sum_{T in S(c)} N_T */
    int64_t case_cells;          /* sum_c sum_{T in S(c)} C_T */
    int64_t device_bytes; /* device memory held by the operator */
    double plan_seconds;
    double matvec_bytes_fp64;    /* algorithmic bytes of one FP64 matvec */
    double matvec_flops;         /* algorithmic flops of one matvec (cell apply) */
} lsg_info;

/* Flattens the grid (AdaptiveSparseGrid in storage order: getIndexOfTable(k),
 * sgrid/sparseGrid.h:566-572, and getActiveTable()) and uploads the tables.
 * Replaces MatrixVectorHomogen(grid, mgrid, symmetry, mpi_on)
 * (MatrixVectorMultiplication/MatrixVectorHomogen.h:72-77) together with
 * MultiLevelAdaptiveSparseGrid and CellData construction.
 * points: n*d 1D indices; active: n flags.  Uses the current CUDA device. */
int lsg_operator_create(int32_t d, const int32_t *points, const uint8_t *active, int64_t n, lsg_operator **out);
void lsg_operator_destroy(lsg_operator *op);
int lsg_operator_info(const lsg_operator *op, lsg_info *info);

/* Sets the coefficient (replaces constructing the StencilTemplate plugin,
 * stencils/Stencil.h:740, and LocalStiffnessMatricesMemoryDistribution,
 * localStiffnessMatrices/LocalStiffnessMatricesMemoryDistribution.h:14-159). */
int lsg_operator_set_coefficient(lsg_operator *op, int32_t family, const double *params, int32_t nparams);

/* y = A_prew x with host buffers of n doubles in storage order; y is written
 * at active points only (hanging entries untouched), as
 * MatrixVectorHomogen::multiplication (MatrixVectorHomogen.h:91-92,659-759). */
int lsg_matvec(lsg_operator *op, const double *x, double *y);

/* Same on device buffers of n elements (double for LSG_FP64, float for
 * LSG_FP32), enqueued on `stream` (a cudaStream_t, 0 = legacy default). */
int lsg_matvec_device(lsg_operator *op, const void *x, void *y, int32_t precision, void *stream);

/* Allocation-free variant of lsg_matvec_device (no counterpart in the
 * reference, which has no device code).  For callers that cannot allocate
 * device memory at call time: hosts whose own allocator owns the whole
 * device, loops that cannot afford the synchronisation of cudaMalloc/cudaFree.
 * Its work space is one fixed 32 MiB
 * array compiled into the library (held on every GPU that loads it until the
 * process exits); grids needing more are rejected with LSG_E_INVALID and a
 * message giving both sizes.  It calls no cudaMalloc/cudaFree.  The first call
 * on a device resolves the array's device address (cudaGetSymbolAddress), so
 * make that first call before any stream capture.  All calls share the array:
 * calls that overlap on the GPU (different streams, or threads without
 * ordering) race and give wrong results.  The operator itself (tables,
 * coefficient) is created beforehand as usual. */
int lsg_matvec_device_noalloc(lsg_operator *op, const void *x, void *y, int32_t precision, void *stream);

/* Times `iters` matvecs on device buffers with CUDA events between the
 * phases; phase_ms[0..4] = mean ms of (nodal transform, P init, prolongation
 * levels, cell operator, restriction wavefronts with the final gather),
 * phase_ms[5] = whole matvec (6 entries).  bytes[0..5] = algorithmic bytes of
 * the same phases for this precision (every vector, slab and table counted
 * once per kernel that must touch it); flops = floating-point operations of
 * the cell operator per matvec, as its kernels issue them. */
int lsg_matvec_profile(lsg_operator *op, const void *x, void *y, int32_t precision, int32_t iters, double *phase_ms,
                       double *bytes, double *flops);

/* Exact Jacobi diagonal a(psi_i, psi_i) at active points (0 at hanging), as
 * Preconditioning::precondLocalStiffnessMatrix (applications/cg_method.h:544-680). */
int lsg_diag(lsg_operator *op, double *diag);
int lsg_diag_device(lsg_operator *op, double *diag, void *stream);

typedef struct {
    double eps;          /* tolerance (meaning set by `criterion`) */
    int32_t criterion;   /* 0: reference rule on delta = r^T D^-1 r (cg_method.h:852,871);
                            1: true relative residual ||f - A x|| / ||f|| <= eps */
    int32_t max_iter;    /* 0 = 500 (cg_method.h:35) */
    int32_t precond;     /* 0 Jacobi (reference), 1 none, 2 learned diagonal (see lsg_set_learned_diag) */
    int32_t precision;   /* LSG_FP64: plain CG; LSG_FP32: FP32 inner CG in FP64 iterative refinement */
    int32_t inner_iter;  /* FP32+IR: inner iterations per refinement step (0 = 1000) */
    double inner_tol;    /* FP32+IR: inner relative reduction (0 = 1e-5) */
    int32_t use_graph;   /* capture one CG iteration as a CUDA graph */
} lsg_solver_opts;

typedef struct {
    int32_t iterations;      /* CG iterations (inner iterations summed for IR) */
    int32_t outer_iterations;
    double rel_residual;     /* ||f - A x|| / ||f|| recomputed in FP64 */
    double seconds;          /* device time of the solve */
    int32_t converged;
    int32_t fell_back;       /* learned preconditioner stalled -> Jacobi */
    int64_t kernel_launches; /* kernels of this library launched by the solve */
} lsg_solve_report;

/* Solves A x = f (CG::solveHomogen, applications/cg_method.h:27-33,759-886).
 * Host buffers of n doubles; x holds the initial guess on entry. */
int lsg_cg_solve(lsg_operator *op, const double *f, double *x, const lsg_solver_opts *opts, lsg_solve_report *rep);
/* Device-buffer variant (double arrays of n). */
int lsg_cg_solve_device(lsg_operator *op, const double *f, double *x, const lsg_solver_opts *opts,
                        lsg_solve_report *rep, void *stream);

/* Installs a diagonal preconditioner (n doubles, host) used by precond = 2. */
int lsg_set_learned_diag(lsg_operator *op, const double *diag);

/* ---- learned diagonal preconditioner (precond = 2).  A small MLP maps
 * per-point features to a positive scaling s = softplus(o) of a cheap
 * constant-coefficient diagonal b (exact for constant a on a complete grid):
 * D = b * s.  No counterpart in the reference (its CG always uses the exact
 * Jacobi diagonal, applications/cg_method.h:805); solves that stall with D
 * fall back to the exact diagonal (lsg_solve_report.fell_back).
 * Features (F = 7d + 5 floats per point, storage order): t_j / 8, x_j,
 * next-to-boundary flags, log a(x), sum_j t_j / (8d),
 * log a(x +- h_j e_j) - log a(x) with h_j = 2^-t_j, per dim two flags (the
 * same-depth point two level steps left / right exists), and mean, min and
 * max of log a - log a(x) over the midpoints of the 2^d surrounding cells. */
typedef struct lsg_mlp lsg_mlp;
/* params: lsg_mlp_num_params(F) floats, layout W1[64][F] b1[64] W2[64][64] b2
 * W3[64][64] b3 W4[64] b4; BF16-rounded weights, FP32 accumulation. */
int64_t lsg_mlp_num_params(int32_t n_features);
int lsg_mlp_create(int32_t n_features, const float *params, lsg_mlp **out);
void lsg_mlp_destroy(lsg_mlp *m);
int lsg_mlp_get_params(const lsg_mlp *m, float *params);
/* out[r] = network output o for rows r < rows (device buffers, X rows x F) */
int lsg_mlp_forward(lsg_mlp *m, const float *X, int64_t rows, float *out, void *stream);
/* gradient of mean_r (log softplus(o_r) - Y_r)^2 w.r.t. the FP32 parameters (host
 * copy; may be NULL) and the loss (host; may be NULL); X, Y device buffers */
int lsg_mlp_gradient(lsg_mlp *m, const float *X, const float *Y, int64_t rows, float *grad, float *loss);
/* one Adam step (beta 0.9/0.999) on that loss */
int lsg_mlp_train_step(lsg_mlp *m, const float *X, const float *Y, int64_t rows, float lr, float *loss);
const char *lsg_mlp_last_error(void);
/* features (device, n x (7d+5) floats) and the cheap base diagonal (device, n doubles) */
int lsg_operator_features(lsg_operator *op, float *feat, void *stream);
int lsg_operator_base_diag(lsg_operator *op, double *base, void *stream);
/* D = base * softplus(mlp(features)) at active points, installed for precond = 2 */
int lsg_operator_install_learned(lsg_operator *op, lsg_mlp *m, void *stream);

/* Selects the bilinear form of the matvec and the diagonal: LSG_FORM_STIFFNESS
 * (default; -div(a grad u)) or LSG_FORM_MASS (a u, the reference's HelmHoltz
 * operator for a = 1: right-hand sides <f, psi_i> from nodal values of f and
 * L2 norms u^T M u).  The CG solvers take either form. */
int lsg_operator_set_form(lsg_operator *op, int32_t form);

/* ---- prewavelet basis transforms (BasisTransformations/BasisTransformations.cpp).
 * lsg_calc_nodal_by_prew: u = values at every grid point (hanging included) of
 * the expansion sum_i prew_i psi_i over all points (calcNodalByPrew, :670-706).
 * lsg_calc_prew_by_nodal: prew = its inverse from the values of u at the active
 * points, 0 at hanging points (calcPrewByNodal, :486-545); u is not modified.
 * Vectors of n doubles in storage order; the tables are built on first use. */
int lsg_calc_nodal_by_prew(lsg_operator *op, const double *prew, double *u);
int lsg_calc_prew_by_nodal(lsg_operator *op, double *prew, const double *u);
int lsg_calc_nodal_by_prew_device(lsg_operator *op, const double *prew, double *u, void *stream);
int lsg_calc_prew_by_nodal_device(lsg_operator *op, double *prew, const double *u, void *stream);
/* H1 seminorm and L2 norm of the function with nodal values u (n doubles,
 * host): H1::getValue / L2::getValue (applications/H1_Norm.cpp): prewavelet
 * coefficients v = calcPrewByNodal(u), value = sqrt(sum over active points of
 * v_i (A v)_i) with A the coefficient-1 stiffness (Poisson) or mass
 * (HelmHoltz) operator; the operator's own coefficient and form stay set. */
int lsg_h1_norm(lsg_operator *op, const double *u, double *value);
int lsg_l2_norm(lsg_operator *op, const double *u, double *value);

/* ---- boundary-data right-hand sides (MatrixVectorMultiplication/RHS.h:278-427,
 * RHS.cpp:6-41,697-1008).  The boundary values g live on a second grid that
 * holds boundary points (a 1D index 0 or 1 in some dimension), e.g. the
 * operator's grid completed by completeNeumannGrid (lsg_grid_adaptive, bit 64
 * of `complete`); nn points, nn x d 1D indices in that grid's storage order.
 * lsg_hierarchize_boundary: CalcHierarchicalBasisForRHS in place on u (nn
 * host doubles): every boundary point loses half the sum of its 1D parents,
 * dimension by dimension, finest depth first; interior entries are untouched;
 * LSG_E_INVALID when a parent is missing from the grid.
 * lsg_boundary_rhs: rhs at the active points of the operator's grid =
 * InHomoBoundaryRHSHierarchical::multiply (LSG_BDRHS_GRADIENT: integrals of
 * grad psi_i . grad g), multiply_mass (LSG_BDRHS_MASS: psi_i g) or
 * multiply_mass_coeff (LSG_BDRHS_MASS_COEFF: psi_i g prod_k (1 - x_k^2)) of
 * the hierarchical coefficients `hier` of the second grid (only its boundary
 * points are read); other entries of rhs keep their values.  Results equal the
 * reference's to the bit.  Host arrays; the _device form takes hier and rhs
 * in device memory (points stay on the host) and runs on `stream`.  The
 * operator needs no coefficient; its tables are built on first use. */
#define LSG_BDRHS_GRADIENT 0
#define LSG_BDRHS_MASS 1
#define LSG_BDRHS_MASS_COEFF 2
int lsg_hierarchize_boundary(int32_t d, int64_t nn, const int32_t *points, double *u);
int lsg_boundary_rhs(lsg_operator *op, int32_t kind, int64_t nn, const int32_t *points, const double *hier,
                     double *rhs);
int lsg_boundary_rhs_device(lsg_operator *op, int32_t kind, int64_t nn, const int32_t *points, const double *hier,
                            double *rhs, void *stream);

/* CalcHierarchicalBasis(u) / CalcNodalBasis(u) (BasisTransformations/
 * BasisTransformations.cpp:390-409, :174-198) on any grid, boundary points
 * included: in place on u (n host doubles in storage order), dimension by
 * dimension; active points only, an absent 1D neighbour reads 0. */
int lsg_hierarchize(int32_t d, int64_t n, const int32_t *points, const uint8_t *active, double *u);
int lsg_dehierarchize(int32_t d, int64_t n, const int32_t *points, const uint8_t *active, double *u);

/* Right-hand side of -lap u = f (LSG_PDE_POISSON, PDE_Poisson_InHomRHS::SetUp,
 * applications/PDE.cpp:9-52) or -lap u + c u = f with c = prod_k (1 - x_k^2)
 * (LSG_PDE_HELMHOLTZ, PDE_Helmholtz_VariableCoeff::SetUp, PDE.h:62-114),
 * u = g on the boundary, on the operator's grid: rhs = <f_inner, psi_i> +
 * <f_boundary, psi_i> - <grad g, grad psi_i> (- <c g, psi_i>).  f holds values
 * at every point, g at the boundary points of the grid with boundary points
 * (nn points, nn x d 1D indices, its active flags); rhs gets n values (0 at
 * hanging points).  As in the reference, f and g are transformed in place:
 * f to hierarchical coefficients with its active interior entries moved out (0), g
 * to hierarchical boundary coefficients.  Host arrays; no coefficient needed. */
#define LSG_PDE_POISSON 0
#define LSG_PDE_HELMHOLTZ 1
int lsg_pde_boundary_rhs(lsg_operator *op, int32_t kind, int64_t nn, const int32_t *npoints, const uint8_t *nactive,
                         double *f, double *g, double *rhs);

/* ---- launch parameters of the matvec and the autotuner that picks them.
 * The defaults (256, 72, 4, 256, 2048, 256) suit large d=5/6 grids;
 * lsg_operator_autotune times matvecs of this operator over a candidate set
 * per parameter (coordinate descent, two passes, best of `reps` timings per
 * setting) and keeps the fastest setting.  Changing cell_space_kb re-plans the
 * dense slabs (and re-orders their collapsed coefficients).
 * No counterpart in the reference (OpenMP schedule only). */
typedef struct {
    int32_t cell_threads;    /* threads per cell-operator CTA: 64..256, multiple of 32 */
    int32_t cell_space_kb;   /* shared-memory work space per cell-operator CTA in KB: 16..200 */
    int32_t class_ratio;     /* work-space (slab-size) ratio that starts a new cell-operator launch: 2..1024 */
    int32_t level_threads;   /* threads per restriction-wavefront CTA: 32..512, multiple of 32 */
    int32_t level_cap;       /* shared-memory elements per wavefront ping-pong buffer: 256..65536 */
    int32_t prolong_threads; /* threads per prolongation CTA: 32..1024, multiple of 32 */
} lsg_tuning;
int lsg_operator_get_tuning(const lsg_operator *op, lsg_tuning *t);
int lsg_operator_set_tuning(lsg_operator *op, const lsg_tuning *t);
/* best (may be NULL): the setting kept; best_ms / default_ms (may be NULL):
 * ms per matvec with it and with the setting the operator had on entry */
int lsg_operator_autotune(lsg_operator *op, int32_t precision, int32_t reps, lsg_tuning *best, double *best_ms,
                          double *default_ms);

/* ---- batched operators and solves: many grids of uneven size (any mix of
 * dimensions), each with its own coefficient and right-hand side, applied and
 * solved together.  Grids of one dimension are concatenated into one
 * operator, so a matvec of the whole group is one launch per level step; the
 * batched CG keeps per-grid scalars and convergence, and one iteration of the
 * whole batch is captured as one CUDA graph.  A batch vector holds the grids'
 * vectors side by side: grid i occupies [offsets[i], offsets[i+1]) in storage
 * order (lsg_batch_offsets; grids are grouped by dimension, so the order of
 * the ranges can differ from the input order).  No counterpart in the
 * reference, which builds one MatrixVectorHomogen per grid
 * (MatrixVectorMultiplication/MatrixVectorHomogen.h:72-77). */
typedef struct lsg_batch lsg_batch;
int lsg_batch_create(int32_t count, const int32_t *dims, const int32_t *const *points, const uint8_t *const *active,
                     const int64_t *n, lsg_batch **out);
void lsg_batch_destroy(lsg_batch *b);
int64_t lsg_batch_size(const lsg_batch *b);
/* offsets[i] = start of grid i in a batch vector; offsets[count] = total size */
int lsg_batch_offsets(const lsg_batch *b, int64_t *offsets);
int lsg_batch_set_coefficient(lsg_batch *b, int32_t grid, int32_t family, const double *params, int32_t nparams);
/* y = A x for every grid (device batch vectors; inactive entries untouched) */
int lsg_batch_matvec_device(lsg_batch *b, const void *x, void *y, int32_t precision, void *stream);
/* CG of every grid (precond 0 or 1; FP64 or FP32+IR); reports[count] per grid
 * and *total for the batch (may be NULL).  Device / host batch vectors. */
int lsg_batch_cg_solve_device(lsg_batch *b, const double *f, double *x, const lsg_solver_opts *opts,
                              lsg_solve_report *reports, lsg_solve_report *total, void *stream);
int lsg_batch_cg_solve(lsg_batch *b, const double *f, double *x, const lsg_solver_opts *opts,
                       lsg_solve_report *reports, lsg_solve_report *total);
/* autotunes the operator of every dimension group of the batch */
int lsg_batch_autotune(lsg_batch *b, int32_t precision, int32_t reps);

/* ---- host-only planner (no GPU needed): the flattened integer tables.
 * lsg_plan_create builds the same tables lsg_operator_create uploads, so the
 * tests can check them bit-exact against the reference's lookups on a CPU. */
typedef struct lsg_plan lsg_plan;
int lsg_plan_create(int32_t d, const int32_t *points, const uint8_t *active, int64_t n, lsg_plan **out);
void lsg_plan_destroy(lsg_plan *plan);
int lsg_plan_info(const lsg_plan *plan, lsg_info *info);
/* DepthList order (iterator/depthIterator.h:14-50): n_depths*d */
int lsg_plan_export_depths(const lsg_plan *plan, int32_t *depths);
/* sortDepths(case c) (iterator/depthIterator.cpp:7-45) as depth ids; *count <= n_depths */
int lsg_plan_export_sorted_depths(const lsg_plan *plan, int32_t c, int32_t *depth_ids, int32_t *count);
/* cells of depth T+1 in the grid per depth (CellData, cells/CellStructure.h:23-61) */
int lsg_plan_export_cell_counts(const lsg_plan *plan, int64_t *counts);
/* Diagnostic for the CPU tests: applies the level-T cell operator of one dense
 * slab (depth id t) to u, given per-cell coefficients acell (the slab's cells,
 * dim 0 fastest), twice on the host: cell by cell as
 * LocalStiffnessMatrices::applyLocalMatrix does
 * (localStiffnessMatrices/LocalStiffnessMatrices.cpp:555-582) -> z_cells, and in
 * the factorised form of the GPU kernel, planned for a work space of wcap
 * elements and a register dimension of at most na_max nodes -> z_sf.
 * info (6 entries, may be NULL): mid dims, chunked dims, chunks, a extent,
 * b extent (0 = none), collapsed dims. */
int lsg_plan_check_slab_operator(const lsg_plan *plan, int32_t t, int32_t form, int64_t wcap, int32_t na_max,
                                 const double *acell, const double *u, double *z_cells, double *z_sf,
                                 int32_t *info);
/* corners (storage index or -1) of every cell of one depth, 2^d per cell,
 * corner id bit k = right side in dim k; cells ordered by min corner */
int lsg_plan_export_cells(const lsg_plan *plan, int32_t depth_id, int64_t *corners, int64_t *count);
/* storage indices of the points with depth <= T (multilevel entries (I,T)) */
int lsg_plan_export_slab(const lsg_plan *plan, int32_t depth_id, int64_t *storage_idx, int64_t *count);
/* same-level neighbours nextLeft/nextRight (indices/index.h:749-789): n*d*2 storage indices or -1 */
int lsg_plan_export_neighbors(const lsg_plan *plan, int64_t *nbr);
/* prewavelet stencil of point k (nextFiveP, indices/index.cc:252-327) in
 * MultiDimFiveCompass order: storage index (or -1 if absent) and weight; at most 5^d */
int lsg_plan_export_stencil(const lsg_plan *plan, int64_t k, int64_t *idx, double *w, int32_t *count);

/* Regular sparse grid AddRecursiveSonsOfPoint(center, level)
 * (sgrid/sparseGrid.cc:557-566) in the reference's storage order; all points
 * active.  Pass points = NULL to query *n. */
int lsg_grid_regular(int32_t d, int32_t level, int32_t *points, int64_t capacity, int64_t *n);

/* Adaptive grid: AddRecursiveSonsOfPoint(center, level), then `refine`
 * rounds adding the sons of every active point with max_k x_k < theta 2^(1-r)
 * (target 0, toward the corner) or |x_0 - 1/2| < theta 2^(1-r) (target 1,
 * toward a hyperplane), then, if `complete`, the reference's completion
 * AdaptiveSparseGrid::completeDirichletGrid (sgrid/sparseGrid.cc:771-787)
 * including hanging nodes.  Storage order as the reference inserts.  The
 * last completion stage (addPoints2, sgrid/GridGeneration.cpp:333-392) visits
 * the reference's pairs of points in its order through the grid's index (1.4 s
 * on a 1.5M-point d=6 grid).  `complete` 1 runs every stage; a larger value is a bit
 * mask of stages (2, 4, 8: the completion passes, 16: hanging nodes, 32:
 * addPoints2), and bit 64 adds completeNeumannGrid (sgrid/sparseGrid.cc:
 * 654-740) at the end: the boundary points of a grid for boundary data.
 * Pass points = active = NULL to query *n. */
int lsg_grid_adaptive(int32_t d, int32_t level, int32_t refine, double theta, int32_t target, int32_t complete,
                      int32_t *points, uint8_t *active, int64_t capacity, int64_t *n);

/* Completion of a caller's grid (points n x d in storage order, active flags):
 * `complete` as for lsg_grid_adaptive (1: completeDirichletGrid,
 * sgrid/sparseGrid.cc:771-787, with its hanging nodes; 64:
 * completeNeumannGrid).  The given points keep their order and flags; added
 * points follow in the reference's insertion order.  Pass out_points =
 * out_active = NULL to query *n_out. */
int lsg_grid_complete(int32_t d, int64_t n, const int32_t *points, const uint8_t *active, int32_t complete,
                      int32_t *out_points, uint8_t *out_active, int64_t capacity, int64_t *n_out);

const char *lsg_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
