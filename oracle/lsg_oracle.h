/*
 * lsg_oracle -- CPU restatement of LoAdSG's prewavelet matvec and CG.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py load this library, and only
 * as the checker.  The product (loadsg_b200) never links or calls it.
 *
 * It follows the reference's algorithm step by step, on full-length vectors
 * indexed by storage index, with a hash map standing in for the reference's
 * hash grids.  Every function cites the reference code it restates
 * (paths relative to library/source/).  Parity with the compiled reference is
 * pinned by the .npz fixtures in tests/golden, generated by oracle/ref_harness.cpp.
 */
#ifndef LSG_ORACLE_H
#define LSG_ORACLE_H
#include <stdint.h>

typedef struct lsgo_grid lsgo_grid;

/* points: N*d 1D indices in storage order; active: N flags (1 = active). */
lsgo_grid *lsgo_grid_create(int d, const int32_t *points, const uint8_t *active, int64_t n);
void lsgo_grid_free(lsgo_grid *g);

/* DepthList (iterator/depthIterator.h:14-50): depths in first-appearance order. */
int lsgo_num_depths(const lsgo_grid *g);
void lsgo_depths(const lsgo_grid *g, int32_t *out /* num_depths*d */);
/* sortDepths (iterator/depthIterator.cpp:7-45) for case bit mask c; returns count. */
int lsgo_sorted_depths(const lsgo_grid *g, int c, int32_t *out /* num_depths*d */);
/* Number of cells of depth T+1 inside the grid (cells/CellStructure.h:23-61). */
int64_t lsgo_num_cells(const lsgo_grid *g, const int32_t *T);
/* Storage index of a point given by its d 1D indices, or -1. */
int64_t lsgo_lookup(const lsgo_grid *g, const int32_t *idx);

/* y[active] = A_prew x  (MatrixVectorHomogen::multiplication over
 * LocalStiffnessMatrices with the midpoint-coefficient plugin); entries of y at
 * hanging nodes are left untouched, as in the reference. */
int lsgo_matvec(lsgo_grid *g, int family, const double *params, const double *x, double *y);
/* Jacobi diagonal a(psi_i, psi_i) (Preconditioning::precondLocalStiffnessMatrix). */
int lsgo_diag(lsgo_grid *g, int family, const double *params, double *diag);
/* CG::solveHomogen with the reference stopping rule (delta = r^T D^-1 r > eps,
 * break when delta' < eps^2, at most maxit iterations).  x is in/out. */
int lsgo_cg(lsgo_grid *g, int family, const double *params, const double *f, double *x, double eps,
            int maxit, int *iterations);

/* Local matrix of the plugin used by lsgo_matvec / lsgo_diag / lsgo_cg:
 * 0 = a(x_c) * Q1 stiffness (default), 1 = a(x_c) * Q1 mass (HelmHoltz). */
void lsgo_set_form(lsgo_grid *g, int form);

/* calcNodalByPrew (BasisTransformations/BasisTransformations.cpp:670-706):
 * u = values at every point of the expansion sum_i prew_i psi_i (all points). */
int lsgo_nodal_by_prew(lsgo_grid *g, const double *prew, double *u);

/* Boundary-data right-hand sides (MatrixVectorMultiplication/RHS.cpp, RHS.h).
 * ng is a grid with boundary points (completeNeumannGrid).
 * lsgo_hierarchize_boundary: CalcHierarchicalBasisForRHS on u (ng's storage
 * order), in place at the boundary points.  lsgo_boundary_rhs: y at the active
 * points of g = InHomoBoundaryRHSHierarchical::multiply (kind 0),
 * multiply_mass (1) or multiply_mass_coeff (2) of the hierarchical boundary
 * coefficients hier (ng's storage order); other entries of y are untouched. */
int lsgo_hierarchize_boundary(lsgo_grid *ng, double *u);
int lsgo_boundary_rhs(lsgo_grid *g, lsgo_grid *ng, int kind, const double *hier, double *y);
/* sign -1: CalcHierarchicalBasis(u) (BasisTransformations.cpp:390-409);
 * sign +1: CalcNodalBasis(u) (:174-198); in place, active points only. */
int lsgo_hierarchize(lsgo_grid *g, double *u, int sign);

#endif
