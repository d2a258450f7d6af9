/*
 * lsg_oracle.c -- CPU restatement of LoAdSG's variable-coefficient prewavelet
 * matvec (MatrixVectorHomogen::multiplication over LocalStiffnessMatrices) and
 * of CG::solveHomogen.  TEST INFRASTRUCTURE ONLY (see lsg_oracle.h).
 *
 * Paths cited are relative to the reference's library/source/ directory.
 * The data layout follows the reference: every vector is a full-length array
 * indexed by storage index; the multilevel store (I,T) is one full-length
 * array per depth T of the depth list, of which only the entries with
 * Depth(I) <= T are meaningful (sgrid/multilevelSparseGrid.cpp:9-34).
 */
#include "lsg_oracle.h"
#include "coefficient.h"

#include <stdlib.h>
#include <string.h>

#define MAXD 16

struct lsgo_grid {
    int d;
    int64_t n;
    int32_t *pts;   /* n*d 1D indices */
    uint8_t *act;   /* n */
    int32_t *dep;   /* n*d depths */
    int64_t cap;    /* hash capacity (power of two) */
    int64_t *slot;  /* storage index or -1 */
    int nD;         /* depth list */
    int32_t *D;     /* nD*d */
    int32_t *did;   /* per point: position of its depth in the depth list */
    int32_t maxdep[MAXD];
    int form;        /* 0 stiffness (diffusion), 1 mass: the local matrix of the plugin */
    int64_t *ex_off; /* points of exact depth, storage order */
    int64_t *ex;
    struct celllist **cells; /* per depth, built on first use */
};

/* in-grid cells of depth T+1 for one depth T of the depth list */
typedef struct celllist {
    int64_t nc;
    int32_t *center;  /* nc*d centre 1D indices */
    int64_t *corner;  /* nc*2^d storage index or -1; bit k of the corner id = right in dim k */
    double *xc;       /* nc*d midpoints */
    double h[16];     /* cell widths (equal for all cells of one depth) */
    int64_t cap;      /* hash of centres -> cell id */
    int64_t *slot;
} celllist;

/* ------------------------------------------------------------ 1D index algebra
 * indices/index.h:656-871: root 2, sons 2i and 2i+1, boundary points 0 and 1. */
static int depth1(int32_t i) { return i == 0 ? 0 : 31 - __builtin_clz((unsigned)i); }
static int intern_depth1(int32_t i) { return i == 0 ? -1 : 31 - __builtin_clz((unsigned)i); }
static int32_t next_left1(int32_t i) { return i >> (__builtin_ctz((unsigned)i) + 1); }
static int32_t next_right1(int32_t i) { return i >> (__builtin_ctz(~(unsigned)i) + 1); }
static int32_t next_left_lv(int32_t i, int level) { /* index.h:834-847 */
    int lv = level - depth1(i);
    if (lv == 0) return next_left1(i);
    i <<= 1;
    for (int k = 1; k < lv; ++k) i = (i << 1) + 1;
    return i;
}
static int32_t next_right_lv(int32_t i, int level) { /* index.h:855-866 */
    int lv = level - intern_depth1(i);
    if (lv == 0) return next_right1(i);
    i = (i << 1) + 1;
    for (int k = 1; k < lv; ++k) i <<= 1;
    return i;
}
static double coord1(int32_t i) { /* index.h:718-730 */
    if (i == 0) return 0.0;
    int t = depth1(i);
    double h = 1.0 / (double)(1u << t);
    int32_t nn = i & ~(1 << t);
    return (double)(2 * nn + 1) * h;
}
static int interior1(int32_t i) { return i != 0 && i != 1; }

/* One-dimensional factor of the prewavelet stencil of a point with 1D index i
 * at depth t (IndexDimension::nextFiveP, indices/index.cc:252-327): order
 * Mitte, Links, Rechts, LinksLinks, RechtsRechts; invalid directions (a
 * neighbour on the boundary) are skipped.  Weights 1 (0.9 next to the boundary
 * for depth > 1), -0.6, 0.1. */
static int stencil1(int32_t i, int t, int32_t *j, double *w) {
    int n = 0;
    int32_t l = next_left1(i), r = next_right1(i);
    int randnah = (l == 0) || (r == 1);
    j[n] = i;
    w[n++] = (depth1(i) > 1 && randnah) ? 0.9 : 1.0;
    if (interior1(l)) { j[n] = l; w[n++] = -0.6; }
    if (interior1(r)) { j[n] = r; w[n++] = -0.6; }
    if (interior1(l)) { j[n] = next_left_lv(l, t); w[n++] = 0.1; }
    if (interior1(r)) { j[n] = next_right_lv(r, t); w[n++] = 0.1; }
    return n;
}

/* ------------------------------------------------------------ hash of points */
static uint64_t hash_idx(const int32_t *idx, int d) {
    uint64_t h = 0x9E3779B97F4A7C15ull;
    for (int k = 0; k < d; ++k) {
        h ^= (uint64_t)(uint32_t)idx[k] + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
        h *= 0xBF58476D1CE4E5B9ull;
    }
    return h ^ (h >> 31);
}
int64_t lsgo_lookup(const lsgo_grid *g, const int32_t *idx) {
    uint64_t m = (uint64_t)g->cap - 1, h = hash_idx(idx, g->d) & m;
    for (;;) {
        int64_t s = g->slot[h];
        if (s < 0) return -1;
        if (memcmp(g->pts + s * g->d, idx, sizeof(int32_t) * g->d) == 0) return s;
        h = (h + 1) & m;
    }
}

static int depth_eq(const int32_t *a, const int32_t *b, int d) {
    for (int k = 0; k < d; ++k)
        if (a[k] != b[k]) return 0;
    return 1;
}
static int depth_le(const int32_t *a, const int32_t *b, int d) {
    for (int k = 0; k < d; ++k)
        if (a[k] > b[k]) return 0;
    return 1;
}
static int find_depth(const lsgo_grid *g, const int32_t *T) { /* DepthList::isIncluded */
    for (int t = 0; t < g->nD; ++t)
        if (depth_eq(g->D + t * g->d, T, g->d)) return t;
    return -1;
}

lsgo_grid *lsgo_grid_create(int d, const int32_t *points, const uint8_t *active, int64_t n) {
    if (d < 1 || d > MAXD || n < 1) return NULL;
    lsgo_grid *g = calloc(1, sizeof *g);
    g->d = d;
    g->n = n;
    g->pts = malloc(sizeof(int32_t) * n * d);
    memcpy(g->pts, points, sizeof(int32_t) * n * d);
    g->act = malloc(n);
    memcpy(g->act, active, n);
    g->dep = malloc(sizeof(int32_t) * n * d);
    for (int64_t k = 0; k < n * d; ++k) g->dep[k] = depth1(points[k]);
    g->cap = 1;
    while (g->cap < 2 * n) g->cap <<= 1;
    g->slot = malloc(sizeof(int64_t) * g->cap);
    for (int64_t k = 0; k < g->cap; ++k) g->slot[k] = -1;
    for (int64_t k = 0; k < n; ++k) {
        uint64_t m = (uint64_t)g->cap - 1, h = hash_idx(points + k * d, d) & m;
        while (g->slot[h] >= 0) h = (h + 1) & m;
        g->slot[h] = k;
    }
    /* DepthList ctor (iterator/depthIterator.h:14-50): first appearance order */
    g->D = malloc(sizeof(int32_t) * n * d);
    g->did = malloc(sizeof(int32_t) * n);
    g->nD = 0;
    for (int64_t k = 0; k < n; ++k) {
        int t = find_depth(g, g->dep + k * d);
        if (t < 0) {
            t = g->nD++;
            memcpy(g->D + t * d, g->dep + k * d, sizeof(int32_t) * d);
        }
        g->did[k] = t;
    }
    for (int k = 0; k < d; ++k) g->maxdep[k] = 0;
    for (int t = 0; t < g->nD; ++t)
        for (int k = 0; k < d; ++k)
            if (g->D[t * d + k] > g->maxdep[k]) g->maxdep[k] = g->D[t * d + k];
    /* points of exact depth (SingleDepthHashGrid::_mapPosToGridPos), storage order */
    g->ex_off = calloc(g->nD + 1, sizeof(int64_t));
    for (int64_t k = 0; k < n; ++k) g->ex_off[g->did[k] + 1]++;
    for (int t = 0; t < g->nD; ++t) g->ex_off[t + 1] += g->ex_off[t];
    g->ex = malloc(sizeof(int64_t) * n);
    int64_t *fill = calloc(g->nD, sizeof(int64_t));
    for (int64_t k = 0; k < n; ++k) g->ex[g->ex_off[g->did[k]] + fill[g->did[k]]++] = k;
    free(fill);
    return g;
}

void lsgo_grid_free(lsgo_grid *g) {
    if (!g) return;
    free(g->pts); free(g->act); free(g->dep); free(g->slot); free(g->D); free(g->did);
    free(g->ex_off); free(g->ex);
    if (g->cells) {
        for (int t = 0; t < g->nD; ++t) {
            celllist *cl = g->cells[t];
            if (!cl) continue;
            free(cl->center); free(cl->corner); free(cl->xc); free(cl->slot); free(cl);
        }
        free(g->cells);
    }
    free(g);
}

int lsgo_num_depths(const lsgo_grid *g) { return g->nD; }
void lsgo_depths(const lsgo_grid *g, int32_t *out) { memcpy(out, g->D, sizeof(int32_t) * g->nD * g->d); }

/* DepthList::recursiveDepth (iterator/depthIterator.cpp:7-45) */
static void rec_depth(const lsgo_grid *g, int c, int checkProl, int dd, int32_t *T, int32_t *out, int *cnt) {
    int d = g->d;
    if (checkProl && dd > 0) {
        if (!((c >> dd) & 1)) {
            for (int t = 1; t <= g->maxdep[dd]; ++t) { T[dd] = t; rec_depth(g, c, checkProl, dd - 1, T, out, cnt); }
        } else rec_depth(g, c, checkProl, dd - 1, T, out, cnt);
    }
    if (checkProl && dd == 0) {
        if (!(c & 1)) {
            for (int t = 1; t <= g->maxdep[0]; ++t) { T[0] = t; rec_depth(g, c, 0, d - 1, T, out, cnt); }
        } else rec_depth(g, c, 0, d - 1, T, out, cnt);
    }
    if (!checkProl && dd >= 0) {
        if ((c >> dd) & 1) {
            for (int t = g->maxdep[dd]; t > 1; --t) { T[dd] = t; rec_depth(g, c, checkProl, dd - 1, T, out, cnt); }
        } else rec_depth(g, c, checkProl, dd - 1, T, out, cnt);
    }
    if (dd < 0 && find_depth(g, T) >= 0) {
        memcpy(out + (*cnt) * d, T, sizeof(int32_t) * d);
        (*cnt)++;
    }
}
int lsgo_sorted_depths(const lsgo_grid *g, int c, int32_t *out) {
    int32_t T[MAXD] = {0};
    int cnt = 0;
    rec_depth(g, c, 1, g->d - 1, T, out, &cnt);
    return cnt;
}

/* ------------------------------------------------------------ cells
 * A cell of depth T+1 is given by its centre (1D indices at level T_k+1); its
 * corners are next_left1/next_right1 of the centre (cells/iterator_neu.h:65-99).
 * It belongs to the grid when all non-boundary corners exist
 * (CellData::cellingrid, cells/CellStructure.h:50-59). */
static uint64_t hash_cell(const int32_t *c, int d) { return hash_idx(c, d) * 0x94D049BB133111EBull; }

/* corners of the cell with the given centre; returns 0 if a non-boundary corner is missing */
static int cell_corners(const lsgo_grid *g, const int32_t *center, int64_t *corner, double *h, double *xc) {
    int d = g->d;
    int32_t lo[MAXD], hi[MAXD], idx[MAXD];
    for (int k = 0; k < d; ++k) {
        lo[k] = next_left1(center[k]);
        hi[k] = next_right1(center[k]);
        double a = coord1(lo[k]), b = coord1(hi[k]);
        if (h) h[k] = b - a;
        if (xc) xc[k] = 0.5 * (a + b);
    }
    for (unsigned m = 0; m < (1u << d); ++m) {
        int bnd = 0;
        for (int k = 0; k < d; ++k) {
            idx[k] = ((m >> k) & 1) ? hi[k] : lo[k];
            if (!interior1(idx[k])) bnd = 1;
        }
        if (bnd) { corner[m] = -1; continue; }
        int64_t s = lsgo_lookup(g, idx);
        if (s < 0) return 0;
        corner[m] = s;
    }
    return 1;
}

/* CellData (cells/CellStructure.h:23-47): all level-T cells whose non-boundary
 * corners are in the grid. */
static celllist *get_cells(lsgo_grid *g, int t) {
    if (!g->cells) g->cells = calloc(g->nD, sizeof(celllist *));
    if (g->cells[t]) return g->cells[t];
    int d = g->d;
    const int32_t *T = g->D + t * d;
    int64_t total = 1;
    for (int k = 0; k < d; ++k) total *= (int64_t)1 << T[k];
    celllist *cl = calloc(1, sizeof *cl);
    int64_t capc = 16;
    cl->center = malloc(sizeof(int32_t) * capc * d);
    cl->corner = malloc(sizeof(int64_t) * capc << d);
    cl->xc = malloc(sizeof(double) * capc * d);
    int32_t center[MAXD];
    int64_t *corner = malloc(sizeof(int64_t) << d);
    double xc[MAXD];
    for (int64_t lin = 0; lin < total; ++lin) {
        int64_t r = lin;
        for (int k = 0; k < d; ++k) {
            int64_t nk = (int64_t)1 << T[k];
            int64_t j = r % nk;
            r /= nk;
            center[k] = (int32_t)(((int64_t)1 << (T[k] + 1)) + j);
        }
        if (!cell_corners(g, center, corner, cl->h, xc)) continue;
        if (cl->nc == capc) {
            capc *= 2;
            cl->center = realloc(cl->center, sizeof(int32_t) * capc * d);
            cl->corner = realloc(cl->corner, sizeof(int64_t) * capc << d);
            cl->xc = realloc(cl->xc, sizeof(double) * capc * d);
        }
        memcpy(cl->center + cl->nc * d, center, sizeof(int32_t) * d);
        memcpy(cl->corner + (cl->nc << d), corner, sizeof(int64_t) << d);
        memcpy(cl->xc + cl->nc * d, xc, sizeof(double) * d);
        cl->nc++;
    }
    free(corner);
    cl->cap = 1;
    while (cl->cap < 2 * cl->nc + 2) cl->cap <<= 1;
    cl->slot = malloc(sizeof(int64_t) * cl->cap);
    for (int64_t k = 0; k < cl->cap; ++k) cl->slot[k] = -1;
    for (int64_t c = 0; c < cl->nc; ++c) {
        uint64_t m = (uint64_t)cl->cap - 1, hsh = hash_cell(cl->center + c * d, d) & m;
        while (cl->slot[hsh] >= 0) hsh = (hsh + 1) & m;
        cl->slot[hsh] = c;
    }
    g->cells[t] = cl;
    return cl;
}
static int64_t find_cell(const lsgo_grid *g, const celllist *cl, const int32_t *center) {
    uint64_t m = (uint64_t)cl->cap - 1, hsh = hash_cell(center, g->d) & m;
    for (;;) {
        int64_t s = cl->slot[hsh];
        if (s < 0) return -1;
        if (memcmp(cl->center + s * g->d, center, sizeof(int32_t) * g->d) == 0) return s;
        hsh = (hsh + 1) & m;
    }
}
int64_t lsgo_num_cells(const lsgo_grid *g, const int32_t *T) {
    int t = find_depth(g, T);
    if (t < 0) return -1;
    return get_cells((lsgo_grid *)g, t)->nc;
}

/* LocalStiffnessMatrixFixedDepthSymmetric::setValues + applyLocalMatrix
 * (localStiffnessMatrices/LocalStiffnessMatrices.cpp:504-582): for corner pairs
 * p <= q with both corners in the grid, z[q] += K u[p] and, if p != q,
 * z[p] += K u[q]. */
static void cells_apply(lsgo_grid *g, int t, int family, const double *params, const double *u, double *z) {
    int d = g->d;
    const unsigned nc = 1u << d;
    celllist *cl = get_cells(g, t);
    /* the Q1 entries depend only on the cell widths, equal for all cells of one
     * depth: one table per call, the same values the plugin returns per cell */
    double *K = malloc(sizeof(double) * nc * nc);
    for (unsigned p = 0; p < nc; ++p)
        for (unsigned q = p; q < nc; ++q) K[p * nc + q] = lsg_q1_entry(g->form, d, cl->h, p, q);
    for (int64_t c = 0; c < cl->nc; ++c) {
        const int64_t *corner = cl->corner + (c << d);
        double a = lsg_coef_eval(family, params, d, cl->xc + c * d);
        for (unsigned p = 0; p < nc; ++p) {
            int64_t kp = corner[p];
            if (kp < 0) continue;
            for (unsigned q = p; q < nc; ++q) {
                int64_t kq = corner[q];
                if (kq < 0) continue;
                double val = a * K[p * nc + q];
                if (p == q) z[kq] += val * u[kp];
                else {
                    z[kq] += val * u[kp];
                    z[kp] += val * u[kq];
                }
            }
        }
    }
    free(K);
}

/* ------------------------------------------------------------ stencils on points */
/* Tensor-product prewavelet stencil of point k at its own depth; calls fn(J,w). */
typedef struct {
    int n[MAXD];
    int32_t j[MAXD][5];
    double w[MAXD][5];
} stencil_t;
static void stencil_build(const lsgo_grid *g, int64_t k, stencil_t *s) {
    for (int dd = 0; dd < g->d; ++dd)
        s->n[dd] = stencil1(g->pts[k * g->d + dd], g->dep[k * g->d + dd], s->j[dd], s->w[dd]);
}
/* iterate combos with dim 0 fastest (MultiDimFiveCompass order) */
static int stencil_next(const lsgo_grid *g, const stencil_t *s, int *pos, int32_t *J, double *w) {
    int d = g->d;
    *w = 1.0;
    for (int dd = 0; dd < d; ++dd) {
        J[dd] = s->j[dd][pos[dd]];
        *w *= s->w[dd][pos[dd]];
    }
    for (int dd = 0; dd < d; ++dd) {
        if (++pos[dd] < s->n[dd]) return 1;
        pos[dd] = 0;
    }
    return 0; /* this was the last combination */
}

/* MatrixVectorHomogen::calcNodal (MatrixVectorMultiplication/MatrixVectorHomogen.cpp:43-74) */
static void calc_nodal(const lsgo_grid *g, int t, const double *prew, double *u) {
    int d = g->d;
    stencil_t s;
    int32_t J[MAXD];
    for (int64_t e = g->ex_off[t]; e < g->ex_off[t + 1]; ++e) {
        int64_t k = g->ex[e];
        if (!g->act[k]) continue;
        double coeff = prew[k], w;
        int pos[MAXD] = {0}, more;
        stencil_build(g, k, &s);
        do {
            more = stencil_next(g, &s, pos, J, &w);
            int64_t j = lsgo_lookup(g, J);
            if (j >= 0) u[j] = u[j] + coeff * w;
        } while (more);
    }
    (void)d;
}

/* MatrixVectorHomogen::ConvertToPrewavelet2 (MatrixVectorHomogen.h:540-562) */
static void convert_prew(const lsgo_grid *g, int t, const double *z, double *ax) {
    stencil_t s;
    int32_t J[MAXD];
    for (int64_t e = g->ex_off[t]; e < g->ex_off[t + 1]; ++e) {
        int64_t k = g->ex[e];
        if (!g->act[k]) continue;
        double coeff = 0.0, w;
        int pos[MAXD] = {0}, more;
        stencil_build(g, k, &s);
        do {
            more = stencil_next(g, &s, pos, J, &w);
            int64_t j = lsgo_lookup(g, J);
            coeff = coeff + (j >= 0 ? z[j] : 0.0) * w;
        } while (more);
        ax[k] = coeff;
    }
}

static int64_t nbr(const lsgo_grid *g, int64_t k, int dd, int right) {
    int32_t J[MAXD];
    memcpy(J, g->pts + k * g->d, sizeof(int32_t) * g->d);
    J[dd] = right ? next_right1(J[dd]) : next_left1(J[dd]);
    return lsgo_lookup(g, J);
}

/* MatrixVectorHomogen::prolongation1D_inplace (MatrixVectorHomogen.h:444-474) */
static void prolongation1d(const lsgo_grid *g, double *v, int t, int dd) {
    for (int td = 0; td < g->nD; ++td) {
        if (g->D[td * g->d + dd] != t) continue;
        for (int64_t e = g->ex_off[td]; e < g->ex_off[td + 1]; ++e) {
            int64_t k = g->ex[e];
            double value = v[k];
            if (interior1(g->pts[k * g->d + dd])) {
                int64_t r = nbr(g, k, dd, 1), l = nbr(g, k, dd, 0);
                value = value + 0.5 * ((r >= 0 ? v[r] : 0.0) + (l >= 0 ? v[l] : 0.0));
            }
            v[k] = value;
        }
    }
}

/* MatrixVectorHomogen::restriction1D_inverted_inplace (MatrixVectorHomogen.h:485-530) */
static void restriction1d(const lsgo_grid *g, double *v, int t, int dd) {
    int d = g->d;
    for (int td = 0; td < g->nD; ++td) {
        const int32_t *Tl = g->D + td * d;
        int pos = 1;
        for (int k = 0; k < d; ++k) if (Tl[k] <= 0) pos = 0;
        if (Tl[dd] != t + 1 || !pos) continue;
        for (int64_t e = g->ex_off[td]; e < g->ex_off[td + 1]; ++e) {
            int64_t k = g->ex[e];
            double value = 0.5 * v[k];
            if (t >= 0) {
                int32_t J[MAXD];
                memcpy(J, g->pts + k * d, sizeof(int32_t) * d);
                J[dd] = next_right1(g->pts[k * d + dd]);
                if (J[dd] != 1) { int64_t r = lsgo_lookup(g, J); if (r >= 0) v[r] += value; }
                J[dd] = next_left1(g->pts[k * d + dd]);
                if (J[dd] != 1) { int64_t l = lsgo_lookup(g, J); if (l >= 0) v[l] += value; }
            }
        }
    }
}

/* multilevel helpers: set / add over the points with Depth <= T
 * (VectorSparseG::setMultiLevelValues2 / addMultiLevelValues2, extemp/vector.cc:600-659;
 *  MultiLevelVector::setMultiLevelValues2 / addMultiLevelValues, extemp/multilevelvector.h:161-298) */
static void vec_from_ml(const lsgo_grid *g, const int32_t *T, const double *ml, double *v) {
    for (int64_t k = 0; k < g->n; ++k)
        if (depth_le(g->dep + k * g->d, T, g->d)) v[k] = ml[k];
}
static void vec_add_ml(const lsgo_grid *g, const int32_t *T, const double *ml, double *v) {
    for (int64_t k = 0; k < g->n; ++k)
        if (depth_le(g->dep + k * g->d, T, g->d)) v[k] += ml[k];
}
static void ml_from_vec(const lsgo_grid *g, const int32_t *T, const double *v, double *ml) {
    for (int64_t k = 0; k < g->n; ++k)
        if (depth_le(g->dep + k * g->d, T, g->d)) ml[k] = v[k];
}
static void ml_add_vec(const lsgo_grid *g, const int32_t *T, const double *v, double *ml) {
    for (int64_t k = 0; k < g->n; ++k)
        if (depth_le(g->dep + k * g->d, T, g->d)) ml[k] = ml[k] + v[k];
}

/* MatrixVectorHomogen::multiplication_LocalStiffnessMatrix_mpi (MatrixVectorHomogen.h:169-257,
 * serial branch) + caseFunction_LocalStiffnessMatrix (MatrixVectorHomogen.h:1618-1738). */
int lsgo_matvec(lsgo_grid *g, int family, const double *params, const double *x, double *y) {
    int d = g->d, nD = g->nD;
    int64_t n = g->n;
    size_t vb = sizeof(double) * (size_t)n;
    double *nodal = calloc((size_t)nD * n, sizeof(double));
    double *P = malloc((size_t)nD * vb);
    double *gM = malloc((size_t)nD * vb);
    double *u = malloc(vb), *z = malloc(vb), *gv = malloc(vb), *ax_neu = malloc(vb), *ax = malloc(vb);
    int32_t *sorted = malloc(sizeof(int32_t) * nD * d);
    if (!nodal || !P || !gM || !u || !z || !gv || !ax_neu || !ax || !sorted) return -1;
    for (int64_t k = 0; k < n; ++k) ax[k] = g->act[k] ? 0.0 : y[k]; /* Ax = 0.0 on active nodes */
    /* prewavelet -> nodal per depth (MatrixVectorHomogen.h:193-217) */
    for (int t = 0; t < nD; ++t) {
        memset(u, 0, vb);
        calc_nodal(g, t, x, u);
        ml_from_vec(g, g->D + t * d, u, nodal + (size_t)t * n);
    }
    for (int c = 0; c < (1 << d); ++c) { /* CasesIterator: bit i = restriction in dim i */
        memset(ax_neu, 0, vb);
        memset(gM, 0, (size_t)nD * vb);
        int ns = lsgo_sorted_depths(g, c, sorted);
        if (ns > 0) {
            memcpy(P, nodal, (size_t)nD * vb); /* P += nodal (an assignment) */
            for (int dd = 0; dd < d; ++dd) {
                if ((c >> dd) & 1) continue;
                for (int s = 0; s < ns; ++s) {
                    const int32_t *T = sorted + s * d;
                    int32_t Tf[MAXD];
                    memcpy(Tf, T, sizeof(int32_t) * d);
                    int t = T[dd] + 1;
                    Tf[dd] = t;
                    int tf = find_depth(g, Tf);
                    if (tf < 0) continue;
                    int ti = find_depth(g, T);
                    memset(u, 0, vb);
                    vec_from_ml(g, T, P + (size_t)ti * n, u);
                    prolongation1d(g, u, t, dd);
                    ml_add_vec(g, Tf, u, P + (size_t)tf * n);
                }
            }
            for (int s = 0; s < ns; ++s) {
                const int32_t *T = sorted + s * d;
                int ti = find_depth(g, T);
                memset(u, 0, vb);
                vec_from_ml(g, T, P + (size_t)ti * n, u);
                memset(z, 0, vb);
                cells_apply(g, ti, family, params, u, z);
                vec_add_ml(g, T, gM + (size_t)ti * n, z);
                int32_t Tc[MAXD];
                memcpy(Tc, T, sizeof(int32_t) * d);
                int tc = -1;
                for (int dd = 0; dd < d; ++dd) {
                    if (!((c >> dd) & 1)) continue;
                    Tc[dd] = T[dd] - 1;
                    tc = find_depth(g, Tc);
                    if (tc >= 0) {
                        restriction1d(g, z, Tc[dd], dd);
                        memcpy(gv, z, vb); /* g = z */
                        vec_add_ml(g, Tc, gM + (size_t)tc * n, z);
                        ml_from_vec(g, Tc, gv, gM + (size_t)tc * n);
                    }
                }
                tc = find_depth(g, Tc);
                if (tc >= 0) convert_prew(g, tc, z, ax_neu);
            }
        }
        for (int64_t k = 0; k < n; ++k) ax[k] = ax[k] + ax_neu[k]; /* Ax = Ax + Ax_neu */
    }
    memcpy(y, ax, vb);
    free(nodal); free(P); free(gM); free(u); free(z); free(gv); free(ax_neu); free(ax); free(sorted);
    return 0;
}

/* Preconditioning::precondLocalStiffnessMatrix (applications/cg_method.h:544-680):
 * diag_i = v^T A_T v with v the nodal values of psi_i on level T = Depth(i)
 * (set only at existing grid points) and A_T the level-T cell operator.  Only
 * cells with a corner in the stencil contribute: in each dimension the six
 * level-T cells whose centres lie at x +- h/2, x +- 3h/2, x +- 5h/2. */
int lsgo_diag(lsgo_grid *g, int family, const double *params, double *diag) {
    int d = g->d;
    double *v = calloc((size_t)g->n, sizeof(double));
    stencil_t s;
    int32_t J[MAXD], center[MAXD];
    int64_t *touched = malloc(sizeof(int64_t) * 15625 * 4);
    for (int64_t k = 0; k < g->n; ++k) diag[k] = 0.0;
    for (int t = 0; t < g->nD; ++t) {
        const int32_t *T = g->D + t * d;
        celllist *cl = get_cells(g, t);
        for (int64_t e = g->ex_off[t]; e < g->ex_off[t + 1]; ++e) {
            int64_t k = g->ex[e];
            if (!g->act[k]) continue;
            int pos[MAXD] = {0}, more;
            double w;
            int nt = 0;
            stencil_build(g, k, &s);
            do {
                more = stencil_next(g, &s, pos, J, &w);
                int64_t j = lsgo_lookup(g, J);
                if (j >= 0) { v[j] = w; touched[nt++] = j; }
            } while (more);
            double acc = 0.0;
            int npos = 1;
            for (int dd = 0; dd < d; ++dd) npos *= 6;
            for (int lin = 0; lin < npos; ++lin) {
                int r = lin, ok = 1;
                for (int dd = 0; dd < d; ++dd) {
                    static const int off[6] = {-5, -3, -1, 1, 3, 5};
                    int o = r % 6;
                    r /= 6;
                    int32_t i = g->pts[k * d + dd];
                    int tk = T[dd];
                    int64_t num = (int64_t)(2 * (i & ~(1 << tk)) + 1) * 2; /* x * 2^(tk+1) */
                    int64_t cnum = num + off[o];
                    if (cnum <= 0 || cnum >= ((int64_t)1 << (tk + 1))) { ok = 0; break; }
                    center[dd] = (int32_t)(((int64_t)1 << (tk + 1)) + (cnum - 1) / 2);
                }
                if (!ok) continue;
                int64_t c = find_cell(g, cl, center);
                if (c < 0) continue;
                const int64_t *corner = cl->corner + (c << d);
                double a = lsg_coef_eval(family, params, d, cl->xc + c * d);
                for (unsigned p = 0; p < (1u << d); ++p) {
                    int64_t kp = corner[p];
                    if (kp < 0 || v[kp] == 0.0) continue;
                    for (unsigned q = 0; q < (1u << d); ++q) {
                        int64_t kq = corner[q];
                        if (kq < 0 || v[kq] == 0.0) continue;
                        acc += v[kp] * a * lsg_q1_entry(g->form, d, cl->h, p, q) * v[kq];
                    }
                }
            }
            diag[k] = acc;
            for (int m = 0; m < nt; ++m) v[touched[m]] = 0.0;
        }
    }
    free(v);
    free(touched);
    return 0;
}

/* CG::solveHomogen (applications/cg_method.h:759-886) with its vector
 * semantics: ET assignments touch every entry, "h = r" and apply_inverse only
 * active entries, product() sums over every entry (extemp/vector.h:466-510). */
int lsgo_cg(lsgo_grid *g, int family, const double *params, const double *f, double *x, double eps,
            int maxit, int *iterations) {
    int64_t n = g->n;
    double *z = malloc(sizeof(double) * n), *r = calloc(n, sizeof(double)), *gg = calloc(n, sizeof(double));
    double *dv = calloc(n, sizeof(double)), *h = calloc(n, sizeof(double));
    lsgo_diag(g, family, params, z);
    lsgo_matvec(g, family, params, x, r);
    for (int64_t k = 0; k < n; ++k) r[k] = f[k] - r[k];
    for (int64_t k = 0; k < n; ++k) if (g->act[k]) h[k] = r[k] / z[k];
    for (int64_t k = 0; k < n; ++k) dv[k] = -1.0 * h[k];
    double delta = 0.0;
    for (int64_t k = 0; k < n; ++k) delta += r[k] * h[k];
    int it = 0;
    for (int i = 1; i <= maxit && delta > eps; ++i) {
        it = i;
        for (int64_t k = 0; k < n; ++k) if (g->act[k]) gg[k] = 0.0;
        lsgo_matvec(g, family, params, dv, gg);
        double dg = 0.0;
        for (int64_t k = 0; k < n; ++k) dg += dv[k] * gg[k];
        double tau = delta / dg;
        for (int64_t k = 0; k < n; ++k) r[k] = r[k] + tau * gg[k];
        for (int64_t k = 0; k < n; ++k) x[k] = x[k] - tau * dv[k];
        for (int64_t k = 0; k < n; ++k) h[k] = 1.0 * r[k];
        for (int64_t k = 0; k < n; ++k) if (g->act[k]) h[k] = h[k] / z[k];
        double dp = 0.0;
        for (int64_t k = 0; k < n; ++k) dp += r[k] * h[k];
        if (dp < eps * eps) break;
        double beta = dp / delta;
        delta = dp;
        for (int64_t k = 0; k < n; ++k) dv[k] = -1.0 * h[k] + beta * dv[k];
    }
    *iterations = it;
    free(z); free(r); free(gg); free(dv); free(h);
    return 0;
}

/* ------------------------------------------------------------ basis transforms
 * BasisTransformations/BasisTransformations.cpp.  Subgrids are visited in the
 * order of ListOfDepthOrderedSubgrids (sgrid/ListOfDepthOrderedGrids.cc:76-150):
 * |T|_1 ascending, first appearance within equal norms; hierarchization runs
 * the list backwards, dehierarchization forwards. */
static int *subgrid_order(const lsgo_grid *g) {
    int *o = (int *)malloc(sizeof(int) * (size_t)g->nD);
    int n = 0, maxl1 = 0;
    for (int t = 0; t < g->nD; ++t) {
        int l1 = 0;
        for (int k = 0; k < g->d; ++k) l1 += g->D[t * g->d + k];
        if (l1 > maxl1) maxl1 = l1;
    }
    for (int l = 0; l <= maxl1; ++l)
        for (int t = 0; t < g->nD; ++t) {
            int l1 = 0;
            for (int k = 0; k < g->d; ++k) l1 += g->D[t * g->d + k];
            if (l1 == l) o[n++] = t;
        }
    return o;
}

/* v = v -+ 0.5 (Links(v) + Rechts(v)) on the points of every subgrid T' (<= lim
 * when lim is given): CalcHierarchicalBasis (:13-38, :390-409, sign -1) and
 * CalcNodalBasis (:174-198, sign +1) */
static void hier_sweep(const lsgo_grid *g, const int *order, double *v, const int32_t *lim, int sign) {
    int d = g->d;
    for (int dd = 0; dd < d; ++dd) {
        for (int q = 0; q < g->nD; ++q) {
            int t = order[sign < 0 ? g->nD - 1 - q : q];
            const int32_t *T = g->D + t * d;
            if (T[dd] == 0 || (lim && !depth_le(T, lim, d))) continue;
            for (int64_t e = g->ex_off[t]; e < g->ex_off[t + 1]; ++e) {
                int64_t k = g->ex[e];
                if (!g->act[k]) continue;  /* expression assignments touch active entries */
                int64_t l = nbr(g, k, dd, 0), r = nbr(g, k, dd, 1);
                double s = 0.5 * ((l >= 0 ? v[l] : 0.0) + (r >= 0 ? v[r] : 0.0));
                v[k] = sign < 0 ? v[k] - s : v[k] + s;
            }
        }
    }
}

int lsgo_nodal_by_prew(lsgo_grid *g, const double *prew, double *u) {
    /* calcNodalByPrew (:670-706) with CalcHierbyPrew (:321-353) */
    int d = g->d;
    int *order = subgrid_order(g);
    double *hier = (double *)calloc((size_t)g->n, sizeof(double));
    double *hnew = (double *)malloc(sizeof(double) * (size_t)g->n);
    if (!order || !hier || !hnew) { free(order); free(hier); free(hnew); return -1; }
    stencil_t s;
    int32_t J[MAXD];
    for (int q = g->nD - 1; q >= 0; --q) {
        int t = order[q];
        const int32_t *T = g->D + t * d;
        memset(hnew, 0, sizeof(double) * (size_t)g->n);
        for (int64_t e = g->ex_off[t]; e < g->ex_off[t + 1]; ++e) {  /* every point of depth T */
            int64_t k = g->ex[e];
            double coeff = prew[k], w;
            int pos[MAXD] = {0}, more;
            stencil_build(g, k, &s);
            do {
                more = stencil_next(g, &s, pos, J, &w);
                int64_t j = lsgo_lookup(g, J);
                if (j >= 0) hnew[j] = hnew[j] + coeff * w;
            } while (more);
        }
        hier_sweep(g, order, hnew, T, -1);
        for (int64_t k = 0; k < g->n; ++k)
            if (depth_le(g->dep + k * d, T, d)) hier[k] = hier[k] + hnew[k];
    }
    for (int64_t k = 0; k < g->n; ++k) u[k] = g->act[k] ? hier[k] : 0.0;  /* u = 0.0; u = hier */
    hier_sweep(g, order, u, NULL, +1);
    free(order);
    free(hier);
    free(hnew);
    return 0;
}

void lsgo_set_form(lsgo_grid *g, int form) { g->form = form; }

/* ------------------------------------------------------------ boundary-data right-hand sides
 * MatrixVectorMultiplication/RHS.cpp and RHS.h:278-427.  The second grid ng
 * holds boundary points (a 1D index 0 or 1 in some dimension, depth 0 there). */

/* CalcHierarchicalBasisForRHS (RHS.cpp:6-41): per dimension, every boundary
 * point with depth > 0 in it loses half the sum of its two 1D parents; the
 * points are visited finest depth first, so a parent still holds the value of
 * the previous dimension's pass when its sons read it. */
int lsgo_hierarchize_boundary(lsgo_grid *ng, double *u) {
    int d = ng->d;
    for (int dd = 0; dd < d; ++dd)
        for (int t = ng->maxdep[dd]; t >= 1; --t)
            for (int64_t k = 0; k < ng->n; ++k) {
                const int32_t *I = ng->pts + k * d;
                int boundary = 0;
                for (int q = 0; q < d; ++q) boundary |= !interior1(I[q]);
                if (!boundary || ng->dep[k * d + dd] != t) continue;
                int64_t l = nbr(ng, k, dd, 0), r = nbr(ng, k, dd, 1);
                if (l < 0 || r < 0) return -1;  /* the reference needs both parents */
                u[k] = u[k] - 0.5 * (u[l] + u[r]);
            }
    return 0;
}

/* integral over [a,b] of (mp x + cp)(mq x + cq) by its antiderivative, and the
 * same with the weight (1 - x^2): RHS.cpp:47-54 and :285-300, evaluated in the
 * reference's order (the form loses digits to cancellation on fine levels). */
static double bd_int(double a, double b, double mp, double mq, double cp, double cq) {
    double t1 = (1.0 / 3.0 * b * b * b * mp * mq) - (1.0 / 3.0 * a * a * a * mp * mq);
    double t2 = (0.5 * b * b * mp * cq) - (0.5 * a * a * mp * cq);
    double t3 = (0.5 * b * b * mq * cp) - (0.5 * a * a * mq * cp);
    double t4 = (b - a) * cp * cq;
    return t1 + t2 + t3 + t4;
}
static double bd_int_w(double a, double b, double mp, double mq, double cp, double cq) {
    double r1 = bd_int(a, b, mp, mq, cp, cq);
    double t1 = (1.0 / 5.0 * b * b * b * b * b * mp * mq) - (1.0 / 5.0 * a * a * a * a * a * mp * mq);
    double t2 = (0.25 * b * b * b * b * mp * cq) - (0.25 * a * a * a * a * mp * cq);
    double t3 = (0.25 * b * b * b * b * mq * cp) - (0.25 * a * a * a * a * mq * cp);
    double t4 = (1.0 / 3.0 * b * b * b * cp * cq) - (1.0 / 3.0 * a * a * a * cp * cq);
    double r2 = t1 + t2 + t3 + t4;
    return r1 - r2;
}

/* One dimension of CalcIntegral / CalcIntegral_mass / CalcIntegral_coeff
 * (RHS.cpp:56-283, :314-503, :505-695): the hat of p (1D index ip, width 2^-tp)
 * against the hat of q (1D index iq, width 2^-tq, only its half inside [0,1]
 * at a boundary index), summed over the four pairs of linear pieces in the
 * order left-left, left-right, right-left, right-right.  kind 0: product of
 * the functions, 1: of their derivatives, 2: of the functions weighted by
 * (1 - x^2). */
static double bd_factor(int32_t ip, int tp, int32_t iq, int tq, int kind) {
    double mpl = (double)(1u << tp), mql = (double)(1u << tq);
    double hp = 1.0 / mpl, hq = 1.0 / mql, xp = coord1(ip), xq = coord1(iq);
    double mp[2] = {mpl, -1.0 * mpl}, mq[2] = {mql, -1.0 * mql};
    double cp[2] = {-(xp - hp) / hp, +(xp + hp) / hp}, cq[2] = {-(xq - hq) / hq, +(xq + hq) / hq};
    double lp[2] = {xp - hp, xp}, rp[2] = {xp, xp + hp}, lq[2] = {xq - hq, xq}, rq[2] = {xq, xq + hq};
    double s = 0.0;
    for (int sp = 0; sp < 2; ++sp)
        for (int sq = 0; sq < 2; ++sq) {
            double v = 0.0;
            int skip = (iq == 0 && sq == 0) || (iq == 1 && sq == 1);
            if (!skip && !(rp[sp] < lq[sq]) && !(rq[sq] < lp[sp])) {
                double a = lq[sq] > lp[sp] ? lq[sq] : lp[sp];
                double b = rp[sp] < rq[sq] ? rp[sp] : rq[sq];
                if (kind == 1) v = (b - a) * mp[sp] * mq[sq];
                else if (kind == 0) v = bd_int(a, b, mp[sp], mq[sq], cp[sp], cq[sq]);
                else v = bd_int_w(a, b, mp[sp], mq[sq], cp[sp], cq[sq]);
            }
            s = s + v;  /* ll + lr + rl + rr, left to right */
        }
    return s;
}

/* InHomoBoundaryRHSHierarchical::multiply / multiply_mass / multiply_mass_coeff
 * (RHS.cpp:697-1008): for every depth T of g, nodal values at the points of
 * depth <= T, sum over the boundary points b of ng of I(p at level T, b) hier[b]
 * (depth-list order of ng, storage order within a depth), then
 * ConvertToPrewavelet2 at the active points of depth T (RHS.h:397-420). */
int lsgo_boundary_rhs(lsgo_grid *g, lsgo_grid *ng, int kind, const double *hier, double *y) {
    int d = g->d;
    if (ng->d != d || kind < 0 || kind > 2) return -1;
    double *nodal = (double *)malloc(sizeof(double) * (size_t)g->n);
    if (!nodal) return -1;
    for (int t = 0; t < g->nD; ++t) {
        const int32_t *T = g->D + t * d;
        for (int64_t k = 0; k < g->n; ++k) {
            nodal[k] = 0.0;
            if (!depth_le(g->dep + k * d, T, d)) continue;
            const int32_t *P = g->pts + k * d;
            double sum = 0.0;
            for (int u = 0; u < ng->nD; ++u) {
                const int32_t *TH = ng->D + u * d;
                int boundary = 0;
                for (int q = 0; q < d; ++q) boundary |= TH[q] == 0;
                if (!boundary) continue;
                for (int64_t e = ng->ex_off[u]; e < ng->ex_off[u + 1]; ++e) {
                    int64_t b = ng->ex[e];
                    const int32_t *Q = ng->pts + b * d;
                    double val;
                    if (kind == 0) {  /* CalcIntegral: sum over the derivative dimension */
                        val = 0.0;
                        for (int o = 0; o < d; ++o) {
                            double prod = 1.0;
                            for (int q = 0; q < d; ++q) prod *= bd_factor(P[q], T[q], Q[q], TH[q], q == o ? 1 : 0);
                            val += prod;
                        }
                    } else {
                        val = 1.0;
                        for (int q = 0; q < d; ++q) val *= bd_factor(P[q], T[q], Q[q], TH[q], kind == 1 ? 0 : 2);
                    }
                    sum += val * hier[b];
                }
            }
            nodal[k] = sum;
        }
        convert_prew(g, t, nodal, y);
    }
    free(nodal);
    return 0;
}

/* CalcHierarchicalBasis(u) (BasisTransformations.cpp:390-409) and
 * CalcNodalBasis(u) (:174-198) over the whole grid: active points only, an
 * absent neighbour reads 0; grids with boundary points included. */
int lsgo_hierarchize(lsgo_grid *g, double *u, int sign) {
    int *order = subgrid_order(g);
    if (!order) return -1;
    hier_sweep(g, order, u, NULL, sign < 0 ? -1 : +1);
    free(order);
    return 0;
}
