/*
 * Diffusion-coefficient families shared by the oracle (C restatement) and the
 * reference harness.  TEST INFRASTRUCTURE ONLY: the product evaluates the same
 * formulas in its own CUDA code (loadsg_b200/csrc/coefficient.cuh); parity
 * tests compare the two.
 *
 * The operator is -div(a grad u) with the coefficient sampled at each cell's
 * midpoint ("midpoint rule"):  the local stiffness entry of corners p,q of a
 * cell c is  a(x_c) * sum_i prod_j k_ij(p,q)  with the exact Q1 factors
 *   i==j : +1/h_j (same side) or -1/h_j (opposite sides)
 *   i!=j : h_j/3  (same side) or  h_j/6 (opposite sides).
 * This is what the reference's StencilTemplate::integration plugin
 * (library/source/stencils/Stencil.h:740) returns for a test-side subclass;
 * with a == 1 it equals Poisson::integration (Stencil.h:1713-1764).
 */
#ifndef LSG_ORACLE_COEFFICIENT_H
#define LSG_ORACLE_COEFFICIENT_H

#include <math.h>

#define LSG_COEF_CONST 0     /* a = p[0]                                              */
#define LSG_COEF_SINPROD 1   /* a = p[0] + p[1] * prod_i sin(pi p[2+i] x_i)          */
#define LSG_COEF_EXPSIN 2    /* a = exp(sum_{k=1..d} p[k-1] sin(k pi x_{k-1}))       */
#define LSG_COEF_LOGNORMAL 3 /* a = exp(sum_j p[1+j] prod_i sin(pi p[1+J+j*d+i] x_i)),
                                J = (int)p[0]                                        */
#define LSG_COEF_SIN2PI 4    /* a = p[0] + p[1] sin(2 pi x_0) cos(2 pi x_1)          */
#define LSG_COEF_MAXPARAM 256

static inline double lsg_coef_eval(int family, const double *p, int d, const double *x) {
    const double PI = 3.14159265358979323846;
    switch (family) {
    case LSG_COEF_CONST:
        return p[0];
    case LSG_COEF_SINPROD: {
        double prod = 1.0;
        for (int i = 0; i < d; ++i) prod *= sin(PI * p[2 + i] * x[i]);
        return p[0] + p[1] * prod;
    }
    case LSG_COEF_EXPSIN: {
        double s = 0.0;
        for (int k = 1; k <= d; ++k) s += p[k - 1] * sin((double)k * PI * x[k - 1]);
        return exp(s);
    }
    case LSG_COEF_LOGNORMAL: {
        int J = (int)p[0];
        double s = 0.0;
        for (int j = 0; j < J; ++j) {
            double prod = 1.0;
            for (int i = 0; i < d; ++i) prod *= sin(PI * p[1 + J + j * d + i] * x[i]);
            s += p[1 + j] * prod;
        }
        return exp(s);
    }
    case LSG_COEF_SIN2PI:
        return p[0] + p[1] * sin(2.0 * PI * x[0]) * cos(2.0 * PI * x[1]);
    default:
        return NAN;
    }
}

/* Exact Q1 stiffness entry (constant coefficient 1) of a cell with widths h[],
 * for corners p and q given as bit masks (bit j set = right side in dim j). */
static inline double lsg_q1_stiffness(int d, const double *h, unsigned p, unsigned q) {
    double sum = 0.0;
    for (int i = 0; i < d; ++i) {
        double prod = 1.0;
        for (int j = 0; j < d; ++j) {
            int same = ((p >> j) & 1u) == ((q >> j) & 1u);
            if (i == j) prod *= same ? 1.0 / h[j] : -1.0 / h[j];
            else prod *= same ? h[j] / 3.0 : h[j] / 6.0;
        }
        sum += prod;
    }
    return sum;
}

/* Exact Q1 mass entry (coefficient 1): prod_j (same side ? h_j/3 : h_j/6), the
 * value HelmHoltz::integration returns (stencils/Stencil.h:900-919 with
 * integral_RR = h^3/3, integral_LR = h^3/6, times exponent^2 = 1/h^2). */
static inline double lsg_q1_mass(int d, const double *h, unsigned p, unsigned q) {
    double prod = 1.0;
    for (int j = 0; j < d; ++j) prod *= (((p >> j) & 1u) == ((q >> j) & 1u)) ? h[j] / 3.0 : h[j] / 6.0;
    return prod;
}

/* form 0: stiffness (diffusion), 1: mass */
static inline double lsg_q1_entry(int form, int d, const double *h, unsigned p, unsigned q) {
    return form == 1 ? lsg_q1_mass(d, h, p, q) : lsg_q1_stiffness(d, h, p, q);
}

#endif
