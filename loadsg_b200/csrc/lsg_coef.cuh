// Diffusion-coefficient families evaluated on the device at cell midpoints.
// Same formulas and parameter layouts as include/lsg.h (LSG_COEF_*).
#pragma once

#define LSG_MAX_COEF_PARAMS 256

__device__ __forceinline__ double lsg_coef_eval_dev(int family, const double* p, int d, const double* x) {
    const double PI = 3.14159265358979323846;
    switch (family) {
    case 0:
        return p[0];
    case 1: {
        double prod = 1.0;
        for (int i = 0; i < d; ++i) prod *= sin(PI * p[2 + i] * x[i]);
        return p[0] + p[1] * prod;
    }
    case 2: {
        double s = 0.0;
        for (int k = 1; k <= d; ++k) s += p[k - 1] * sin((double)k * PI * x[k - 1]);
        return exp(s);
    }
    case 3: {
        int J = (int)p[0];
        double s = 0.0;
        for (int j = 0; j < J; ++j) {
            double prod = 1.0;
            for (int i = 0; i < d; ++i) prod *= sin(PI * p[1 + J + j * d + i] * x[i]);
            s += p[1 + j] * prod;
        }
        return exp(s);
    }
    case 4:
        return p[0] + p[1] * sin(2.0 * PI * x[0]) * cos(2.0 * PI * x[1]);
    default:
        return 0.0;
    }
}
