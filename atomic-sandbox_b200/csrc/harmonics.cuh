// harmonics.cuh -- real regular solid harmonics R_lm(r), l <= 6, Racah normalisation, in f64:
// the recursion on the complex C_l^m of crates/qm/src/poisson.rs:89-120 (diagonal ladder without
// the Condon-Shortley sign, three-term recursion in l at fixed m), written to out[l*l + l + m].
#pragma once
#include <cuda_runtime.h>

namespace ks {

__device__ __forceinline__ void solid_harmonics_dev(double x, double y, double z, double* out) {
    double cr[7][7], ci[7][7];
    double r2 = x * x + y * y + z * z;
    cr[0][0] = 1.0;
    ci[0][0] = 0.0;
#pragma unroll
    for (int l = 1; l <= 6; ++l) {
        double lf = l;
        double f = sqrt((2.0 * lf - 1.0) / (2.0 * lf));
        double pr = cr[l - 1][l - 1], pi = ci[l - 1][l - 1];
        cr[l][l] = f * (x * pr - y * pi);
        ci[l][l] = f * (x * pi + y * pr);
#pragma unroll
        for (int m = 0; m < l; ++m) {
            double mf = m;
            double a = (2.0 * lf - 1.0) * z;
            double r1 = cr[l - 1][m], i1 = ci[l - 1][m];
            double r0 = 0.0, i0 = 0.0;
            if (l >= 2 && m <= l - 2) { r0 = cr[l - 2][m]; i0 = ci[l - 2][m]; }
            double b = sqrt(fmax((lf - 1.0) * (lf - 1.0) - mf * mf, 0.0)) * r2;
            double d = sqrt(lf * lf - mf * mf);
            cr[l][m] = (a * r1 - b * r0) / d;
            ci[l][m] = (a * i1 - b * i0) / d;
        }
    }
    const double s2 = 1.4142135623730951;
#pragma unroll
    for (int l = 0; l <= 6; ++l) {
        out[l * l + l] = cr[l][0];
#pragma unroll
        for (int m = 1; m <= l; ++m) {
            out[l * l + l + m] = s2 * cr[l][m];
            out[l * l + l - m] = s2 * ci[l][m];
        }
    }
}


}  // namespace ks
