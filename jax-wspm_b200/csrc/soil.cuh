// Soil constitutive laws evaluated per node in FP64.
//
// van Genuchten-Mualem: src/models/van_genuchten.py:24-47 (branch on h < 0).
// Gardner exponential:  src/models/exponential.py:24-41 (branch on h <= 0).
// The operation order of the reference's jnp expressions is kept so results
// agree with the oracle to a few ulps.
#pragma once
#include "common.cuh"

namespace wspm {

struct SoilParams {
    int model;        // WSPM_SOIL_*
    double p[6];      // VG: alpha, thS, thR, n, m, Ks ; EXP: alpha0, thS, thR, Ks
};

__device__ __forceinline__ void soil_eval(const SoilParams &sp, double h,
                                          double &C, double &K, double &theta) {
    if (sp.model == WSPM_SOIL_VAN_GENUCHTEN) {
        const double alpha = sp.p[0], thS = sp.p[1], thR = sp.p[2], n = sp.p[3], m = sp.p[4], Ks = sp.p[5];
        if (h < 0.0) {
            // (a|h|)^(n-1) by pow (exact enough down to |h| ~ 1e-300, where exp(x log a|h|) loses ~|x| ulps),
            // (a|h|)^n by one multiply, (1 + (a|h|)^n)^-m through log1p/exp and (1 + (a|h|)^n)^(-m-1) by one
            // division (the reference evaluates six pow() calls)
            const double ah = alpha * fabs(h);
            const double ahn1 = pow(ah, n - 1.0);
            const double ahn = ahn1 * ah;
            const double onep = 1.0 + ahn;
            const double tm = exp(-m * log1p(ahn));
            theta = (thS - thR) * tm + thR;
            const double Se = (theta - thR) / (thS - thR);
            const double t = 1.0 - pow(1.0 - pow(Se, 1.0 / m), m);
            K = Ks * (sqrt(Se) * (t * t));
            C = (thS - thR) * alpha * m * n * ahn1 * (tm / onep);
        } else {
            theta = thS;
            K = Ks;
            C = 0.0;
        }
    } else {
        const double a0 = sp.p[0], thS = sp.p[1], thR = sp.p[2], Ks = sp.p[3];
        if (h <= 0.0) {
            const double e = exp(a0 * h);
            theta = (thS - thR) * e + thR;
            K = Ks * e;
            C = a0 * (thS - thR) * e;
        } else {
            theta = thS;
            K = Ks;
            C = 0.0;
        }
    }
}

}  // namespace wspm
