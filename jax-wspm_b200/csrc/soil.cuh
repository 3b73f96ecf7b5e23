// Soil constitutive laws evaluated per node in FP64.
//
// van Genuchten-Mualem: src/models/van_genuchten.py:24-47 (branch on h < 0).
// Gardner exponential:  src/models/exponential.py:24-41 (branch on h <= 0).
// theta and C follow the reference's expressions; K is the same function
// evaluated without the reference's cancellation (agrees with it to the
// conditioning of its form).
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
        if (h < 0.0 && n == 2.0 && m == 0.5) {
            // n = 2, m = 1/2 (the Mualem pair for n = 2): every power is a square or a square root.
            //   a = (alpha|h|)^2, Se = (1 + a)^-1/2, (a/(1+a))^1/2 = alpha|h| Se,
            //   1 - (a/(1+a))^1/2 = Se^2 / (1 + alpha|h| Se)   (no cancellation at large a)
            const double ah = alpha * fabs(h);
            const double onep = 1.0 + ah * ah;
            const double tm = 1.0 / sqrt(onep);
            theta = (thS - thR) * tm + thR;
            const double t = (tm * tm) / (1.0 + ah * tm);
            K = Ks * (sqrt(tm) * (t * t));
            C = (thS - thR) * alpha * m * n * ah * (tm / onep);
        } else if (h < 0.0) {
            // Same functions as the reference, with its six pow() calls reduced algebraically:
            //   a = (alpha|h|)^n, Se = (1 + a)^-m, Se^(1/m) = 1/(1 + a), 1 - Se^(1/m) = a/(1 + a)
            //   K = Ks sqrt(Se) (1 - (a/(1+a))^m)^2,  (a/(1+a))^m = exp(m log(a/(1+a)))
            // log(a/(1+a)) is -log1p(1/a) for a >= 1 and log(a/(1+a)) below, and 1 - exp(.) is -expm1(.), so
            // neither end of the curve loses digits to cancellation (the reference's form does, at both ends).
            // (alpha|h|)^(n-1) stays a pow: exp((n-1) log(alpha|h|)) loses ~|log| ulps at |h| ~ 1e-300.
            const double ah = alpha * fabs(h);
            const double ahn1 = pow(ah, n - 1.0);
            const double ahn = ahn1 * ah;
            const double onep = 1.0 + ahn;
            const double tm = exp(-m * log1p(ahn));
            theta = (thS - thR) * tm + thR;
            const double log1mu = ahn >= 1.0 ? -log1p(1.0 / ahn) : log(ahn / onep);
            const double t = -expm1(m * log1mu);
            K = Ks * (sqrt(tm) * (t * t));
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
