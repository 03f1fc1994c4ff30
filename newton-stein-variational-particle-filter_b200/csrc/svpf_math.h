// svpf_math.h -- scalar helpers shared by device and host code (plain C++
// when compiled without nvcc, so they can be exercised on the CPU too).
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define SVPF_HD __host__ __device__
#else
#define SVPF_HD
#endif

namespace svpf {

// psi(x), the digamma function, for the nu-derivative of the Student-t
// normaliser lgamma((nu+1)/2) - lgamma(nu/2) - log(nu pi)/2.
// Recurrence psi(x) = psi(x+1) - 1/x until x >= 8, then the asymptotic series
// of Abramowitz & Stegun 6.3.18.  Any finite x > 0 reaches 8 within eight
// shifts, and the loop is capped at eight, so no input keeps it running:
// x <= 0, -inf and NaN return NaN, +inf returns +inf.
SVPF_HD inline double digamma_bounded(double x) {
    if (!(x > 0.0)) return NAN;
    double acc = 0.0;
    for (int k = 0; k < 8 && x < 8.0; ++k) {
        acc -= 1.0 / x;
        x += 1.0;
    }
    const double r = 1.0 / x, r2 = r * r;
    return acc + log(x) - 0.5 * r -
           r2 * (1.0 / 12 - r2 * (1.0 / 120 - r2 * (1.0 / 252 - r2 * (1.0 / 240 - r2 * (1.0 / 132)))));
}

// Model parameters a filter can run with: every component finite, nu > 0,
// sigma_z > 0 and |rho| < 1 (the stationary law of the AR(1) needs it).
// Comparisons are written so that NaN fails every one of them.
SVPF_HD inline bool theta_ok(float mu, float rho, float sigma_z, float nu) {
    const float inf = INFINITY;
    return (mu > -inf && mu < inf) && (rho > -1.0f && rho < 1.0f) && (sigma_z > 0.0f && sigma_z < inf) &&
           (nu > 0.0f && nu < inf);
}

}  // namespace svpf
