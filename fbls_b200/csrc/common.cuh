// Shared constants and scalar helpers of the FBLS search path (sm_100a).
//
// Every kernel translation unit is compiled with --fmad=false: the bin index
// floor(t * scale), the template width floor(D * scale + 0.5) and the f32
// pre-ranking merit must round each multiply and add separately, as the
// reference's arithmetic does (src/search/kernels.rs:314-327, :679, :400-402).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fbls {

constexpr int TILE = 128;        // phase lanes per scan tile (kernels.rs:26)
constexpr int NF = 3;            // folded fields v, w, count (kernels.rs:28-31)
constexpr int F_V = 0, F_W = 1, F_N = 2;
constexpr int PART_STRIDE = 9;   // kernels.rs:38
constexpr int RECORD_STRIDE = 9; // kernels.rs:39
constexpr int EV_TILE = 64;      // evidence.rs:29
constexpr int EV_PART = 15;      // evidence.rs:30
constexpr int NORB = 3;          // evidence.rs:31
constexpr int NPARAM = 30;       // evidence.rs:32
constexpr uint64_t KEY_MAX = ~0ull;

__host__ __device__ inline double neg_inf() { return -__builtin_huge_val(); }

// Rust f64::max / f64::min semantics (a NaN operand loses).
__host__ __device__ inline double rmax(double a, double b) {
    return a != a ? b : (b != b ? a : (a > b ? a : b));
}
__host__ __device__ inline double rmin(double a, double b) {
    return a != a ? b : (b != b ? a : (a < b ? a : b));
}
__host__ __device__ inline float rmaxf(float a, float b) {
    return a != a ? b : (b != b ? a : (a > b ? a : b));
}

// Rust `f64 as usize` for the non-negative finite values the path produces
// (saturating at 0 for negatives and NaN).
__host__ __device__ inline uint64_t as_u64(double x) {
    return x > 0.0 ? (uint64_t)x : 0ull;
}

// Template width in bins: max(1, floor(D * scale + 0.5)) (kernels.rs:679).
__host__ __device__ inline uint32_t template_width(double duration, double scale) {
    uint64_t k = as_u64(floor(duration * scale + 0.5));
    return k < 1 ? 1u : (uint32_t)k;
}

// Layer width of a staircase: max(1, floor(k * factor + 0.5)) (kernels.rs:105).
__host__ __device__ inline uint32_t layer_width(uint32_t k, double factor) {
    uint64_t w = as_u64(floor((double)k * factor + 0.5));
    return w < 1 ? 1u : (uint32_t)w;
}

// Complementary error function by W. J. Cody's rational Chebyshev
// approximations ("Rational Chebyshev approximations for the error
// function", Math. Comp. 23 (1969) 631-637), with the coefficient set and
// evaluation order the reference uses (src/search/math.rs:8-100). exp() is
// the platform's.
__host__ __device__ inline double cody_erfc(double x) {
    const double A0 = 3.16112374387056560e0, A1 = 1.13864154151050156e2, A2 = 3.77485237685302021e2,
                 A3 = 3.20937758913846947e3, A4 = 1.85777706184603153e-1;
    const double B0 = 2.36012909523441209e1, B1 = 2.44024637934444173e2, B2 = 1.28261652607737228e3,
                 B3 = 2.84423683343917062e3;
    const double C[9] = {5.64188496988670089e-1, 8.88314979438837594e0, 6.61191906371416295e1,
                         2.98635138197400131e2,  8.81952221241769090e2, 1.71204761263407058e3,
                         2.05107837782607147e3,  1.23033935479799725e3, 2.15311535474403846e-8};
    const double D[8] = {1.57449261107098347e1, 1.17693950891312499e2, 5.37181101862009858e2,
                         1.62138957456669019e3, 3.29079923573345963e3, 4.36261909014324716e3,
                         3.43936767414372164e3, 1.23033935480374942e3};
    const double P[6] = {3.05326634961232344e-1, 3.60344899949804439e-1, 1.25781726111229246e-1,
                         1.60837851487422766e-2, 6.58749161529837803e-4, 1.63153871373020978e-2};
    const double Q[5] = {2.56852019228982242e0, 1.87295284992346725e0, 5.27905102951428412e-1,
                         6.05183413124413191e-2, 2.33520497626869185e-3};
    const double SQRPI = 5.6418958354775628695e-1;
    double y = fabs(x);
    double result;
    if (y <= 0.46875) {
        double ysq = y > 1.11e-16 ? y * y : 0.0;
        double xnum = A4 * ysq, xden = ysq;
        xnum = (xnum + A0) * ysq;
        xden = (xden + B0) * ysq;
        xnum = (xnum + A1) * ysq;
        xden = (xden + B1) * ysq;
        xnum = (xnum + A2) * ysq;
        xden = (xden + B2) * ysq;
        return 1.0 - x * (xnum + A3) / (xden + B3);
    } else if (y <= 4.0) {
        double xnum = C[8] * y, xden = y;
        for (int i = 0; i < 7; i++) {
            xnum = (xnum + C[i]) * y;
            xden = (xden + D[i]) * y;
        }
        double r = (xnum + C[7]) / (xden + D[7]);
        double ysq = trunc(y * 16.0) / 16.0;
        double del = (y - ysq) * (y + ysq);
        result = exp(-ysq * ysq) * exp(-del) * r;
    } else if (y < 26.543) {
        double ysq = 1.0 / (y * y);
        double xnum = P[5] * ysq, xden = ysq;
        for (int i = 0; i < 4; i++) {
            xnum = (xnum + P[i]) * ysq;
            xden = (xden + Q[i]) * ysq;
        }
        double r = ysq * (xnum + P[4]) / (xden + Q[4]);
        r = (SQRPI - r) / y;
        double ysq2 = trunc(y * 16.0) / 16.0;
        double del = (y - ysq2) * (y + ysq2);
        result = exp(-ysq2 * ysq2) * exp(-del) * r;
    } else {
        result = 0.0;
    }
    return x < 0.0 ? 2.0 - result : result;
}

// log(exp(x) + exp(y)) (math.rs:103-110).
__host__ __device__ inline double log_add(double x, double y) {
    double high = rmax(x, y);
    if (high == neg_inf()) return high;
    return high + log(1.0 + exp(rmin(x, y) - high));
}

// Log evidence of a positive amplitude with a half-normal prior of scale tau
// (math.rs:115-140): log of the Gaussian integral of the likelihood ratio
// over depth >= 0, with the asymptotic expansion of erfc below z = -26.
__host__ __device__ inline double positive_amplitude_evidence(double a, double q, double tau) {
    q = rmax(q, 0.0);
    double precision = 1.0 + tau * tau * q;
    double z = tau * a / sqrt(precision);
    if (z < -26.0) {
        double zz = rmax(z * z, 1.0);
        double inverse = 1.0 / zz;
        double series =
            1.0 + inverse * (-1.0 + inverse * (3.0 + inverse * (-15.0 + inverse * (105.0 + inverse * (-945.0 + inverse * (10395.0 - inverse * 135135.0))))));
        return -0.5 * log(precision) - log(rmax(-z, 1.0)) - 0.22579135264472743236 + log(series);
    }
    return -0.5 * log(precision) + 0.5 * z * z + log(rmax(cody_erfc(-z * 0.70710678118654752440), 1e-300));
}

// Upper bound of the log evidence over positive mixtures of two templates
// (math.rs:145-177).
__host__ __device__ inline double subspace_upper(double a, double b, double q, double r, double cross, double rho2) {
    double product = q * r;
    double det = q * r - cross * cross;
    double energy = (a * a * r + b * b * q - 2.0 * a * b * cross) / rmax(det * rho2, 1e-300);
    bool safe = q > 0.0 && r > 0.0 && det > 1e-8 * product;
    double pa = rmax(a, 0.0), pb = rmax(b, 0.0);
    double boundary = 0.5 * rmax(pa * pa / rmax(q * rho2, 1e-300), pb * pb / rmax(r * rho2, 1e-300));
    bool interior = a * r - b * cross > 0.0 && b * q - a * cross > 0.0;
    double upper = safe ? (interior ? 0.5 * rmax(energy, 0.0) : boundary) : __builtin_huge_val();
    bool only_a = r == 0.0 && b == 0.0 && cross == 0.0;
    bool only_b = q == 0.0 && a == 0.0 && cross == 0.0;
    if (only_a && q > 0.0) upper = 0.5 * a * a / (q * rho2);
    if (only_b && r > 0.0) upper = 0.5 * b * b / (r * rho2);
    if (only_a && only_b) upper = 0.0;
    if (a <= 0.0 && b <= 0.0) upper = 0.0;
    return upper * 1.000001 + 1e-6;
}

}  // namespace fbls
