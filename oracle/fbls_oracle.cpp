// FBLS search hot path: CPU oracle.
//
// TEST INFRASTRUCTURE ONLY. This file restates, on the CPU and in plain C++,
// the arithmetic of the reference's search path so that the CUDA path in
// fbls_b200/ can be checked against it. Only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline leg may load it. The product never calls it.
//
// Parity status: the reference (isakruas/fbls, Rust + cuda-oxide) cannot be
// built here (no cargo/rustc, cuda-rust git dependencies not vendored), so
// there is no oracle/_ref. This restatement is pinned by every known-answer
// test the reference holds for the path:
//   * erfc table            src/search/math.rs:183-210 (16 values, 1e-14 rel.)
//   * period grid property  src/search/grid.rs:34-42
//   * noise model           src/prep/curve.rs:636-661
//   * transit mask count    src/prep/curve.rs:663-673
// The fold / prefix / tile-scan / evidence outputs have no golden vectors in
// the reference; they are pinned here only through brute-force identities
// (direct per-observation box sums) and injected-signal recovery, i.e. the
// scan and evidence outputs are "parity unpinned" against reference output.
//
// Arithmetic order follows the reference expression by expression; compile
// with -ffp-contract=off so no multiply-add is fused. The only freedom taken
// is the order of the fold's additions, which the reference leaves to
// unordered f64 atomics (src/search/kernels.rs:491, :540); here they run in
// observation order, and prefix sums run sequentially.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace {

constexpr double NEG_INF = -std::numeric_limits<double>::infinity();
constexpr uint64_t KEY_MAX = std::numeric_limits<uint64_t>::max();
constexpr int TILE = 128;  // src/search/kernels.rs:26
constexpr int NF = 3;      // fields v, w, 1 (kernels.rs:28-31)
constexpr int F_V = 0, F_W = 1, F_N = 2;

// Rust f64::max / f32::max: NaN loses to a number.
inline double rmax(double a, double b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a > b ? a : b)); }
inline double rmin(double a, double b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a < b ? a : b)); }
inline float rmaxf(float a, float b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a > b ? a : b)); }

// Rust `f64 as usize` / `as i64`: truncation with saturation, NaN -> 0.
inline uint64_t as_usize(double x) {
    if (!(x > 0.0)) return 0;
    if (x >= 18446744073709551615.0) return UINT64_MAX;
    return (uint64_t)x;
}
inline int64_t as_i64(double x) {
    if (std::isnan(x)) return 0;
    if (x >= 9223372036854775807.0) return INT64_MAX;
    if (x <= -9223372036854775808.0) return INT64_MIN;
    return (int64_t)x;
}

}  // namespace

// ---------------------------------------------------------------------------
// Scalar math, src/search/math.rs:8-177
// ---------------------------------------------------------------------------

extern "C" double orc_erfc(double x) {
    // Cody's rational Chebyshev approximations (W. J. Cody, Math. Comp. 23
    // (1969) 631-637) with the coefficient set of math.rs:9-58.
    static const double A[5] = {3.16112374387056560e0, 1.13864154151050156e2, 3.77485237685302021e2,
                                3.20937758913846947e3, 1.85777706184603153e-1};
    static const double B[4] = {2.36012909523441209e1, 2.44024637934444173e2, 1.28261652607737228e3,
                                2.84423683343917062e3};
    static const double C[9] = {5.64188496988670089e-1, 8.88314979438837594e0, 6.61191906371416295e1,
                                2.98635138197400131e2,  8.81952221241769090e2, 1.71204761263407058e3,
                                2.05107837782607147e3,  1.23033935479799725e3, 2.15311535474403846e-8};
    static const double D[8] = {1.57449261107098347e1, 1.17693950891312499e2, 5.37181101862009858e2,
                                1.62138957456669019e3, 3.29079923573345963e3, 4.36261909014324716e3,
                                3.43936767414372164e3, 1.23033935480374942e3};
    static const double P[6] = {3.05326634961232344e-1, 3.60344899949804439e-1, 1.25781726111229246e-1,
                                1.60837851487422766e-2, 6.58749161529837803e-4, 1.63153871373020978e-2};
    static const double Q[5] = {2.56852019228982242e0, 1.87295284992346725e0, 5.27905102951428412e-1,
                                6.05183413124413191e-2, 2.33520497626869185e-3};
    const double SQRPI = 5.6418958354775628695e-1;
    const double THRESH = 0.46875;
    const double XBIG = 26.543;
    double y = std::fabs(x);
    double result;
    if (y <= THRESH) {
        double ysq = y > 1.11e-16 ? y * y : 0.0;
        double xnum = A[4] * ysq;
        double xden = ysq;
        for (int i = 0; i < 3; i++) {
            xnum = (xnum + A[i]) * ysq;
            xden = (xden + B[i]) * ysq;
        }
        return 1.0 - x * (xnum + A[3]) / (xden + B[3]);
    } else if (y <= 4.0) {
        double xnum = C[8] * y;
        double xden = y;
        for (int i = 0; i < 7; i++) {
            xnum = (xnum + C[i]) * y;
            xden = (xden + D[i]) * y;
        }
        double r = (xnum + C[7]) / (xden + D[7]);
        double ysq = std::trunc(y * 16.0) / 16.0;
        double del = (y - ysq) * (y + ysq);
        result = std::exp(-ysq * ysq) * std::exp(-del) * r;
    } else if (y < XBIG) {
        double ysq = 1.0 / (y * y);
        double xnum = P[5] * ysq;
        double xden = ysq;
        for (int i = 0; i < 4; i++) {
            xnum = (xnum + P[i]) * ysq;
            xden = (xden + Q[i]) * ysq;
        }
        double r = ysq * (xnum + P[4]) / (xden + Q[4]);
        r = (SQRPI - r) / y;
        double ysq2 = std::trunc(y * 16.0) / 16.0;
        double del = (y - ysq2) * (y + ysq2);
        result = std::exp(-ysq2 * ysq2) * std::exp(-del) * r;
    } else {
        result = 0.0;
    }
    return x < 0.0 ? 2.0 - result : result;
}

extern "C" double orc_log_add(double x, double y) {
    double high = rmax(x, y);
    if (high == NEG_INF) return high;
    return high + std::log(1.0 + std::exp(rmin(x, y) - high));
}

extern "C" double orc_positive_amplitude_evidence(double a, double q, double tau) {
    q = rmax(q, 0.0);
    double precision = 1.0 + tau * tau * q;
    double z = tau * a / std::sqrt(precision);
    if (z < -26.0) {
        double zz = rmax(z * z, 1.0);
        double inverse = 1.0 / zz;
        double series =
            1.0 + inverse * (-1.0 + inverse * (3.0 + inverse * (-15.0 + inverse * (105.0 + inverse * (-945.0 + inverse * (10395.0 - inverse * 135135.0))))));
        return -0.5 * std::log(precision) - std::log(rmax(-z, 1.0)) - 0.22579135264472743236 + std::log(series);
    }
    return -0.5 * std::log(precision) + 0.5 * z * z +
           std::log(rmax(orc_erfc(-z * 0.70710678118654752440), 1e-300));
}

extern "C" double orc_subspace_upper(double a, double b, double q, double r, double cross, double rho2) {
    double product = q * r;
    double det = q * r - cross * cross;
    double energy = (a * a * r + b * b * q - 2.0 * a * b * cross) / rmax(det * rho2, 1e-300);
    bool safe = q > 0.0 && r > 0.0 && det > 1e-8 * product;
    double pa = rmax(a, 0.0), pb = rmax(b, 0.0);
    double boundary = 0.5 * rmax(pa * pa / rmax(q * rho2, 1e-300), pb * pb / rmax(r * rho2, 1e-300));
    bool interior = a * r - b * cross > 0.0 && b * q - a * cross > 0.0;
    double upper = safe ? (interior ? 0.5 * rmax(energy, 0.0) : boundary) : std::numeric_limits<double>::infinity();
    bool only_a = r == 0.0 && b == 0.0 && cross == 0.0;
    bool only_b = q == 0.0 && a == 0.0 && cross == 0.0;
    if (only_a && q > 0.0) upper = 0.5 * a * a / (q * rho2);
    if (only_b && r > 0.0) upper = 0.5 * b * b / (r * rho2);
    if (only_a && only_b) upper = 0.0;
    if (a <= 0.0 && b <= 0.0) upper = 0.0;
    return upper * 1.000001 + 1e-6;
}

// ---------------------------------------------------------------------------
// Period grid, src/search/grid.rs:5-28
// ---------------------------------------------------------------------------

extern "C" int64_t orc_period_grid(double minimum, double maximum, double baseline, double minimum_duration,
                                   double oversample, double* out, int64_t capacity) {
    double log_step = std::log1p(minimum_duration / (oversample * baseline));
    int64_t count = (int64_t)as_usize(std::ceil(std::log(maximum / minimum) / log_step)) + 1;
    if (out == nullptr || capacity < count) return count;
    double a = std::log(minimum), b = std::log(maximum);
    for (int64_t i = 0; i < count; i++) {
        double x = count == 1 ? a : a + (b - a) * (double)i / (double)(count - 1);
        out[i] = std::exp(x);
    }
    out[0] = minimum;
    out[count - 1] = maximum;
    return count;
}

// ---------------------------------------------------------------------------
// Host preparation in prepared mode: src/prep/stats.rs:4-18,
// src/prep/curve.rs:89-198 (bin_minutes = 0, one group), :427-450, :456-539,
// :541-569.
// ---------------------------------------------------------------------------

static double median_lower(const std::vector<double>& values) {
    std::vector<double> v;
    v.reserve(values.size());
    for (double x : values)
        if (std::isfinite(x)) v.push_back(x);
    if (v.empty()) return std::nan("");
    std::sort(v.begin(), v.end());
    return v[(v.size() - 1) / 2];
}

static double mad_scale(const std::vector<double>& values) {
    double m = median_lower(values);
    std::vector<double> dev(values.size());
    for (size_t i = 0; i < values.size(); i++) dev[i] = std::fabs(values[i] - m);
    return 1.4826 * median_lower(dev);
}

extern "C" double orc_median_lower(const double* v, int64_t n) {
    return median_lower(std::vector<double>(v, v + n));
}

// fit_segment_noise with err given, no groups and no binning, as family_state
// calls it (curve.rs:548). Inputs are sorted by time by the caller
// (search_prepared sorts, pipeline.rs:52-58); a stable argsort is applied anyway.
// Returns 0, or 1 "insufficient usable observations", 2 "mission flux must have
// a positive median", 3 "no adjacent observations available".
static int fit_segment_noise_nobin(const double* time, const double* flux, const double* err, int64_t n_in,
                                   double gap_days, std::vector<double>& t, std::vector<double>& deficit,
                                   std::vector<double>& variance, double& origin, double& inflation,
                                   int64_t& segments) {
    std::vector<int64_t> keep;
    for (int64_t i = 0; i < n_in; i++)
        if (std::isfinite(time[i]) && std::isfinite(flux[i]) && std::isfinite(err[i]) && err[i] > 0.0) keep.push_back(i);
    std::vector<size_t> order(keep.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return time[keep[a]] < time[keep[b]]; });
    size_t n = keep.size();
    t.resize(n);
    std::vector<double> f(n), e(n);
    for (size_t i = 0; i < n; i++) {
        int64_t k = keep[order[i]];
        t[i] = time[k];
        f[i] = flux[k];
        e[i] = err[k];
    }
    if (n < 6) return 1;
    double m = median_lower(f);
    if (!(m > 0.0)) return 2;
    for (size_t i = 0; i < n; i++) {
        f[i] = f[i] / m - 1.0;
        e[i] /= m;
    }
    origin = t[0];
    for (size_t i = 0; i < n; i++) t[i] -= origin;
    std::vector<double> standardized;
    for (size_t i = 1; i < n; i++) {
        if (t[i] - t[i - 1] < gap_days) {
            double d = f[i] - f[i - 1];
            standardized.push_back(d / std::sqrt(e[i] * e[i] + e[i - 1] * e[i - 1]));
        }
    }
    if (standardized.empty()) return 3;
    inflation = rmax(mad_scale(standardized), 1.0);
    variance.resize(n);
    for (size_t i = 0; i < n; i++) {
        double x = e[i] * inflation;
        variance[i] = x * x;
    }
    segments = 1;
    for (size_t i = 1; i < n; i++)
        if (t[i] - t[i - 1] > gap_days) segments++;
    deficit.resize(n);
    for (size_t i = 0; i < n; i++) deficit[i] = -f[i];
    return 0;
}

static std::vector<double> correlated_noise_factors(const std::vector<double>& time, const std::vector<double>& residual,
                                                    const std::vector<double>& sigma, const double* durations, int nd) {
    const double min_fill = 0.5;
    const size_t minimum_bins = 20;
    size_t n = time.size();
    std::vector<double> weights(n);
    for (size_t i = 0; i < n; i++) weights[i] = 1.0 / (sigma[i] * sigma[i]);
    std::vector<double> steps;
    for (size_t i = 1; i < n; i++) {
        double s = time[i] - time[i - 1];
        if (s > 0.0) steps.push_back(s);
    }
    double cadence = median_lower(steps);
    std::vector<double> measured;
    std::vector<size_t> counts;
    for (int di = 0; di < nd; di++) {
        double d = durations[di];
        std::vector<double> z;
        double total = 0.0, acc = 0.0;
        size_t cnt = 0;
        int64_t current = INT64_MIN;
        auto flush = [&]() {
            if (cnt > 0 && (double)cnt >= min_fill * d / cadence) z.push_back((acc / total) * std::sqrt(total));
        };
        for (size_t i = 0; i < n; i++) {
            int64_t cell = as_i64(std::floor((time[i] - time[0]) / d));
            if (cell != current) {
                flush();
                current = cell;
                total = 0.0;
                acc = 0.0;
                cnt = 0;
            }
            total += weights[i];
            acc += weights[i] * residual[i];
            cnt += 1;
        }
        flush();
        counts.push_back(z.size());
        measured.push_back(z.size() >= 3 ? rmax(mad_scale(z), 1.0) : 1.0);
    }
    std::vector<bool> supported(nd);
    bool any = false;
    for (int i = 0; i < nd; i++) {
        supported[i] = counts[i] >= minimum_bins;
        any = any || supported[i];
    }
    std::vector<double> inherited(nd);
    if (any) {
        std::vector<int> valid;
        for (int i = 0; i < nd; i++)
            if (supported[i]) valid.push_back(i);
        for (int i = 0; i < nd; i++) {
            double d = durations[i];
            // Iterator::min_by keeps the first minimum.
            int anchor = valid[0];
            double best = std::fabs(std::log(d) - std::log(durations[anchor]));
            for (size_t v = 1; v < valid.size(); v++) {
                double dist = std::fabs(std::log(d) - std::log(durations[valid[v]]));
                if (dist < best) {
                    best = dist;
                    anchor = valid[v];
                }
            }
            inherited[i] = measured[anchor] * std::sqrt(rmax(d / durations[anchor], 1.0));
        }
    } else {
        std::vector<double> standardized(n);
        for (size_t i = 0; i < n; i++) standardized[i] = residual[i] / sigma[i];
        double scatter = rmax(mad_scale(standardized), 1.0);
        for (int i = 0; i < nd; i++) inherited[i] = scatter * std::sqrt(rmax(durations[i] / cadence, 1.0));
    }
    std::vector<double> out(nd);
    for (int i = 0; i < nd; i++) out[i] = supported[i] ? measured[i] : rmax(measured[i], inherited[i]);
    return out;
}

// family_state in prepared mode. out_* arrays hold at least n_in entries; the
// number of usable observations is written to *out_n. Status as
// fit_segment_noise_nobin, or 4 "invalid baseline precision".
extern "C" int orc_family_state(const double* time, const double* flux, const double* sigma, int64_t n_in,
                                const double* durations, int nd, int correlated, int64_t* out_n, double* out_time,
                                double* out_v, double* out_w, double* out_deficit, double* out_scalars,
                                double* out_rho) {
    std::vector<double> flux1(n_in);
    for (int64_t i = 0; i < n_in; i++) flux1[i] = 1.0 + flux[i];
    std::vector<double> t, deficit, variance;
    double origin = 0.0, inflation = 0.0;
    int64_t segments = 0;
    int st = fit_segment_noise_nobin(time, flux1.data(), sigma, n_in, 0.75, t, deficit, variance, origin, inflation,
                                     segments);
    if (st) return st;
    size_t n = t.size();
    std::vector<double> p(n);
    for (size_t i = 0; i < n; i++) p[i] = 1.0 / variance[i];
    double c = 0.0;
    for (size_t i = 0; i < n; i++) c += p[i];
    if (!(std::isfinite(c) && c > 0.0)) return 4;
    std::vector<double> py(n);
    for (size_t i = 0; i < n; i++) py[i] = p[i] * deficit[i];
    double s = 0.0;
    for (size_t i = 0; i < n; i++) s += py[i];
    double mean = s / c;
    double energy = 0.0;
    for (size_t i = 0; i < n; i++) {
        double v = py[i] - p[i] * mean;
        out_v[i] = v;
        out_w[i] = p[i];
        out_time[i] = t[i];
        out_deficit[i] = deficit[i];
        energy += deficit[i] * v;
    }
    *out_n = (int64_t)n;
    out_scalars[0] = c;
    out_scalars[1] = origin;
    out_scalars[2] = energy;
    out_scalars[3] = inflation;
    out_scalars[4] = (double)segments;
    if (correlated) {
        std::vector<double> resid(n), sig(n);
        for (size_t i = 0; i < n; i++) {
            resid[i] = -deficit[i];
            sig[i] = std::sqrt(variance[i]);
        }
        std::vector<double> rho = correlated_noise_factors(t, resid, sig, durations, nd);
        for (int i = 0; i < nd; i++) out_rho[i] = rho[i];
    } else {
        for (int i = 0; i < nd; i++) out_rho[i] = 1.0;
    }
    return 0;
}

// Noise model of an arbitrary (time, flux, err) series (curve.rs:89-198 with
// bin_minutes = 0 and no groups), for the reference's noise-model test.
extern "C" int orc_fit_segment_noise(const double* time, const double* flux, const double* err, int64_t n_in,
                                     double gap_days, int64_t* out_n, double* out_time, double* out_deficit,
                                     double* out_variance, double* out_scalars) {
    std::vector<double> t, deficit, variance;
    double origin = 0.0, inflation = 0.0;
    int64_t segments = 0;
    int st = fit_segment_noise_nobin(time, flux, err, n_in, gap_days, t, deficit, variance, origin, inflation, segments);
    if (st) return st;
    *out_n = (int64_t)t.size();
    for (size_t i = 0; i < t.size(); i++) {
        out_time[i] = t[i];
        out_deficit[i] = deficit[i];
        out_variance[i] = variance[i];
    }
    out_scalars[0] = origin;
    out_scalars[1] = inflation;
    out_scalars[2] = (double)segments;
    return 0;
}

// Biweight detrending, both of the reference's forms: the GPU kernel's
// (kernels.rs:1051-1110: lower medians by bisection on the value range,
// window_median :333-377) and the CPU function's (curve.rs:202-250: lower
// medians by sorting). Windows [t - window/2, t + window/2] within
// gap-separated segments; out = (1 + f) / location - 1.
namespace {
double bisect_median(const double* x, size_t a, size_t e, size_t k, double center, bool absolute) {
    auto value = [&](size_t j) { return absolute ? std::fabs(x[j] - center) : x[j]; };
    double vlo = INFINITY, vhi = -INFINITY;
    for (size_t j = a; j < e; j++) {
        vlo = std::fmin(vlo, value(j));
        vhi = std::fmax(vhi, value(j));
    }
    for (int it = 0; it < 64 && vhi > vlo; it++) {
        const double mid = 0.5 * (vlo + vhi);
        if (mid <= vlo || mid >= vhi) break;
        size_t below = 0;
        for (size_t j = a; j < e; j++) below += value(j) < mid ? 1 : 0;
        if (below <= k)
            vlo = mid;
        else
            vhi = mid;
    }
    double best = INFINITY;
    for (size_t j = a; j < e; j++)
        if (value(j) >= vlo && value(j) < best) best = value(j);
    return best;
}
}  // namespace

extern "C" void orc_biweight_flatten(const double* time, const double* relative, int64_t n, double window, double gap,
                                     double c, int iterations, int sorted_medians, double* out) {
    std::vector<double> flux(n);
    for (int64_t i = 0; i < n; i++) flux[i] = 1.0 + relative[i];
    int64_t start = 0;
    for (int64_t i = 1; i <= n; i++) {
        if (i < n && !(time[i] - time[i - 1] > gap)) continue;
        const double* t0 = time + start;
        const double* t1 = time + i;
        for (int64_t p = start; p < i; p++) {
            const size_t a = (size_t)(std::lower_bound(t0, t1, time[p] - window / 2.0) - time);
            const size_t e = (size_t)(std::upper_bound(t0, t1, time[p] + window / 2.0) - time);
            const size_t k = (e - a - 1) / 2;
            std::vector<double> vals(flux.begin() + a, flux.begin() + e);
            double location = sorted_medians ? median_lower(vals) : bisect_median(flux.data(), a, e, k, 0.0, false);
            for (int it = 0; it < iterations; it++) {
                double med;
                if (sorted_medians) {
                    std::vector<double> dev(vals.size());
                    for (size_t j = 0; j < vals.size(); j++) dev[j] = std::fabs(vals[j] - location);
                    med = median_lower(dev);
                } else {
                    med = bisect_median(flux.data(), a, e, k, location, true);
                }
                const double scale = std::fmax(c * med, 1e-12);
                double total = 0.0, acc = 0.0;
                for (size_t j = a; j < e; j++) {
                    const double v = flux[j];
                    const double u = (v - location) / scale;
                    if (std::fabs(u) < 1.0) {
                        const double wt = (1.0 - u * u) * (1.0 - u * u);
                        total += wt;
                        acc += wt * v;
                    }
                }
                if (total > 0.0) location = acc / total;
            }
            out[p] = flux[p] / location - 1.0;
        }
        start = i;
    }
}

// transit_mask, curve.rs:572-585: count of masked observations and the mask.
extern "C" int64_t orc_transit_mask(const double* time, int64_t n, double period, double epoch, double duration,
                                    double margin, uint8_t* mask) {
    int64_t count = 0;
    for (int64_t i = 0; i < n; i++) {
        double x = time[i] - epoch + period / 2.0;
        double r = std::fmod(x, period);
        if (r < 0.0) r += period;  // rem_euclid
        double phase = r - period / 2.0;
        bool m = std::fabs(phase) <= (1.0 + margin) * duration / 2.0;
        if (mask) mask[i] = m;
        count += m;
    }
    return count;
}

// Peak-selection rescoring, kernels.rs:936-1042 (RESCORE_BLOCK = 256, :41):
// per row, lane l of 256 sums the observations i = l (mod 256) in increasing
// i, then the lanes' partial sums meet in the tree red[l] += red[l + s] for
// s = 128, 64, ..., 1. Every observation is visited, as in the reference.
namespace {
constexpr int RESCORE_LANES = 256;

template <typename T>
T lane_tree(std::vector<T>& red) {
    for (int stride = RESCORE_LANES / 2; stride > 0; stride /= 2)
        for (int l = 0; l < stride; l++) red[l] = red[l] + red[l + stride];
    return red[0];
}
}  // namespace

extern "C" void orc_rescore_rows(const double* time, const double* v, const double* w, const uint8_t* excluded,
                                 int64_t n, const double* rows, int64_t R, double origin, double* sums) {
    std::vector<double> ra(RESCORE_LANES), rh(RESCORE_LANES), rn(RESCORE_LANES);
    for (int64_t r = 0; r < R; r++) {
        const double period = rows[3 * r], epoch = rows[3 * r + 1], duration = rows[3 * r + 2];
        const double inverse = 1.0 / period;
        const double half = duration / 2.0;
        for (int l = 0; l < RESCORE_LANES; l++) {
            double a = 0.0, hp = 0.0, norm = 0.0;
            for (int64_t i = l; i < n; i += RESCORE_LANES) {
                if (excluded[i] != 0) continue;
                const double x = (time[i] + origin - epoch) * inverse + 0.5;
                const double phase = (x - std::floor(x) - 0.5) * period;
                if (std::fabs(phase) <= half) {
                    a += v[i];
                    hp += w[i];
                    norm += w[i];
                }
            }
            ra[l] = a;
            rh[l] = hp;
            rn[l] = norm;
        }
        sums[3 * r] = lane_tree(ra);
        sums[3 * r + 1] = lane_tree(rh);
        sums[3 * r + 2] = lane_tree(rn);
    }
}

extern "C" void orc_count_rows(const double* time, const uint8_t* excluded, int64_t n, const double* rows, int64_t R,
                               uint32_t* counts) {
    std::vector<uint32_t> rt(RESCORE_LANES), ru(RESCORE_LANES);
    for (int64_t r = 0; r < R; r++) {
        const double period = rows[3 * r], epoch = rows[3 * r + 1], duration = rows[3 * r + 2];
        const double inverse = 1.0 / period;
        const double half = duration / 2.0;
        for (int l = 0; l < RESCORE_LANES; l++) {
            uint32_t total = 0, unshared = 0;
            for (int64_t i = l; i < n; i += RESCORE_LANES) {
                const double x = (time[i] - epoch) * inverse + 0.5;
                const double phase = (x - std::floor(x) - 0.5) * period;
                if (std::fabs(phase) <= half) {
                    total += 1;
                    unshared += excluded[i] == 0 ? 1u : 0u;
                }
            }
            rt[l] = total;
            ru[l] = unshared;
        }
        counts[2 * r] = lane_tree(rt);
        counts[2 * r + 1] = lane_tree(ru);
    }
}

// ---------------------------------------------------------------------------
// Scan path: fold (kernels.rs:465-553), doubled prefix sums (:237-309),
// tile scan (:610-845, helpers :51-146, :389-455), merge (:1115-1155).
// ---------------------------------------------------------------------------

namespace {

struct Bank {
    const double* durations;
    const double* rho;
    int nd;
    const double* ingress;
    int ns;
    int layers;
    const double* factors;  // ns * layers, scan.rs:157-171
    double gate;            // shape gate in score units
    double baseline;        // baseline_norm c
    double n;               // observation count as f64
};

struct PeriodView {
    const double* cum;   // NF x (2nb+1), field-major
    const float* cum32;  // NF x (2nb+1) x (hi, lo)
    int nb;
    int stride;
};

inline double interval(const PeriodView& P, int field, size_t start, size_t width) {
    size_t base = (size_t)field * P.stride;
    return P.cum[base + start + width] - P.cum[base + start];
}

inline float interval32(const PeriodView& P, int field, size_t start, size_t width) {
    size_t base = 2 * ((size_t)field * P.stride + start);
    size_t end = base + 2 * width;
    return (P.cum32[end] - P.cum32[base]) + (P.cum32[end + 1] - P.cum32[base + 1]);
}

inline size_t layer_width(size_t k, double factor) {
    size_t w = as_usize(std::floor((double)k * factor + 0.5));
    return w < 1 ? 1 : w;
}

inline void shape_sums(const PeriodView& P, size_t j, size_t k, double oa, double ohp, double onorm, double ingress,
                       const Bank& B, int si, double& a, double& hp, double& norm) {
    if (ingress == 0.0) {
        a = oa;
        hp = ohp;
        norm = onorm;
        return;
    }
    int layers = B.layers;
    double l = (double)layers;
    a = oa / l;
    hp = ohp / l;
    norm = onorm / (l * l);
    for (int layer = 1; layer < layers; layer++) {
        double factor = B.factors[si * layers + layer];
        size_t width = layer_width(k, factor);
        size_t start = j + (k - width) / 2;
        double dw = interval(P, F_W, start, width);
        a += interval(P, F_V, start, width) / l;
        hp += dw / l;
        norm += dw * ((2.0 * (double)layer + 1.0) / (l * l));
    }
}

inline void shape_sums_f32(const PeriodView& P, size_t j, size_t k, float oa, float ohp, float onorm, double ingress,
                           const Bank& B, int si, float& a, float& hp, float& norm) {
    if (ingress == 0.0) {
        a = oa;
        hp = ohp;
        norm = onorm;
        return;
    }
    int layers = B.layers;
    float l = (float)layers;
    a = oa / l;
    hp = ohp / l;
    norm = onorm / (l * l);
    for (int layer = 1; layer < layers; layer++) {
        double factor = B.factors[si * layers + layer];
        size_t width = layer_width(k, factor);
        size_t start = j + (k - width) / 2;
        float dw = interval32(P, F_W, start, width);
        a += interval32(P, F_V, start, width) / l;
        hp += dw / l;
        norm += dw * ((2.0f * (float)layer + 1.0f) / (l * l));
    }
}

struct Lane {
    double best;
    uint64_t key;
    uint32_t di;
    bool bad, sensitive, unsafe_merit;
    void reset() {
        best = NEG_INF;
        key = KEY_MAX;
        di = 0;
        bad = sensitive = unsafe_merit = false;
    }
};

inline float rank_fast(Lane& lane, float a32, float hp32, float norm32, double rho, double baseline, bool valid,
                       uint64_t key, uint32_t di) {
    float cn = (float)baseline * norm32;
    float qq = (float)(rho * rho) * (cn - hp32 * hp32);
    float merit = a32 * a32 / qq;
    bool safe = cn > 0.0f && qq >= 0.001f * cn && merit >= 1e-30f && merit <= 1e30f;
    lane.unsafe_merit = lane.unsafe_merit || (valid && !safe);
    float best = (float)lane.best;
    const float guard = 1e-5f;
    bool near = best > 0.0f && std::fabs(merit - best) <= guard * rmaxf(merit, best);
    bool far_better = merit > best * (1.0f + 4.0f * guard);
    if (valid && safe && far_better)
        lane.sensitive = false;
    else
        lane.sensitive = lane.sensitive || (valid && safe && near);
    bool better = valid && safe && (merit > best || (merit == best && key < lane.key));
    if (better) {
        lane.best = (double)merit;
        lane.key = key;
        lane.di = di;
    }
    return (valid && safe) ? merit : -std::numeric_limits<float>::infinity();
}

inline double rank_exact(Lane& lane, double a, double hp, double norm, double rho, double baseline, bool valid,
                         uint64_t key, uint32_t di) {
    double d = hp * hp / baseline;
    double q = norm - d;
    lane.bad = lane.bad || (valid && q <= 0.0);
    double candidate = (a / rho) / std::sqrt(rmax(q, 1e-300));
    double merit = (valid && q > 0.0 && candidate < std::numeric_limits<double>::infinity()) ? candidate : NEG_INF;
    bool better = merit > lane.best || (merit == lane.best && key < lane.key);
    if (better) {
        lane.best = merit;
        lane.key = key;
        lane.di = di;
    }
    return merit;
}

// One tile of TILE phase lanes of one period: returns the 9 part values, the
// winner key and the flags word (bit 0 retry as the reference reports it,
// bit 1 nonpositive precision). *retried is set when the f64 rescan ran.
void scan_tile(const PeriodView& P, double scale, const Bank& B, int tile, bool mixed, double part[9],
               uint64_t& out_key, uint32_t& out_flags, bool& retried) {
    const int nb = P.nb;
    const uint64_t nb1 = (uint64_t)nb + 1;
    Lane st[TILE];
    float outer32[TILE][3];
    bool usable[TILE];
    bool fast = mixed;
    bool retry = false;
    uint64_t winner_key = KEY_MAX;
    uint32_t winner_di = 0;
    double winner_value = NEG_INF;
    bool bad_any = false;
    retried = false;
    for (int l = 0; l < TILE; l++) st[l].reset();
    for (int pass = 0; pass < 2; pass++) {
        if (pass == 1) {
            if (!retry) break;
            fast = false;
            retried = true;
            for (int l = 0; l < TILE; l++) st[l].reset();
        }
        double gate_value = fast ? B.gate * B.gate / B.baseline : B.gate;
        for (int di = 0; di < B.nd; di++) {
            size_t raw_k = as_usize(std::floor(B.durations[di] * scale + 0.5));
            if (raw_k < 1) raw_k = 1;
            size_t k = std::min(raw_k, (size_t)(nb / 2));
            double r = B.rho[di];
            bool passing = false;
            for (int lane = 0; lane < TILE; lane++) {
                size_t j = (size_t)tile * TILE + lane;
                size_t jj = std::min(j, (size_t)(nb - 1));
                uint64_t key = (uint64_t)k * nb1 + jj;
                double merit;
                bool valid;
                if (fast) {
                    float count = interval32(P, F_N, jj, k);
                    float w = interval32(P, F_W, jj, k);
                    float a = interval32(P, F_V, jj, k);
                    outer32[lane][0] = a;
                    outer32[lane][1] = w;
                    outer32[lane][2] = w;
                    usable[lane] = j < (size_t)nb && raw_k < (size_t)(nb / 2) && count >= 3.0f && (double)count <= B.n - 3.0;
                    valid = usable[lane] && a > 0.0f;
                    merit = (double)rank_fast(st[lane], a, w, w, r, B.baseline, valid, key, (uint32_t)di);
                } else {
                    double count = interval(P, F_N, jj, k);
                    double w = interval(P, F_W, jj, k);
                    double a = interval(P, F_V, jj, k);
                    usable[lane] = j < (size_t)nb && raw_k < (size_t)(nb / 2) && count >= 3.0 && count <= B.n - 3.0;
                    valid = usable[lane] && a > 0.0;
                    merit = rank_exact(st[lane], a, w, w, r, B.baseline, valid, key, (uint32_t)di);
                }
                passing = passing || (valid && merit >= gate_value);
            }
            if (!passing) continue;
            for (int si = 1; si < B.ns; si++) {
                double ing = B.ingress[si];
                for (int lane = 0; lane < TILE; lane++) {
                    size_t j = (size_t)tile * TILE + lane;
                    size_t jj = std::min(j, (size_t)(nb - 1));
                    uint64_t key = ((uint64_t)si * nb1 + k) * nb1 + jj;
                    if (fast) {
                        float a, hp, norm;
                        shape_sums_f32(P, jj, k, outer32[lane][0], outer32[lane][1], outer32[lane][2], ing, B, si, a,
                                       hp, norm);
                        rank_fast(st[lane], a, hp, norm, r, B.baseline, usable[lane] && a > 0.0f, key, (uint32_t)di);
                    } else {
                        double w = interval(P, F_W, jj, k);
                        double oa = interval(P, F_V, jj, k);
                        double a, hp, norm;
                        shape_sums(P, jj, k, oa, w, w, ing, B, si, a, hp, norm);
                        rank_exact(st[lane], a, hp, norm, r, B.baseline, usable[lane] && a > 0.0, key, (uint32_t)di);
                    }
                }
            }
        }
        if (fast) {
            for (int lane = 0; lane < TILE; lane++) {
                size_t j = (size_t)tile * TILE + lane;
                size_t jj = std::min(j, (size_t)(nb - 1));
                if (st[lane].best <= 0.0) st[lane].key = nb1 + jj;
            }
        }
        // block_winner: largest value, then smallest key, then lowest lane.
        int chosen = 0;
        for (int lane = 1; lane < TILE; lane++) {
            const Lane& c = st[lane];
            const Lane& b = st[chosen];
            if (c.best > b.best || (c.best == b.best && c.key < b.key)) chosen = lane;
        }
        double value = st[chosen].best;
        uint64_t key = st[chosen].key;
        double guard = fast ? 1e-5 : 1e-10;
        int near_count = 0;
        bool near_sensitive = false, unsafe_any = false, bad = false;
        for (int lane = 0; lane < TILE; lane++) {
            bool near_top = st[lane].best > 0.0 && st[lane].best >= value * (1.0 - guard);
            near_count += near_top;
            near_sensitive = near_sensitive || (near_top && st[lane].sensitive);
            unsafe_any = unsafe_any || st[lane].unsafe_merit;
            bad = bad || st[lane].bad;
        }
        winner_key = key;
        winner_value = value;
        winner_di = st[chosen].di;
        retry = fast && (unsafe_any || near_count > 1 || near_sensitive);
        bad_any = bad_any || bad;
    }
    // Lane 0 recomputes the winner in f64 (kernels.rs:800-843).
    size_t phase = (size_t)(winner_key % nb1);
    size_t width = (size_t)((winner_key / nb1) % nb1);
    size_t si = (size_t)(winner_key / (nb1 * nb1));
    size_t sic = std::min(si, (size_t)(B.ns - 1));
    double ing = B.ingress[sic];
    double r = B.rho[winner_di];
    double w = interval(P, F_W, phase, width);
    double oa = interval(P, F_V, phase, width);
    double a0, hp, norm;
    shape_sums(P, phase, width, oa, w, w, ing, B, (int)sic, a0, hp, norm);
    double a = a0 / r;
    double d = hp * hp / B.baseline;
    double q = rmax(norm - d, 1e-300);
    double value = winner_value > NEG_INF ? a / std::sqrt(q) : NEG_INF;
    double depth = a / q * r;
    part[0] = (double)phase;
    part[1] = (double)width;
    part[2] = a;
    part[3] = norm;
    part[4] = d;
    part[5] = ing;
    part[6] = r;
    part[7] = value;
    part[8] = depth;
    out_key = winner_key;
    out_flags = (uint32_t)retry | ((uint32_t)bad_any << 1);
}

// Inclusive scan of 32 values in the order of a warp-shuffle Hillis-Steele
// scan (kernels.rs:221-232): step `off` adds the value `off` lanes below.
inline void warp_scan32(double x[32]) {
    for (int off = 1; off < 32; off <<= 1) {
        double prev[32];
        std::memcpy(prev, x, sizeof(prev));
        for (int l = off; l < 32; l++) x[l] = prev[l] + prev[l - off];
    }
}

// Doubled exclusive prefix of one field row with the association of the
// reference's prefix_block (kernels.rs:237-309): segments of 256 bins, each
// scanned as 8 warps of 32 (Hillis-Steele), warp offsets = carry plus the
// earlier warp totals in order, the carry grows by the sum of the 8 totals;
// the second copy is the first plus the final carry.
void prefix_row(const double* h, int nb, double* row) {
    row[0] = 0.0;
    double carry = 0.0;
    for (int seg = 0; seg < nb; seg += 256) {
        double local[8][32], wt[8];
        for (int wi = 0; wi < 8; wi++) {
            for (int l = 0; l < 32; l++) {
                int b = seg + wi * 32 + l;
                local[wi][l] = b < nb ? h[b] : 0.0;
            }
            warp_scan32(local[wi]);
            wt[wi] = local[wi][31];
        }
        for (int wi = 0; wi < 8; wi++) {
            double offset = carry;
            for (int u = 0; u < wi; u++) offset += wt[u];
            for (int l = 0; l < 32; l++) {
                int b = seg + wi * 32 + l;
                if (b < nb) row[b + 1] = local[wi][l] + offset;
            }
        }
        double total = 0.0;
        for (int wi = 0; wi < 8; wi++) total += wt[wi];
        carry += total;
    }
    for (int b = 0; b < nb; b++) row[nb + b + 1] = row[b + 1] + carry;
}

// Fold in observation order (each bin's additions in increasing observation
// index, one valid order of the reference's unordered atomics), then the
// doubled prefix sums and their (hi, lo) f32 pairs.
void fold_and_prefix(const double* time, const double* v, const double* w, int64_t n, double scale, int nb,
                     std::vector<double>& folded, std::vector<double>& cum, std::vector<float>& cum32) {
    folded.assign((size_t)nb * NF, 0.0);
    for (int64_t i = 0; i < n; i++) {
        double x = std::floor(time[i] * scale);
        uint32_t vv = (uint32_t)as_usize(x);
        uint32_t cell = vv % (uint32_t)nb;
        double* h = &folded[(size_t)cell * NF];
        h[F_V] += v[i];
        h[F_W] += w[i];
        h[F_N] += 1.0;
    }
    int stride = 2 * nb + 1;
    cum.assign((size_t)NF * stride, 0.0);
    cum32.assign((size_t)NF * stride * 2, 0.0f);
    std::vector<double> field(nb);
    for (int f = 0; f < NF; f++) {
        double* row = &cum[(size_t)f * stride];
        for (int b = 0; b < nb; b++) field[b] = folded[(size_t)b * NF + f];
        prefix_row(field.data(), nb, row);
        float* r32 = &cum32[(size_t)f * stride * 2];
        for (int b = 0; b < stride; b++) {
            float hi = (float)row[b];
            r32[2 * b] = hi;
            r32[2 * b + 1] = (float)(row[b] - (double)hi);
        }
    }
}

}  // namespace

// Per-period winners of scan_bank (scan.rs:144-357) for the periods given, at
// nb phase bins. records: P x 9 (period, scale, phase, width, a, norm, d,
// ingress, rho); score, depth: P. flags_or: per period OR of the tile flags.
// mode 0 = mixed precision (the reference's kernels), 1 = f64 ranking only.
// Returns the count of tiles whose f64 rescan ran.
extern "C" int64_t orc_scan_bank(const double* time, const double* v, const double* w, int64_t n, double baseline_norm,
                                 const double* periods, int64_t P, int nb, const double* durations, const double* rho,
                                 int nd, const double* ingress, int ns, int layers, double shape_gate, int mode,
                                 int threads, double* records, double* score, double* depth, uint32_t* flags_or) {
    std::vector<double> factors((size_t)ns * layers);
    for (int s = 0; s < ns; s++)
        for (int l = 0; l < layers; l++)
            factors[(size_t)s * layers + l] =
                1.0 - 2.0 * ingress[s] * (layers > 1 ? (double)l / (double)(layers - 1) : 0.0);
    Bank B{durations, rho, nd, ingress, ns, layers, factors.data(), shape_gate, baseline_norm, (double)n};
    int tiles = (nb + TILE - 1) / TILE;
    std::atomic<int64_t> next{0};
    std::atomic<int64_t> retries{0};
    auto work = [&]() {
        std::vector<double> folded, cum;
        std::vector<float> cum32;
        std::vector<double> parts((size_t)tiles * 9);
        std::vector<uint64_t> keys(tiles);
        int64_t local_retries = 0;
        for (;;) {
            int64_t f = next.fetch_add(1);
            if (f >= P) break;
            double scale = (double)nb / periods[f];
            fold_and_prefix(time, v, w, n, scale, nb, folded, cum, cum32);
            PeriodView PV{cum.data(), cum32.data(), nb, 2 * nb + 1};
            uint32_t fo = 0;
            for (int t = 0; t < tiles; t++) {
                uint32_t fl;
                bool retried;
                scan_tile(PV, scale, B, t, mode == 0, &parts[(size_t)t * 9], keys[t], fl, retried);
                fo |= fl;
                local_retries += retried;
            }
            // merge_tiles
            double best = NEG_INF;
            uint64_t key = KEY_MAX;
            int chosen = 0;
            for (int t = 0; t < tiles; t++) {
                double val = parts[(size_t)t * 9 + 7];
                if (val > best || (val == best && keys[t] < key)) {
                    best = val;
                    key = keys[t];
                    chosen = t;
                }
            }
            double* rec = &records[f * 9];
            rec[0] = periods[f];
            rec[1] = scale;
            for (int i = 0; i < 7; i++) rec[2 + i] = parts[(size_t)chosen * 9 + i];
            score[f] = best;
            depth[f] = parts[(size_t)chosen * 9 + 8];
            if (flags_or) flags_or[f] = fo;
        }
        retries += local_retries;
    };
    if (threads <= 1) {
        work();
    } else {
        std::vector<std::thread> pool;
        for (int i = 0; i < threads; i++) pool.emplace_back(work);
        for (auto& th : pool) th.join();
    }
    return retries.load();
}

// The folded histogram and doubled prefix sums of one period (for tests of
// the fold and prefix kernels): folded nb x 3, cum 3 x (2nb+1), cum32 2x that.
extern "C" void orc_fold_prefix(const double* time, const double* v, const double* w, int64_t n, double scale, int nb,
                                double* folded_out, double* cum_out, float* cum32_out) {
    std::vector<double> folded, cum;
    std::vector<float> cum32;
    fold_and_prefix(time, v, w, n, scale, nb, folded, cum, cum32);
    std::memcpy(folded_out, folded.data(), folded.size() * sizeof(double));
    std::memcpy(cum_out, cum.data(), cum.size() * sizeof(double));
    std::memcpy(cum32_out, cum32.data(), cum32.size() * sizeof(float));
}

// Direct per-observation box statistic of phase window [j, j+k) (mod nb) at
// one period, without fold or prefix: (a, hp, count). A brute-force check of
// the fold + prefix + interval arithmetic.
extern "C" void orc_box_direct(const double* time, const double* v, const double* w, int64_t n, double scale, int nb,
                               int64_t j, int64_t k, double* out3) {
    double a = 0.0, hp = 0.0, c = 0.0;
    for (int64_t i = 0; i < n; i++) {
        int64_t cell = (int64_t)((uint32_t)as_usize(std::floor(time[i] * scale)) % (uint32_t)nb);
        int64_t off = cell - j;
        if (off < 0) off += nb;
        if (off < k) {
            a += v[i];
            hp += w[i];
            c += 1.0;
        }
    }
    out3[0] = a;
    out3[1] = hp;
    out3[2] = c;
}

// Single-event scan, events.rs:18-153 with scan_all (kernels.rs:851-921):
// the fold and doubled prefix of one trial period at `scale` with nb bins,
// then every template (phase j, duration, shape) whose exact f64 score
// reaches the threshold, in (j, duration, shape) order: records of (j, k,
// score, depth = a / q). Returns the count; records beyond `capacity` are
// not written.
extern "C" int64_t orc_single_event_scan(const double* time, const double* v, const double* w, int64_t n,
                                         double baseline_norm, double scale, int nb, const double* durations,
                                         const double* rho, int nd, const double* ingress, int ns, int layers,
                                         double threshold, int64_t capacity, double* records) {
    std::vector<double> folded, cum;
    std::vector<float> cum32;
    fold_and_prefix(time, v, w, n, scale, nb, folded, cum, cum32);
    const PeriodView P{cum.data(), cum32.data(), nb, 2 * nb + 1};
    std::vector<double> factors;
    for (int s = 0; s < ns; s++)
        for (int l = 0; l < layers; l++)
            factors.push_back(1.0 - 2.0 * ingress[s] * (layers > 1 ? (double)l / (double)(layers - 1) : 0.0));
    const Bank B{durations, rho, nd, ingress, ns, layers, factors.data(), 0.0, baseline_norm, (double)n};
    const size_t half = (size_t)nb / 2;
    int64_t count = 0;
    for (size_t j = 0; j < (size_t)nb; j++) {
        for (int di = 0; di < nd; di++) {
            size_t raw = as_usize(std::floor(durations[di] * scale + 0.5));
            if (raw < 1) raw = 1;
            const size_t k = raw < half ? raw : half;
            const double r = rho[di];
            const double cnt = interval(P, F_N, j, k);
            const double ww = interval(P, F_W, j, k);
            const double oa = interval(P, F_V, j, k);
            if (!(raw < half && cnt >= 3.0 && cnt <= (double)n - 3.0)) continue;
            for (int si = 0; si < ns; si++) {
                double a, hp, norm;
                shape_sums(P, j, k, oa, ww, ww, ingress[si], B, si, a, hp, norm);
                const double q = norm - hp * hp / baseline_norm;
                if (!(a > 0.0 && q > 0.0)) continue;
                const double score = (a / r) / std::sqrt(q);
                if (score >= threshold) {
                    if (count < capacity) {
                        double* rec = records + 4 * count;
                        rec[0] = (double)j;
                        rec[1] = (double)k;
                        rec[2] = score;
                        rec[3] = a / q;
                    }
                    count++;
                }
            }
        }
    }
    return count;
}

// ---------------------------------------------------------------------------
// Evidence: src/search/evidence.rs:37-67 (helpers), :75-144 (fold, prefix),
// :151-273 (screen), :280-632 (joint tiles), :655-1003 (host).
// ---------------------------------------------------------------------------

namespace {

constexpr int EV_TILE = 64;
constexpr int PART = 15;
constexpr int NORB = 3;
constexpr int NPARAM = 30;

inline double circular_sum(const double* cum, size_t row, size_t start, size_t width, size_t nb2) {
    size_t j = start % nb2;
    size_t end = j + width;
    double left = cum[row + j];
    double right = cum[row + std::min(end, nb2)];
    double wrap = cum[row + (end > nb2 ? end - nb2 : 0)];
    return right - left + wrap;
}

inline double layered_sum(const double* cum, size_t row, size_t start, size_t width, const double* shapes, int si,
                          size_t nb2, int layers, bool squared) {
    double value = 0.0;
    for (int layer = 0; layer < layers; layer++) {
        double fraction = shapes[((size_t)si * layers + layer) * 3];
        size_t inner = as_usize(std::floor((double)width * fraction + 0.5));
        if (inner < 1) inner = 1;
        double coefficient = shapes[((size_t)si * layers + layer) * 3 + (squared ? 2 : 1)];
        value += coefficient * circular_sum(cum, row, start + (width - inner) / 2, inner, nb2);
    }
    return value;
}

double logsumexp(const std::vector<double>& v) {
    double high = NEG_INF;
    for (double x : v) high = rmax(high, x);
    if (high == NEG_INF) return high;
    double s = 0.0;
    for (double x : v) s += std::exp(x - high);
    return high + std::log(s);
}

struct EvidenceInputs {
    const double* cum;  // 3 x (nb2+1)
    double scale;
    const double* durations;
    const double* rho;
    const double* dlm;
    const double* shapes;
    const double* priors;
    const double* params;
    const double* orbit;
    double baseline;
    double threshold;
    double n;
    size_t nb2;
    int nd, ns, layers;
};

void comparison_screen_tile(const EvidenceInputs& E, int tile, double* screen) {
    size_t nb2 = E.nb2, nb = nb2 / 2;
    double best[EV_TILE], bound_merit[EV_TILE];
    double best_a[EV_TILE], best_q[EV_TILE], best_null[EV_TILE], best_ps[EV_TILE], best_bs[EV_TILE];
    uint64_t best_key[EV_TILE];
    double c = E.baseline;
    for (int lane = 0; lane < EV_TILE; lane++) {
        size_t j = (size_t)tile * EV_TILE + lane;
        size_t jj = std::min(j, nb - 1);
        best[lane] = NEG_INF;
        bound_merit[lane] = NEG_INF;
        best_a[lane] = 0.0;
        best_q[lane] = 1.0;
        best_null[lane] = best_ps[lane] = best_bs[lane] = 0.0;
        best_key[lane] = 0;
        for (int di = 0; di < E.nd; di++) {
            size_t raw_k = as_usize(std::floor(E.durations[di] * E.scale + 0.5));
            if (raw_k < 1) raw_k = 1;
            size_t k = std::min(raw_k, nb2 / 8 - 1);
            double r = E.rho[di];
            double count = circular_sum(E.cum, 2 * (nb2 + 1), jj, k, nb2) + circular_sum(E.cum, 2 * (nb2 + 1), jj + nb, k, nb2);
            bool usable = j < nb && raw_k < nb2 / 8 && count >= 3.0 && count <= E.n - 3.0;
            for (int si = 0; si < E.ns; si++) {
                double a = layered_sum(E.cum, 0, jj, k, E.shapes, si, nb2, E.layers, false) +
                           layered_sum(E.cum, 0, jj + nb, k, E.shapes, si, nb2, E.layers, false);
                double pe = layered_sum(E.cum, nb2 + 1, jj, k, E.shapes, si, nb2, E.layers, false);
                double po = layered_sum(E.cum, nb2 + 1, jj + nb, k, E.shapes, si, nb2, E.layers, false);
                double ne = layered_sum(E.cum, nb2 + 1, jj, k, E.shapes, si, nb2, E.layers, true);
                double no = layered_sum(E.cum, nb2 + 1, jj + nb, k, E.shapes, si, nb2, E.layers, true);
                double qe = ne - pe * pe / c, qo = no - po * po / c, qeo = -pe * po / c;
                double q = qe + qo + 2.0 * qeo;
                double score = a / std::sqrt(rmax(q * (r * r), 1e-300));
                bool score_valid = usable && a > 0.0 && q > 0.0;
                double merit = 0.5 * score * score + E.dlm[di] + E.priors[si * 2];
                if (score_valid && merit > bound_merit[lane]) {
                    best_a[lane] = a / (r * r);
                    best_q[lane] = q / (r * r);
                    best_null[lane] = E.dlm[di];
                    best_ps[lane] = E.priors[si * 2];
                    best_bs[lane] = E.priors[si * 2 + 1];
                    best_key[lane] = (uint64_t)(si * E.nd + di) * nb + jj;
                    bound_merit[lane] = merit;
                }
                if (score_valid && score > best[lane]) best[lane] = score;
            }
        }
    }
    double maximum = NEG_INF, bound_maximum = NEG_INF;
    int chosen = EV_TILE;
    for (int l = 0; l < EV_TILE; l++) {
        if (best[l] > maximum) maximum = best[l];
        if (bound_merit[l] > bound_maximum) {
            bound_maximum = bound_merit[l];
            chosen = l;
        }
    }
    if (chosen == EV_TILE) return;  // the zeroed screen entry stays as it is
    int L = chosen;
    double lower_p = orc_positive_amplitude_evidence(best_a[L], best_q[L], E.params[0]) + std::log(0.75) + best_null[L] +
                     best_ps[L];
    double lower_b = orc_log_add(orc_positive_amplitude_evidence(best_a[L], best_q[L], E.params[1]),
                                 orc_positive_amplitude_evidence(best_a[L], best_q[L], E.params[2])) +
                     std::log(0.025) + best_null[L] + best_bs[L];
    double* out = &screen[(size_t)tile * 4];
    out[0] = maximum;
    out[1] = bound_maximum > NEG_INF ? lower_p : NEG_INF;
    out[2] = bound_maximum > NEG_INF ? lower_b : NEG_INF;
    out[3] = (double)best_key[L];
}

struct JointLane {
    double best_joint, best_signal;
    uint64_t joint_key, signal_key;
    double j_out[9], s_out[9];
    double sum_p, sum_b;
    uint32_t omitted;
};

void joint_tile(const EvidenceInputs& E, int tile, bool pilot, const double floors[3], double* parts) {
    size_t nb2 = E.nb2, nb = nb2 / 2;
    const int nd = E.nd;
    uint64_t pilot_key = as_usize(floors[2]);
    double c = E.baseline;
    double tau_p = E.params[0], tau_b = E.params[1], tau_d = E.params[2];
    double floor_p = pilot ? NEG_INF : floors[0];
    double floor_b = pilot ? NEG_INF : floors[1];
    JointLane L[EV_TILE];
    size_t jv[EV_TILE], jjv[EV_TILE];
    for (int lane = 0; lane < EV_TILE; lane++) {
        JointLane& s = L[lane];
        s.best_joint = s.best_signal = NEG_INF;
        s.joint_key = s.signal_key = KEY_MAX;
        for (int i = 0; i < 9; i++) s.j_out[i] = s.s_out[i] = 0.0;
        s.sum_p = s.sum_b = NEG_INF;
        s.omitted = 0;
        size_t j = pilot ? (size_t)(pilot_key % nb) : (size_t)tile * EV_TILE + lane;
        jv[lane] = j;
        jjv[lane] = std::min(j, nb - 1);
    }
    int di_begin = 0, di_end = nd;
    if (pilot) {
        di_begin = (int)((pilot_key / nb) % (uint64_t)nd);
        di_end = di_begin + 1;
    }
    // Per-lane quantities carried across the tile-wide reductions.
    struct Tmp {
        double ae, ao, pe, po, qe, qo, qeo, ap, qp, snr, depth;
        bool valid;
        double lp, lb, component_best, sec_ratio, sec_phase, odd_ratio, binary_multiple, omitted_upper;
        double pa, pb, pq, pr, px, raw_upper;
    };
    Tmp T[EV_TILE];
    for (int di = di_begin; di < di_end; di++) {
        size_t raw_k = as_usize(std::floor(E.durations[di] * E.scale + 0.5));
        if (raw_k < 1) raw_k = 1;
        size_t k = std::min(raw_k, nb2 / 8 - 1);
        double rho2 = E.rho[di] * E.rho[di];
        double dlm = E.dlm[di];
        int si_begin = 0, si_end = E.ns;
        if (pilot) {
            si_begin = (int)(pilot_key / ((uint64_t)nb * (uint64_t)nd));
            si_end = si_begin + 1;
        }
        bool usable[EV_TILE];
        for (int lane = 0; lane < EV_TILE; lane++) {
            size_t jj = jjv[lane];
            double count = circular_sum(E.cum, 2 * (nb2 + 1), jj, k, nb2) + circular_sum(E.cum, 2 * (nb2 + 1), jj + nb, k, nb2);
            usable[lane] = jv[lane] < nb && raw_k < nb2 / 8 && count >= 3.0 && count <= E.n - 3.0;
        }
        for (int si = si_begin; si < si_end; si++) {
            for (int lane = 0; lane < EV_TILE; lane++) {
                Tmp& t = T[lane];
                size_t jj = jjv[lane];
                t.ae = layered_sum(E.cum, 0, jj, k, E.shapes, si, nb2, E.layers, false);
                t.ao = layered_sum(E.cum, 0, jj + nb, k, E.shapes, si, nb2, E.layers, false);
                t.pe = layered_sum(E.cum, nb2 + 1, jj, k, E.shapes, si, nb2, E.layers, false);
                t.po = layered_sum(E.cum, nb2 + 1, jj + nb, k, E.shapes, si, nb2, E.layers, false);
                double ne = layered_sum(E.cum, nb2 + 1, jj, k, E.shapes, si, nb2, E.layers, true);
                double no = layered_sum(E.cum, nb2 + 1, jj + nb, k, E.shapes, si, nb2, E.layers, true);
                t.qe = ne - t.pe * t.pe / c;
                t.qo = no - t.po * t.po / c;
                t.qeo = -t.pe * t.po / c;
                t.ap = t.ae + t.ao;
                t.qp = t.qe + t.qo + 2.0 * t.qeo;
                t.snr = t.ap / std::sqrt(rmax(t.qp * rho2, 1e-300));
                t.depth = t.ap / rmax(t.qp, 1e-300);
                t.valid = usable[lane] && t.ap > 0.0 && t.qp > 0.0 && t.snr >= E.threshold;
            }
            if (!(raw_k < nb2 / 8)) continue;
            for (int lane = 0; lane < EV_TILE; lane++) {
                Tmp& t = T[lane];
                t.lp = t.lb = NEG_INF;
                t.component_best = NEG_INF;
                t.sec_ratio = 0.0;
                t.sec_phase = 0.5;
                t.odd_ratio = 1.0;
                t.binary_multiple = 1.0;
                t.omitted_upper = NEG_INF;
            }
            for (int phase_index = 0; phase_index < NORB; phase_index++) {
                size_t orbital = ((size_t)di * NORB + phase_index) * 4;
                double phase = E.orbit[orbital];
                double duration_ratio = E.orbit[orbital + 1];
                double logwp = E.orbit[orbital + 2], logwb = E.orbit[orbital + 3];
                int64_t offset = as_i64(std::floor(phase * (double)nb + 0.5));
                int64_t sk64 = as_i64(std::floor((double)k * duration_ratio + 0.5));
                if (sk64 < 1) sk64 = 1;
                if (sk64 > (int64_t)nb - 1) sk64 = (int64_t)nb - 1;
                size_t sk = (size_t)sk64;
                double upper_l[EV_TILE];
                for (int lane = 0; lane < EV_TILE; lane++) {
                    Tmp& t = T[lane];
                    size_t jj = jjv[lane];
                    size_t s0 = (size_t)((int64_t)jj + offset + as_i64(std::floor(((double)k - (double)sk) / 2.0)));
                    size_t s1 = s0 + nb;
                    double ass = layered_sum(E.cum, 0, s0, sk, E.shapes, si, nb2, E.layers, false) +
                                 layered_sum(E.cum, 0, s1, sk, E.shapes, si, nb2, E.layers, false);
                    double ps = layered_sum(E.cum, nb2 + 1, s0, sk, E.shapes, si, nb2, E.layers, false) +
                                layered_sum(E.cum, nb2 + 1, s1, sk, E.shapes, si, nb2, E.layers, false);
                    double nsum = layered_sum(E.cum, nb2 + 1, s0, sk, E.shapes, si, nb2, E.layers, true) +
                                  layered_sum(E.cum, nb2 + 1, s1, sk, E.shapes, si, nb2, E.layers, true);
                    double qs = nsum - ps * ps / c;
                    double qps = -(t.pe + t.po) * ps / c;
                    t.pa = t.ap / rho2;
                    t.pb = ass / rho2;
                    t.pq = t.qp / rho2;
                    t.pr = qs / rho2;
                    t.px = qps / rho2;
                    double cu = 1e-6;
                    double pu = orc_subspace_upper(t.pa, t.pb, t.pq, t.pr, t.px, 1.0) + logwp + cu;
                    double bu = orc_subspace_upper(t.pa, t.pb, t.pq, t.pr, t.px, 1.0) + logwb + cu;
                    double upper = rmax(pu - floor_p, bu - floor_b) + dlm;
                    if (!(logwp > NEG_INF || logwb > NEG_INF)) upper = NEG_INF;
                    t.raw_upper = logwb > NEG_INF ? bu : NEG_INF;
                    upper_l[lane] = jv[lane] < nb ? upper : NEG_INF;
                }
                double tile_max = NEG_INF;
                for (int l = 0; l < EV_TILE; l++)
                    if (upper_l[l] > tile_max) tile_max = upper_l[l];
                for (int lane = 0; lane < EV_TILE; lane++) {
                    Tmp& t = T[lane];
                    if (tile_max >= 0.0) {
                        for (int ri = 0; ri < 5; ri++) {
                            double ratio = E.params[6 + ri * 3];
                            double wp = E.params[7 + ri * 3], wb = E.params[8 + ri * 3];
                            double aa = t.pa + ratio * t.pb;
                            double qq = t.pq + 2.0 * ratio * t.px + ratio * ratio * t.pr;
                            double ep = orc_positive_amplitude_evidence(aa, qq, tau_p) + std::log(wp) + logwp;
                            double diluted = orc_positive_amplitude_evidence(aa, qq, tau_d);
                            double eb = orc_log_add(orc_positive_amplitude_evidence(aa, qq, tau_b), diluted) +
                                        std::log(0.25 * wb) + logwb;
                            t.lp = orc_log_add(t.lp, ep);
                            t.lb = orc_log_add(t.lb, eb);
                            if (eb > t.component_best) {
                                t.sec_ratio = ratio;
                                t.sec_phase = phase;
                                t.component_best = eb;
                            }
                        }
                    } else {
                        L[lane].omitted += 1;
                        if (t.raw_upper > t.omitted_upper) t.omitted_upper = t.raw_upper;
                    }
                }
            }
            // Alternating primaries at twice the period (binary family).
            double alias_mass = k < nb2 / 8 ? 0.0 : NEG_INF;
            double upper_l[EV_TILE];
            for (int lane = 0; lane < EV_TILE; lane++) {
                Tmp& t = T[lane];
                double ba = t.ae / rho2, bb = t.ao / rho2, bq = t.qe / rho2, br = t.qo / rho2, bx = t.qeo / rho2;
                t.raw_upper = orc_subspace_upper(ba, bb, bq, br, bx, 1.0) + 1e-6 + alias_mass;
                double upper = t.raw_upper + dlm;
                upper_l[lane] = jv[lane] < nb ? upper : NEG_INF;
            }
            double tile_max = NEG_INF;
            for (int l = 0; l < EV_TILE; l++)
                if (upper_l[l] > tile_max) tile_max = upper_l[l];
            for (int lane = 0; lane < EV_TILE; lane++) {
                Tmp& t = T[lane];
                JointLane& s = L[lane];
                double ba = t.ae / rho2, bb = t.ao / rho2, bq = t.qe / rho2, br = t.qo / rho2, bx = t.qeo / rho2;
                if (tile_max >= floor_b) {
                    for (int ri = 0; ri < 7; ri++) {
                        double ratio = E.params[21 + ri];
                        double aa = ba + ratio * bb;
                        double qq = bq + 2.0 * ratio * bx + ratio * ratio * br;
                        double diluted = orc_positive_amplitude_evidence(aa, qq, tau_d);
                        double eb = orc_log_add(orc_positive_amplitude_evidence(aa, qq, tau_b), diluted) + alias_mass +
                                    std::log(0.25 / 7.0);
                        t.lb = orc_log_add(t.lb, eb);
                        if (eb > t.component_best) {
                            t.sec_ratio = 0.0;
                            t.sec_phase = 0.5;
                            t.odd_ratio = ratio;
                            t.binary_multiple = 2.0;
                            t.component_best = eb;
                        }
                    }
                } else {
                    s.omitted += 1;
                    if (t.raw_upper > t.omitted_upper) t.omitted_upper = t.raw_upper;
                }
                bool certain = t.component_best > t.omitted_upper;
                if (!certain) {
                    t.sec_ratio = t.sec_phase = t.odd_ratio = t.binary_multiple = std::nan("");
                }
                t.lp += E.priors[si * 2] + dlm;
                t.lb += E.priors[si * 2 + 1] + dlm;
                if (jv[lane] < nb) {
                    s.sum_p = orc_log_add(s.sum_p, t.lp);
                    s.sum_b = orc_log_add(s.sum_b, t.lb);
                }
                double joint = t.lp;
                uint64_t key = (uint64_t)(si * nd + di) * nb + jjv[lane];
                bool bj = t.valid && (joint > s.best_joint || (joint == s.best_joint && key < s.joint_key));
                bool bs = t.valid && (t.snr > s.best_signal || (t.snr == s.best_signal && key < s.signal_key));
                double vals[9] = {t.snr, t.depth, t.lp, t.lb, t.sec_ratio, t.sec_phase, t.odd_ratio, t.binary_multiple, joint};
                if (bj) {
                    std::memcpy(s.j_out, vals, sizeof(vals));
                    s.best_joint = joint;
                    s.joint_key = key;
                }
                if (bs) {
                    std::memcpy(s.s_out, vals, sizeof(vals));
                    s.best_signal = t.snr;
                    s.signal_key = key;
                }
            }
        }
    }
    for (int selection = 0; selection < 2; selection++) {
        double maximum = NEG_INF;
        for (int l = 0; l < EV_TILE; l++) {
            double v = selection == 0 ? L[l].best_joint : L[l].best_signal;
            if (v > maximum) maximum = v;
        }
        uint64_t best_key = KEY_MAX;
        int chosen = EV_TILE;
        for (int l = 0; l < EV_TILE; l++) {
            double v = selection == 0 ? L[l].best_joint : L[l].best_signal;
            uint64_t k = selection == 0 ? L[l].joint_key : L[l].signal_key;
            if (v == maximum && k < best_key) {
                best_key = k;
                chosen = l;
            }
        }
        double high = NEG_INF;
        for (int l = 0; l < EV_TILE; l++) {
            double v = selection == 0 ? L[l].sum_p : L[l].sum_b;
            if (v > high) high = v;
        }
        double log_sum = high;
        if (high > NEG_INF) {
            double acc = 0.0;
            for (int l = 0; l < EV_TILE; l++) acc += std::exp((selection == 0 ? L[l].sum_p : L[l].sum_b) - high);
            log_sum = high + std::log(acc);
        }
        int wl = std::min(chosen, EV_TILE - 1);
        const JointLane& s = L[wl];
        const double* vals = selection == 0 ? s.j_out : s.s_out;
        double* out = &parts[((size_t)tile * 2 + selection) * PART];
        out[0] = (double)best_key;
        out[1] = maximum;
        out[2] = selection == 0 ? vals[0] : s.best_signal;
        out[3] = vals[1];
        for (int i = 0; i < 6; i++) out[4 + i] = vals[2 + i];
        out[10] = selection == 0 ? s.best_joint : vals[8];
        out[13] = (double)s.omitted;
        out[11 + selection] = log_sum;
    }
    double* out0 = &parts[(size_t)tile * 2 * PART];
    double sp = out0[11];
    double sb = out0[PART + 12];
    out0[12] = sb;
    out0[PART + 11] = sp;
}

void evidence_parameters(const double* cfg, double* p) {
    // cfg: target_flux_fraction, planet_depth_scale, binary_depth_scale,
    // diluted_binary_depth_scale, planet_prior, binary_prior,
    // stellar_radius_solar (NaN = none), planet_radius_scale_rj.
    double dilution = cfg[0];
    double planet_scale = cfg[1];
    if (!std::isnan(cfg[6])) {
        double x = 0.10045 * cfg[7] / cfg[6];
        planet_scale = x * x;
    }
    p[0] = planet_scale * dilution;
    p[1] = cfg[2] * dilution;
    p[2] = cfg[3];
    p[3] = std::log(cfg[4]);
    p[4] = std::log(cfg[5]);
    p[5] = std::log(1.0 - cfg[4] - cfg[5]);
    const double ratios[5] = {0.0, 0.01, 0.1, 0.5, 1.0};
    const double wp[5] = {0.75, 0.15, 0.08, 0.015, 0.005};
    const double wb[5] = {0.10, 0.10, 0.20, 0.25, 0.35};
    for (int i = 0; i < 5; i++) {
        p[6 + 3 * i] = ratios[i];
        p[7 + 3 * i] = wp[i];
        p[8 + 3 * i] = wb[i];
    }
    const double odd[7] = {0.25, 0.5, 0.75, 1.0, 4.0 / 3.0, 2.0, 4.0};
    for (int i = 0; i < 7; i++) p[21 + i] = odd[i];
    p[28] = 0.001;
    p[29] = 0.05;
}

}  // namespace

extern "C" void orc_evidence_parameters(const double* cfg, double* p) { evidence_parameters(cfg, p); }

// compare_search (evidence.rs:693-1003) for one family state and one trial
// period. durations/rho are the family's (any order). cfg holds the 8 values
// of evidence_parameters followed by threshold, evidence_rtol,
// phase_oversample, shape_layers. rows_out: up to 2 rows of 14 values
// (period, epoch, duration, snr, depth, planet_log_odds, log_bf_planet_noise,
// log_bf_binary_noise, binary_secondary_ratio, binary_secondary_phase,
// binary_odd_even_ratio, binary_period_days, ingress_fraction,
// selection_flags). Returns the row count (0, 1 or 2). diag (optional, 8
// values): nb, nd, tiles, screen maximum, pilot key, floor_p, floor_b,
// log_mass.
extern "C" int orc_compare_search(const double* time, const double* v, const double* w, int64_t n,
                                  double baseline_norm, double origin, double residual_energy,
                                  const double* durations_in, const double* rho_in, int nd_in, const double* ingress,
                                  int ns, double period, const double* cfg, double* rows_out, double* diag) {
    std::vector<std::pair<double, double>> ds;
    for (int i = 0; i < nd_in; i++)
        if (durations_in[i] < period / 4.0) ds.push_back({durations_in[i], rho_in[i]});
    std::stable_sort(ds.begin(), ds.end(), [](auto& a, auto& b) { return a.first < b.first; });
    if (ds.empty()) return 0;
    int nd = (int)ds.size();
    std::vector<double> durations(nd), rho(nd);
    for (int i = 0; i < nd; i++) {
        durations[i] = ds[i].first;
        rho[i] = ds[i].second;
    }
    double threshold = cfg[8], rtol = cfg[9];
    int phase_oversample = (int)cfg[10];
    int layers = (int)cfg[11];
    double dmin = durations[0];
    size_t nb = 4 * as_usize(std::ceil((double)phase_oversample * period / dmin / 4.0));
    if (nb < 8) nb = 8;
    size_t nb2 = 2 * nb;
    double scale = (double)nb / period;
    std::vector<double> dlm(nd);
    for (int i = 0; i < nd; i++) {
        double r = rho[i];
        dlm[i] = -0.5 * (((double)n - 1.0) * std::log(r * r) + residual_energy / (r * r));
    }
    double dmax = NEG_INF;
    for (double x : dlm) dmax = rmax(dmax, x);
    for (double& x : dlm) x -= dmax;
    std::vector<double> lpl(ns), lbl(ns);
    for (int s = 0; s < ns; s++) {
        lpl[s] = -4.0 * ingress[s];
        lbl[s] = 2.0 * ingress[s];
    }
    double lp0 = logsumexp(lpl), lb0 = logsumexp(lbl);
    std::vector<double> priors(2 * ns);
    for (int s = 0; s < ns; s++) {
        priors[2 * s] = lpl[s] - lp0;
        priors[2 * s + 1] = lbl[s] - lb0;
    }
    std::vector<double> shapes;
    for (int s = 0; s < ns; s++) {
        double previous = 0.0;
        for (int layer = 0; layer < layers; layer++) {
            double fraction = 1.0 - 2.0 * ingress[s] * (double)layer / (double)(std::max(layers, 2) - 1);
            double inc = 1.0 / (double)layers;
            shapes.push_back(fraction);
            shapes.push_back(inc);
            shapes.push_back(inc * (2.0 * previous + inc));
            previous += inc;
        }
    }
    double params[NPARAM];
    evidence_parameters(cfg, params);
    const double phases[3] = {0.25, 0.5, 0.75};
    const double logw[3] = {std::log(0.1), std::log(0.8), std::log(0.1)};
    std::vector<double> lp_bank((size_t)nd * NORB, NEG_INF), lb_bank((size_t)nd * NORB, NEG_INF);
    size_t valid_count = 0;
    for (int di = 0; di < nd; di++) {
        double k = rmax(std::floor(durations[di] * scale + 0.5), 1.0);
        if (k < (double)(nb / 4)) valid_count++;
        for (int o = 0; o < NORB; o++) {
            double ks = rmax(std::floor(k + 0.5), 1.0);
            double shift = std::floor(phases[o] * (double)nb + 0.5);
            double start = shift + std::floor((k - ks) / 2.0);
            bool valid = k < (double)(nb / 4) && ks < (double)(nb / 2) && start >= k && start + ks <= (double)nb;
            if (valid) {
                lp_bank[(size_t)di * NORB + o] = logw[o];
                lb_bank[(size_t)di * NORB + o] = logw[o];
            }
        }
    }
    double count = std::log((double)valid_count);
    double norm_p = count - logsumexp(lp_bank);
    double norm_b = count - logsumexp(lb_bank);
    std::vector<double> orbit;
    for (int di = 0; di < nd; di++)
        for (int o = 0; o < NORB; o++) {
            orbit.push_back(phases[o]);
            orbit.push_back(1.0);
            orbit.push_back(lp_bank[(size_t)di * NORB + o] + norm_p);
            orbit.push_back(lb_bank[(size_t)di * NORB + o] + norm_b);
        }
    // fold_two + prefix_fields (sequential order).
    std::vector<double> folded(3 * nb2, 0.0);
    for (int64_t i = 0; i < n; i++) {
        int64_t cell64 = as_i64(std::floor(time[i] * scale));
        int64_t m = (int64_t)nb2;
        int64_t cell = ((cell64 % m) + m) % m;
        folded[0 * nb2 + cell] += v[i];
        folded[1 * nb2 + cell] += w[i];
        folded[2 * nb2 + cell] += 1.0;
    }
    // prefix_fields (evidence.rs:96-144): per segment of 256 bins a block-wide
    // Hillis-Steele scan (stride 1 .. 128), plus the running carry.
    std::vector<double> cum(3 * (nb2 + 1), 0.0);
    for (int f = 0; f < 3; f++) {
        double* row = &cum[(size_t)f * (nb2 + 1)];
        row[0] = 0.0;
        double carry = 0.0;
        for (size_t seg = 0; seg < nb2; seg += 256) {
            double scan[256], prev[256];
            for (int l = 0; l < 256; l++) scan[l] = seg + l < nb2 ? folded[f * nb2 + seg + l] : 0.0;
            for (int stride = 1; stride < 256; stride <<= 1) {
                std::memcpy(prev, scan, sizeof(prev));
                for (int l = stride; l < 256; l++) scan[l] = prev[l] + prev[l - stride];
            }
            for (int l = 0; l < 256; l++)
                if (seg + l < nb2) row[seg + l + 1] = scan[l] + carry;
            carry += scan[255];
        }
    }
    EvidenceInputs E{cum.data(), scale, durations.data(), rho.data(), dlm.data(), shapes.data(), priors.data(), params,
                     orbit.data(), baseline_norm, threshold, (double)n, nb2, nd, ns, layers};
    int tiles = (int)((nb + EV_TILE - 1) / EV_TILE);
    std::vector<double> screen((size_t)tiles * 4, 0.0);
    for (int t = 0; t < tiles; t++) comparison_screen_tile(E, t, screen.data());
    double maximum = NEG_INF;
    for (int t = 0; t < tiles; t++) maximum = rmax(maximum, screen[(size_t)t * 4]);
    if (diag) {
        diag[0] = (double)nb;
        diag[1] = nd;
        diag[2] = tiles;
        diag[3] = maximum;
    }
    if (!(maximum >= threshold * (1.0 - 1e-12))) return 0;
    // Iterator::max_by keeps the last maximum.
    int winner = 0;
    for (int t = 1; t < tiles; t++)
        if (screen[(size_t)t * 4 + 1] >= screen[(size_t)winner * 4 + 1]) winner = t;
    double pilot_key = screen[(size_t)winner * 4 + 3];
    double margin = rtol > 0.0 ? std::log(rtol) - std::log((double)((NORB + 1) * nb * nd * ns)) : NEG_INF;
    std::vector<double> parts((size_t)tiles * 2 * PART, 0.0);
    double floors0[3] = {NEG_INF, NEG_INF, pilot_key};
    joint_tile(E, 0, true, floors0, parts.data());
    double floors[3] = {parts[11] + margin, parts[12] + margin, pilot_key};
    for (int t = 0; t < tiles; t++) joint_tile(E, t, false, floors, parts.data());
    if (diag) {
        diag[4] = pilot_key;
        diag[5] = floors[0];
        diag[6] = floors[1];
    }
    std::vector<double> in_bank_dlm;
    for (int i = 0; i < nd; i++)
        if (rmax(std::floor(durations[i] * scale + 0.5), 1.0) < (double)(nb / 4)) in_bank_dlm.push_back(dlm[i]);
    double log_mass = std::log((double)nb) + logsumexp(in_bank_dlm);
    if (diag) diag[7] = log_mass;
    double rows[2][14];
    for (int selection = 0; selection < 2; selection++) {
        auto value = [&](int t, int i) { return parts[((size_t)t * 2 + selection) * PART + i]; };
        double mx = NEG_INF;
        for (int t = 0; t < tiles; t++) mx = rmax(mx, value(t, 1));
        double key = std::numeric_limits<double>::infinity();
        for (int t = 0; t < tiles; t++)
            if (value(t, 1) == mx) key = rmin(key, value(t, 0));
        int tile = 0;
        for (int t = 0; t < tiles; t++)
            if (value(t, 1) == mx && value(t, 0) == key) {
                tile = t;
                break;
            }
        std::vector<double> s11(tiles), s12(tiles);
        for (int t = 0; t < tiles; t++) {
            s11[t] = value(t, 11);
            s12[t] = value(t, 12);
        }
        double lp = logsumexp(s11) - log_mass;
        double lb = logsumexp(s12) - log_mass;
        double joint = params[3] + lp - orc_log_add(params[5], params[4] + lb);
        uint64_t decoded = mx > NEG_INF ? as_usize(key) : 0;
        size_t j = (size_t)(decoded % nb);
        size_t di = (size_t)((decoded / nb) % (uint64_t)nd);
        size_t si = (size_t)(decoded / ((uint64_t)nb * (uint64_t)nd));
        double width = rmax(std::floor(durations[di] * scale + 0.5), 1.0);
        double snr = mx > NEG_INF ? value(tile, 2) : NEG_INF;
        double* r = rows[selection];
        r[0] = period;
        r[1] = ((double)j + width / 2.0) / scale + origin;
        r[2] = width / scale;
        r[3] = snr;
        r[4] = value(tile, 3);
        r[5] = joint;
        r[6] = lp;
        r[7] = lb;
        r[8] = value(tile, 6);
        r[9] = value(tile, 7);
        r[10] = value(tile, 8);
        r[11] = value(tile, 9) * period;
        r[12] = ingress[std::min(si, (size_t)(ns - 1))];
        r[13] = selection == 0 ? 1.0 : 2.0;
    }
    bool hit0 = std::isfinite(rows[0][3]), hit1 = std::isfinite(rows[1][3]);
    bool same = hit0 && hit1 && rows[0][0] == rows[1][0] && rows[0][1] == rows[1][1] && rows[0][2] == rows[1][2] &&
                rows[0][3] == rows[1][3] && rows[0][4] == rows[1][4] && rows[0][12] == rows[1][12];
    int count_out = 0;
    if (hit0) {
        std::memcpy(rows_out + 14 * count_out, rows[0], sizeof(rows[0]));
        if (same) rows_out[14 * count_out + 13] = 3.0;
        count_out++;
    }
    if (hit1 && !same) {
        std::memcpy(rows_out + 14 * count_out, rows[1], sizeof(rows[1]));
        count_out++;
    }
    return count_out;
}
