// Host-side preparation of a prepared-mode family (the inputs of the search
// path): the diagonal noise model, the precision-weighted fields and the
// correlated-noise factors. C++ restatement of the reference's host code:
//   family_state              src/prep/curve.rs:541-569
//   fit_segment_noise         src/prep/curve.rs:89-198 (prepared mode: bin 0,
//                             one group; raw mode: fit_segment_noise below)
//   segment_edges, detrending_windows  src/prep/curve.rs:332-370
//   prepare_ready             src/prep/curve.rs:427-450
//   correlated_noise_factors  src/prep/curve.rs:456-539
//   median_lower, mad_scale   src/prep/stats.rs:4-18
// plus period_grid, src/search/grid.rs:5-28.
// Built with -ffp-contract=off: every operation rounds as the Rust does.
#include "prep.h"

#include <algorithm>
#include <cmath>
#include <limits>

namespace fbls {

namespace {

double fmax_rust(double a, double b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a > b ? a : b)); }

double median_lower(std::vector<double> v) {
    v.erase(std::remove_if(v.begin(), v.end(), [](double x) { return !std::isfinite(x); }), v.end());
    if (v.empty()) return std::numeric_limits<double>::quiet_NaN();
    size_t k = (v.size() - 1) / 2;
    std::nth_element(v.begin(), v.begin() + (ptrdiff_t)k, v.end());
    return v[k];
}

double mad_scale(const std::vector<double>& values) {
    double m = median_lower(values);
    std::vector<double> dev(values.size());
    for (size_t i = 0; i < values.size(); i++) dev[i] = std::fabs(values[i] - m);
    return 1.4826 * median_lower(std::move(dev));
}

// Per-duration correlated-noise factor rho_D >= 1: robust scatter of the
// standardized inverse-variance means of the residuals in contiguous time
// cells of length D, with under-sampled durations inheriting sqrt(D/D_ref)
// scaling from the nearest supported duration (curve.rs:452-539).
std::vector<double> noise_factors(const std::vector<double>& time, const std::vector<double>& residual,
                                  const std::vector<double>& sigma, const double* durations, size_t nd) {
    const double min_fill = 0.5;
    const size_t minimum_bins = 20;
    const size_t n = time.size();
    std::vector<double> weight(n);
    for (size_t i = 0; i < n; i++) weight[i] = 1.0 / (sigma[i] * sigma[i]);
    std::vector<double> steps;
    steps.reserve(n);
    for (size_t i = 1; i < n; i++) {
        double s = time[i] - time[i - 1];
        if (s > 0.0) steps.push_back(s);
    }
    const double cadence = median_lower(steps);
    std::vector<double> measured(nd);
    std::vector<size_t> cells(nd);
    for (size_t di = 0; di < nd; di++) {
        const double d = durations[di];
        std::vector<double> z;
        double total = 0.0, acc = 0.0;
        size_t count = 0;
        int64_t current = std::numeric_limits<int64_t>::min();
        for (size_t i = 0; i <= n; i++) {
            int64_t cell = current;
            if (i < n) {
                double c = std::floor((time[i] - time[0]) / d);
                cell = (int64_t)c;
            }
            if (i == n || cell != current) {
                if (count > 0 && (double)count >= min_fill * d / cadence) z.push_back((acc / total) * std::sqrt(total));
                if (i == n) break;
                current = cell;
                total = 0.0;
                acc = 0.0;
                count = 0;
            }
            total += weight[i];
            acc += weight[i] * residual[i];
            count += 1;
        }
        cells[di] = z.size();
        measured[di] = z.size() >= 3 ? fmax_rust(mad_scale(z), 1.0) : 1.0;
    }
    std::vector<size_t> supported;
    for (size_t i = 0; i < nd; i++)
        if (cells[i] >= minimum_bins) supported.push_back(i);
    std::vector<double> inherited(nd);
    if (!supported.empty()) {
        for (size_t i = 0; i < nd; i++) {
            size_t anchor = supported[0];
            double best = std::fabs(std::log(durations[i]) - std::log(durations[anchor]));
            for (size_t s = 1; s < supported.size(); s++) {
                double dist = std::fabs(std::log(durations[i]) - std::log(durations[supported[s]]));
                if (dist < best) {
                    best = dist;
                    anchor = supported[s];
                }
            }
            inherited[i] = measured[anchor] * std::sqrt(fmax_rust(durations[i] / durations[anchor], 1.0));
        }
    } else {
        std::vector<double> standardized(n);
        for (size_t i = 0; i < n; i++) standardized[i] = residual[i] / sigma[i];
        double scatter = fmax_rust(mad_scale(standardized), 1.0);
        for (size_t i = 0; i < nd; i++) inherited[i] = scatter * std::sqrt(fmax_rust(durations[i] / cadence, 1.0));
    }
    std::vector<double> out(nd);
    for (size_t i = 0; i < nd; i++)
        out[i] = cells[i] >= minimum_bins ? measured[i] : fmax_rust(measured[i], inherited[i]);
    return out;
}

}  // namespace

int prepare_family(const double* time, const double* flux, const double* sigma, size_t n_in, const double* durations,
                   size_t nd, bool correlated, PreparedFamily& out, std::string& error) {
    // Usable observations, in time order (search_prepared, pipeline.rs:46-58).
    std::vector<size_t> keep;
    keep.reserve(n_in);
    for (size_t i = 0; i < n_in; i++)
        if (std::isfinite(time[i]) && std::isfinite(flux[i]) && std::isfinite(sigma[i]) && sigma[i] > 0.0)
            keep.push_back(i);
    std::stable_sort(keep.begin(), keep.end(), [&](size_t a, size_t b) { return time[a] < time[b]; });
    const size_t n = keep.size();
    if (n < 6) {
        error = "insufficient usable observations";
        return 1;
    }
    // Noise model of 1 + flux (family_state, curve.rs:547-548).
    std::vector<double> t(n), f(n), e(n);
    for (size_t i = 0; i < n; i++) {
        t[i] = time[keep[i]];
        f[i] = 1.0 + flux[keep[i]];
        e[i] = sigma[keep[i]];
    }
    const double m = median_lower(f);
    if (!(m > 0.0)) {
        error = "mission flux must have a positive median";
        return 1;
    }
    for (size_t i = 0; i < n; i++) {
        f[i] = f[i] / m - 1.0;
        e[i] /= m;
    }
    const double origin = t[0];
    for (size_t i = 0; i < n; i++) t[i] -= origin;
    const double gap = 0.75;
    std::vector<double> standardized;
    standardized.reserve(n);
    for (size_t i = 1; i < n; i++)
        if (t[i] - t[i - 1] < gap) standardized.push_back((f[i] - f[i - 1]) / std::sqrt(e[i] * e[i] + e[i - 1] * e[i - 1]));
    if (standardized.empty()) {
        error = "no adjacent observations available for noise estimation";
        return 1;
    }
    const double inflation = fmax_rust(mad_scale(standardized), 1.0);
    size_t segments = 1;
    for (size_t i = 1; i < n; i++)
        if (t[i] - t[i - 1] > gap) segments++;
    std::vector<double> variance(n), deficit(n);
    for (size_t i = 0; i < n; i++) {
        double x = e[i] * inflation;
        variance[i] = x * x;
        deficit[i] = -f[i];
    }
    // Precision-weighted fields (prepare_ready, curve.rs:427-450).
    std::vector<double> p(n);
    double c = 0.0;
    for (size_t i = 0; i < n; i++) {
        p[i] = 1.0 / variance[i];
        c += p[i];
    }
    if (!(std::isfinite(c) && c > 0.0)) {
        error = "invalid baseline precision";
        return 1;
    }
    double spy = 0.0;
    for (size_t i = 0; i < n; i++) spy += p[i] * deficit[i];
    const double mean = spy / c;
    out.time = t;
    out.v.resize(n);
    out.w = p;
    double energy = 0.0;
    for (size_t i = 0; i < n; i++) {
        out.v[i] = p[i] * deficit[i] - p[i] * mean;
        energy += deficit[i] * out.v[i];
    }
    out.baseline_norm = c;
    out.origin = origin;
    out.residual_energy = energy;
    out.inflation = inflation;
    out.segments = segments;
    if (correlated) {
        std::vector<double> resid(n), sig(n);
        for (size_t i = 0; i < n; i++) {
            resid[i] = -deficit[i];
            sig[i] = std::sqrt(variance[i]);
        }
        out.rho = noise_factors(t, resid, sig, durations, nd);
    } else {
        out.rho.assign(nd, 1.0);
    }
    return 0;
}

int fit_segment_noise(const double* time, const double* flux, const double* err, const int64_t* group, size_t n_in,
                      double bin_minutes, double gap_days, DiagonalNoise& out, std::string& error) {
    auto e_in = [&](size_t i) { return err ? err[i] : 1.0; };
    auto g_in = [&](size_t i) { return group ? group[i] : (int64_t)0; };
    std::vector<size_t> keep;
    for (size_t i = 0; i < n_in; i++)
        if (std::isfinite(time[i]) && std::isfinite(flux[i]) && std::isfinite(e_in(i)) && e_in(i) > 0.0)
            keep.push_back(i);
    std::stable_sort(keep.begin(), keep.end(), [&](size_t a, size_t b) { return time[a] < time[b]; });
    size_t n = keep.size();
    std::vector<double> t(n), f(n), e(n);
    std::vector<int64_t> sec(n);
    for (size_t i = 0; i < n; i++) {
        t[i] = time[keep[i]];
        f[i] = flux[keep[i]];
        e[i] = e_in(keep[i]);
        sec[i] = g_in(keep[i]);
    }
    if (n < 6) {
        error = "insufficient usable observations";
        return 1;
    }
    std::vector<int64_t> labels = sec;
    std::sort(labels.begin(), labels.end());
    labels.erase(std::unique(labels.begin(), labels.end()), labels.end());
    for (int64_t label : labels) {
        std::vector<double> vals;
        for (size_t i = 0; i < n; i++)
            if (sec[i] == label) vals.push_back(f[i]);
        const double m = median_lower(vals);
        if (!(m > 0.0)) {
            error = "mission flux must have a positive median";
            return 1;
        }
        for (size_t i = 0; i < n; i++)
            if (sec[i] == label) {
                f[i] = f[i] / m - 1.0;
                e[i] /= m;
            }
    }
    const double origin = t[0];
    for (size_t i = 0; i < n; i++) t[i] -= origin;
    if (bin_minutes > 0.0) {
        // Inverse-variance means per (bin, group), keys in sorted order.
        const double width = bin_minutes / 1440.0;
        std::vector<std::pair<int64_t, int64_t>> keys(n);
        for (size_t i = 0; i < n; i++) keys[i] = {(int64_t)std::floor(t[i] / width), sec[i]};
        std::vector<std::pair<int64_t, int64_t>> unique = keys;
        std::sort(unique.begin(), unique.end());
        unique.erase(std::unique(unique.begin(), unique.end()), unique.end());
        const size_t m = unique.size();
        std::vector<double> den(m, 0.0), st(m, 0.0), sf(m, 0.0);
        for (size_t i = 0; i < n; i++) {
            const size_t k = (size_t)(std::lower_bound(unique.begin(), unique.end(), keys[i]) - unique.begin());
            const double w = 1.0 / (e[i] * e[i]);
            den[k] += w;
            st[k] += t[i] * w;
            sf[k] += f[i] * w;
        }
        std::vector<double> tb(m), fb(m), eb(m);
        std::vector<int64_t> sb(m);
        for (size_t k = 0; k < m; k++) {
            tb[k] = st[k] / den[k];
            fb[k] = sf[k] / den[k];
            eb[k] = 1.0 / std::sqrt(den[k]);
            sb[k] = unique[k].second;
        }
        std::vector<size_t> order(m);
        for (size_t k = 0; k < m; k++) order[k] = k;
        std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return tb[a] < tb[b]; });
        t.resize(m);
        f.resize(m);
        e.resize(m);
        sec.resize(m);
        for (size_t k = 0; k < m; k++) {
            t[k] = tb[order[k]];
            f[k] = fb[order[k]];
            e[k] = eb[order[k]];
            sec[k] = sb[order[k]];
        }
        n = m;
    }
    std::vector<double> standardized, deltas;
    for (size_t i = 1; i < n; i++)
        if (t[i] - t[i - 1] < gap_days && sec[i] == sec[i - 1]) {
            const double d = f[i] - f[i - 1];
            deltas.push_back(d);
            standardized.push_back(d / std::sqrt(e[i] * e[i] + e[i - 1] * e[i - 1]));
        }
    if (deltas.empty()) {
        error = "no adjacent observations available for noise estimation";
        return 1;
    }
    const double inflation = fmax_rust(mad_scale(standardized), 1.0);
    out.variance.resize(n);
    if (err) {
        for (size_t i = 0; i < n; i++) {
            const double x = e[i] * inflation;
            out.variance[i] = x * x;
        }
    } else {
        const double m = median_lower(deltas);
        std::vector<double> dev(deltas.size());
        for (size_t i = 0; i < deltas.size(); i++) dev[i] = std::fabs(deltas[i] - m);
        const double white = fmax_rust(1.4826 / std::sqrt(2.0) * median_lower(dev), 1e-12);
        for (size_t i = 0; i < n; i++) out.variance[i] = white * white;
    }
    size_t segments = 1;
    for (size_t i = 1; i < n; i++)
        if (t[i] - t[i - 1] > gap_days || sec[i] != sec[i - 1]) segments++;
    out.time = t;
    out.deficit.resize(n);
    for (size_t i = 0; i < n; i++) out.deficit[i] = -f[i];
    out.group = sec;
    out.origin = origin;
    out.inflation = inflation;
    out.segments = segments;
    return 0;
}

std::vector<double> segment_edges(const std::vector<double>& time, double gap) {
    const size_t n = time.size();
    std::vector<double> out(n, 0.0);
    size_t start = 0;
    for (size_t i = 1; i <= n; i++)
        if (i == n || time[i] - time[i - 1] > gap) {
            for (size_t j = start; j < i; j++) {
                const double a = time[j] - time[start], b = time[i - 1] - time[j];
                out[j] = std::isnan(a) ? b : (std::isnan(b) ? a : (a < b ? a : b));
            }
            start = i;
        }
    return out;
}

std::vector<std::pair<double, std::vector<uint32_t>>> detrending_windows(const double* durations, size_t nd,
                                                                          double minimum, double factor,
                                                                          double maximum) {
    std::vector<double> windows(nd);
    for (size_t i = 0; i < nd; i++) {
        double x = factor * durations[i];
        if (x < minimum) x = minimum;  // f64::clamp
        if (x > maximum) x = maximum;
        windows[i] = std::round(x * 1e6) / 1e6;  // f64::round: halves away from zero
    }
    std::vector<double> uniq = windows;
    std::sort(uniq.begin(), uniq.end());
    uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
    std::vector<std::pair<double, std::vector<uint32_t>>> out;
    for (double w : uniq) {
        std::vector<uint32_t> idx;
        for (size_t i = 0; i < nd; i++)
            if (windows[i] == w) idx.push_back((uint32_t)i);
        out.push_back({w, idx});
    }
    return out;
}

double robust_scale(const std::vector<double>& values) { return mad_scale(values); }

int64_t period_grid(double minimum, double maximum, double baseline, double minimum_duration, double oversample,
                    double* out, int64_t capacity) {
    const double log_step = std::log1p(minimum_duration / (oversample * baseline));
    const double c = std::ceil(std::log(maximum / minimum) / log_step);
    // An infinite quotient (a zero minimum or a zero step) saturates the
    // reference's count (grid.rs:12), which then fails to allocate or index
    // the grid; such grids, and any above 2^53 periods, are refused here.
    // A NaN or negative quotient gives one period, as there.
    if (c >= 9007199254740992.0) return -1;
    const int64_t count = (c > 0.0 ? (int64_t)c : 0) + 1;
    if (out == nullptr || capacity < count) return count;
    const double a = std::log(minimum), b = std::log(maximum);
    for (int64_t i = 0; i < count; i++) out[i] = std::exp(count == 1 ? a : a + (b - a) * (double)i / (double)(count - 1));
    out[0] = minimum;
    out[count - 1] = maximum;
    return count;
}

}  // namespace fbls
