// Host-side preparation of a prepared-mode family (internal to the library).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace fbls {

struct PreparedFamily {
    std::vector<double> time;  // relative to origin, ascending
    std::vector<double> v;
    std::vector<double> w;
    std::vector<double> rho;   // per duration, in the order given
    double baseline_norm = 0.0;
    double origin = 0.0;
    double residual_energy = 0.0;
    double inflation = 1.0;
    size_t segments = 0;
};

// family_state of a prepared curve (src/prep/curve.rs:541-569). Returns 0, or
// 1 with the reference's message in `error`.
int prepare_family(const double* time, const double* flux, const double* sigma, size_t n_in, const double* durations,
                   size_t nd, bool correlated, PreparedFamily& out, std::string& error);

// The diagonal noise model of raw mission flux (DiagonalNoise, fit_segment_noise
// src/prep/curve.rs:89-198): each group (sector) normalised by its lower
// median, times relative to the first, optional inverse-variance bins of
// bin_minutes per (bin, group), inflation from the adjacent differences, and
// with no errors given a white level from the differences' scatter.
struct DiagonalNoise {
    std::vector<double> time;      // relative to origin, ascending
    std::vector<double> deficit;   // -(flux / median - 1)
    std::vector<double> variance;
    std::vector<int64_t> group;
    double origin = 0.0;
    double inflation = 1.0;
    size_t segments = 0;
};
// err and group may be null (unit errors, one group). Returns 0, or 1 with
// the reference's message in `error`.
int fit_segment_noise(const double* time, const double* flux, const double* err, const int64_t* group, size_t n_in,
                      double bin_minutes, double gap_days, DiagonalNoise& out, std::string& error);

// Distance of every observation to the nearer edge of its gap-separated
// segment (segment_edges, curve.rs:332-345).
std::vector<double> segment_edges(const std::vector<double>& time, double gap);

// Durations grouped by detrending window clamp(factor D, minimum, maximum)
// rounded to 1e-6 d, sorted by window (detrending_windows, curve.rs:349-370).
std::vector<std::pair<double, std::vector<uint32_t>>> detrending_windows(const double* durations, size_t nd,
                                                                          double minimum, double factor,
                                                                          double maximum);

// mad_scale (src/prep/stats.rs:14-18).
double robust_scale(const std::vector<double>& values);

// period_grid (src/search/grid.rs:5-28).
int64_t period_grid(double minimum, double maximum, double baseline, double minimum_duration, double oversample,
                    double* out, int64_t capacity);

}  // namespace fbls
