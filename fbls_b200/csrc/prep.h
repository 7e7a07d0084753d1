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

// period_grid (src/search/grid.rs:5-28).
int64_t period_grid(double minimum, double maximum, double baseline, double minimum_duration, double oversample,
                    double* out, int64_t capacity);

}  // namespace fbls
