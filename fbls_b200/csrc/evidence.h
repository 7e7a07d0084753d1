// Joint planet / binary / noise evidence at one trial period (internal).
#pragma once

#include <cstddef>
#include <cstdint>
#include <functional>
#include <string>

#include <cuda_runtime.h>

#include "../../include/fbls_b200.h"

namespace fbls {

struct EvidenceReady {
    const double* time;  // device, n
    const double* v;     // device, n
    const double* w;     // device, n
    uint32_t n;
    double baseline_norm;
    double origin;
    double residual_energy;
    double t_last;            // last relative time
    const double* time_host;  // host copy of time (fold chunk boundaries)
};

// compare_search (src/search/evidence.rs:693-1003). `workspace(bytes)`
// returns a device buffer of at least that many bytes (or null). Returns 0
// or an FBLS_ERR_* status with `message` set.
int compare_search(cudaStream_t stream, void* ws_ptr, size_t ws_bytes, const EvidenceReady& r,
                   const double* durations, const double* rho, uint32_t nd, double period, const fbls_config& cfg,
                   fbls_evidence_row* rows_out, uint32_t* n_rows, std::string& message,
                   const std::function<void*(size_t)>& workspace);

// parameters() (evidence.rs:665-689): 30 values.
void evidence_parameters(const fbls_config& cfg, double* p);

}  // namespace fbls
