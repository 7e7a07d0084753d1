// Joint planet / binary / noise evidence (internal): compare_search over a
// batch of candidates, each one trial period of one prepared family.
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

// One candidate: a family, its durations and correlated-noise factors (host,
// any order, nd of them) and the trial period. Outputs: rows (0, 1 or 2),
// their count and the candidate's status (0 or FBLS_ERR_*; message when set).
struct EvidenceCandidate {
    EvidenceReady r;
    const double* durations;
    const double* rho;
    uint32_t nd;
    double period;
    fbls_evidence_row rows[2];
    uint32_t n_rows;
    int status;
    std::string message;
};

// compare_search (src/search/evidence.rs:693-1003) for every candidate, on
// `stream`: host plans, one upload, the folds, prefix sums, screens, pilots
// and joint tiles of all candidates as shared launches, one download and one
// synchronisation. `workspace(bytes)` returns a device buffer of at least
// that many bytes (or null). Returns 0 when every planned candidate ran (a
// candidate the planner rejects gets its own status and is skipped), or an
// FBLS_ERR_* status of the whole batch with `message` set. `launches`, when
// given, counts the kernels launched.
int compare_batch(cudaStream_t stream, EvidenceCandidate* cands, size_t count, const fbls_config& cfg,
                  std::string& message, const std::function<void*(size_t)>& workspace, int sm_count,
                  uint64_t* launches = nullptr);

// parameters() (evidence.rs:665-689): 30 values.
void evidence_parameters(const fbls_config& cfg, double* p);

}  // namespace fbls
