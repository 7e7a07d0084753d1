// Launch interfaces of the FBLS device kernels (internal to the library).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace fbls {

constexpr int FOLD_THREADS = 512;
constexpr int MAX_GROUP = 32;               // periods per fold CTA
constexpr size_t MAX_FOLD_SMEM = 225 * 1024;  // dynamic shared memory of k_fold_prefix
constexpr int GLOBAL_FOLD_PERIODS = 4;
constexpr int MAX_DURATIONS = 64;
constexpr int MAX_SHAPES = 8;
constexpr int MAX_LAYERS = 16;

// Bytes of shared memory one period's histogram needs (f64 v, f64 w, u32 count).
constexpr size_t fold_bytes_per_bin = 2 * sizeof(double) + sizeof(uint32_t);

struct FoldArgs {
    const double* time;    // n, relative days, ascending
    const double* v;       // n
    const double* w;       // n
    const double* scales;  // periods: nb / period
    int n;
    int nb;
    int periods;
    int group;             // periods per CTA (shared-memory path)
    double* cum;           // periods x NF x (2nb+1)
    float2* cum32;         // periods x NF x (2nb+1) (hi, lo)
};

struct ScanArgs {
    const double* cum;
    const float2* cum32;
    const double* scales;
    const double* durations;  // nd, ascending
    const double* rho;        // nd
    const double* ingress;    // ns
    const double* factors;    // ns x layers
    double baseline;          // baseline_norm c
    double gate;              // shape gate (score units)
    double n;                 // observation count
    int nb, nd, ns, layers;
    int mixed;                // 1 = f32 pre-rank + f64 rescans, 0 = f64 only
    double* parts;            // periods x tiles x 9
    uint64_t* keys;           // periods x tiles
    uint32_t* flags;          // periods x tiles
};

struct MergeArgs {
    const double* parts;
    const uint64_t* keys;
    const uint32_t* flags;
    const double* periods_in;
    const double* scales;
    int periods;
    int tiles;
    int offset;        // first output row
    double* records;   // rows x 9
    double* score;
    double* depth;
    uint32_t* flags_out;
};

cudaError_t launch_fold_prefix(const FoldArgs& a, size_t smem_bytes, cudaStream_t stream);
cudaError_t launch_fold_global(const FoldArgs& a, double* hist, cudaStream_t stream);
cudaError_t launch_scan_tiles(const ScanArgs& a, int periods, cudaStream_t stream);
cudaError_t launch_merge(const MergeArgs& a, cudaStream_t stream);

}  // namespace fbls
