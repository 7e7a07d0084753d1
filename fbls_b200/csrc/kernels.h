// Launch interfaces of the FBLS device kernels (internal to the library).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include <vector>

namespace fbls {

constexpr int MAX_GROUP = 32;               // periods per fold CTA (the built-in rule's largest group)
constexpr int WALK_MAX_GROUP = 128;         // periods per walking-fold CTA (tuned group caps)
constexpr int WALK_MIN_LANES = 8;           // lanes per period of a walking-fold CTA at least
constexpr size_t MAX_FOLD_SMEM = 225 * 1024;  // dynamic shared memory of k_fold
constexpr int MAX_DURATIONS = 64;
constexpr int MAX_SHAPES = 8;
constexpr int MAX_LAYERS = 16;

// Bytes of shared memory one period's histogram needs (f64 v, f64 w, u32 count).
constexpr size_t fold_bytes_per_bin = 2 * sizeof(double) + sizeof(uint32_t);

// Fold kernels: TMA-staged walk with shared-memory histograms (FOLD_WALK),
// or the staged-by-threads fold that can also keep its histograms in global
// scratch, for nb too large for the first (FOLD_SMEM).
constexpr int FOLD_SMEM = 0;
constexpr int FOLD_WALK = 2;

// Device copies of the observations: time, v and w at a stride of
// fold_field_stride(n) doubles, so each field starts on a 16-byte boundary
// and has one readable slot past its end (the fold's bulk copies round a
// chunk out to whole 16-byte pieces).
inline size_t fold_field_stride(size_t n) { return (n + 2) & ~(size_t)1; }

struct ScanArgs;
struct MergeArgs;

struct FoldArgs {
    const double* time;    // n, relative days, ascending
    const double* v;       // n
    const double* w;       // n
    const double* scales;  // periods: nb / period
    int n;
    int nb;
    int periods;
    int group;             // periods per CTA
    double* cum;           // periods x NF x (2nb+1)
    float2* cum32;         // periods x NF x (2nb+1) (hi, lo)
    double* hist_global;   // null: histograms in shared memory; else 3 G nb doubles per CTA
    double* hist_out;      // non-null (one period): write the raw histogram [3][nb], no prefix
    const int* chunks;     // nchunks + 1 observation offsets (fold_chunks)
    int nchunks;
    int stage_field;       // staged slots per field (FoldShape::stage_field)
    int window;            // 0: whole histogram in shared memory; else window rows
    int row_stride;        // FoldShape::row_stride
    uint32_t* fault;       // FOLD_WALK: set nonzero when a staging wait gives up
    int rows32_only;       // FOLD_WALK: write only the (hi, lo) f32 rows (the f32 form reads no f64 rows)
    int lockstep_min;      // FOLD_WALK: segments at least this long are walked in lockstep (0: the built-in 11)
    // Fused tile scan and merge (FOLD_WALK job launches): when set (device
    // memory, both), the prefix rows stay in shared memory (cum / cum32
    // unused), the CTA scans its periods' tiles into shared memory and
    // merges them into the records as k_merge does (the scan's parts, keys
    // and flags unused).
    const ScanArgs* scan;
    const MergeArgs* merge;
    // Coarse-map epilogue (FOLD_WALK only): when map_out is set, the prefix
    // rows stay in shared memory (cum / cum32 unused) and each period's best
    // box score per map duration, as k_box_map computes it, goes to
    // map_out[period * map_nd + d].
    float* map_out;
    const double* map_durations;  // map_nd
    const double* map_rho;        // map_nd
    int map_nd;
    double map_baseline;          // baseline_norm c
};

// Launch shape of the fold (fold_group_shape).
struct FoldShape {
    int kind;           // FOLD_WALK (k_fold_walk) or FOLD_SMEM (k_fold)
    int group;          // periods per CTA, a power of two <= MAX_GROUP (FOLD_WALK: <= WALK_MAX_GROUP)
    bool hist_in_smem;  // else window mode: 3 G nb doubles of global histogram per CTA
    int window;         // 0 (full mode) or the window's rows (cells)
    int row_stride;     // shared-memory row stride of a period's bins
    int span_cap;       // cells a chunk may span (window mode)
    int chunk_cap;      // observations per chunk at most
    int threads;        // CTA size
    int stage_field;    // staged slots per field: chunk_cap + segments
    size_t smem;        // dynamic shared memory bytes
    int lockstep_min;   // FOLD_WALK: FoldArgs::lockstep_min for this shape (0: built-in)
    bool pair;          // FOLD_WALK: the paired walk (two periods per lane; group >= 2, <= 512 threads)
};

// Measured tuning of the fold's launch shape (process-wide): per nb class
// floor(log2(nb)) the largest period group (0 = the built-in rule), the
// walking fold's CTA size (128, 256, 512 or 1024; 0 = 1024) and its lockstep
// threshold (0 = the built-in 11); the periods per launch (0 = 16,384), and
// whether a batch's walking-fold jobs run as a persistent work-stealing grid.
struct FoldTuning {
    uint32_t group_cap[32];
    uint32_t threads[32];
    uint32_t lockstep_min[32];
    uint32_t pair[32];
    uint32_t launch_periods;
    uint32_t steal;
    uint32_t fused_scan;  // nonzero: the walking fold scans and merges its own tiles (else separate kernels)
    uint32_t map_lockstep_min;  // the coarse maps' folds: lockstep threshold (0: built-in)
    uint32_t map_threads;       // the coarse maps' walking folds: CTA size (0: 1024)
    uint32_t map_group_max;     // the coarse maps' walking folds: largest period group (0: built-in)
    uint32_t batch_no_fill;     // nonzero: a batch's job launches never cut a pass's groups (else to its share of the SMs)
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
    int mixed;                // 1 = f32 pre-rank + f64 rescans, 0 = f64 only, 2 = f32 only (no f64 rows read)
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

// Single-event scan (scan_all, kernels.rs:851-921): every template of one
// trial period whose exact f64 score reaches the threshold, appended through
// a counter as (j, k, score, depth, duration index, shape index).
constexpr int EVENT_RECORD = 6;
struct EventArgs {
    const double* cum;        // NF x (2nb+1)
    const double* durations;  // nd, ascending
    const double* rho;        // nd
    const double* ingress;    // ns
    const double* factors;    // ns x layers
    double scale;
    double baseline;          // baseline_norm c
    double threshold;
    double n;                 // observation count
    int nb, nd, ns, layers;
    uint32_t capacity;        // records
    uint32_t* counter;        // templates above threshold (may exceed capacity)
    double* records;          // capacity x EVENT_RECORD
};

// Coarse periodogram of the proposal path (proposal.cu).
constexpr int MAP_MAX_DURATIONS = 8;
struct MapArgs {
    const double* cum;        // periods x NF x (2nb+1), from the fold
    const double* scales;     // periods
    const double* durations;  // nd
    const double* rho;        // nd
    int nd;
    int nb;
    double baseline;          // baseline_norm c
    double n;                 // observation count
    float* out;               // periods x nd: best box score per duration
};

// One star's time bins for k_bin_fields_jobs: vb[b], wb[b] = sums of v, w
// over observations [starts[b], starts[b + 1]).
struct BinJob {
    const double* v;
    const double* w;
    const int* starts;  // nbins + 1
    int nbins;
    double* vb;
    double* wb;
};

// One star's coarse map for k_map_features: map is P x nd floats on the
// device; its features go to x[c][star][offset .. offset + P).
struct FeatJob {
    const float* map;
    int P;
    int nd;
    int star;
    int offset;
};

// Peak-selection rescoring (rescore.cu): rows are (period, epoch, duration)
// triples; RESCORE_BLOCK lanes per row (kernels.rs:41).
constexpr int RESCORE_BLOCK = 256;
struct RescoreArgs {
    const double* time;        // n, ascending: family-relative (rescore) or absolute (count)
    const double* v;           // n (rescore)
    const double* w;           // n (rescore)
    const uint8_t* excluded;   // n
    const double* rows;        // R x 3
    double origin;             // added to time before the phase (rescore)
    int n;
    int R;
    double* sums;              // R x 3: a, hp, norm (rescore)
    uint32_t* counts;          // R x 2: in transit, of which not excluded (count)
};

// Biweight detrending (biweight.cu): blocks of up to BIWEIGHT_THREADS
// consecutive observations; a block's window union is staged in shared
// memory when it holds at most BIWEIGHT_STAGE values.
constexpr int BIWEIGHT_THREADS = 128;
constexpr int BIWEIGHT_STAGE = 25600;  // doubles (200 KB)
struct BiweightArgs {
    const double* flux;      // n: 1 + relative flux
    const uint32_t* lo;      // n: first index of each window
    const uint32_t* hi;      // n: one past the last
    const uint32_t* blocks;  // 4 per block: first, count, union start, union end
    double c;                // tuning constant
    int iterations;
    double* out;             // n: flux / location - 1
};

// Launch shape of a fold of `periods` periods at nb bins. `tuned`: the
// walking fold takes its CTA size and lockstep threshold from the tuning
// table (callers whose job launches mix shapes keep 1024 threads).
// `fill_ctas`: period groups are cut until the fold has at least this many
// CTAs (-1: sm_count; 0: no cut, for a job launch holding many such folds).
FoldShape fold_group_shape(int nb, int periods, int sm_count, bool tuned = false, int fill_ctas = -1);
// The coarse maps' fold shape: the walking fold with the tuning table's map
// CTA size, group cap (nonzero: groups up to the cap whatever the SM count,
// as a batch's launch holds every star's groups) and lockstep threshold,
// else fold_group_shape's.
FoldShape fold_map_shape(int nb, int periods, int sm_count);
void set_fold_tuning(const FoldTuning& t);
void get_fold_tuning(FoldTuning* t);
uint32_t tuned_launch_periods();
bool tuned_fused_scan();
bool tuned_batch_no_fill();
bool tuned_fold_steal();
// Cuts n ascending times into fold chunks of at most chunk_cap observations
// spanning at most min(nb, span_cap) - 2 cells at any scale <= scale_max.
// Writes count + 1 offsets; returns count, or -1 when capacity is too small.
int fold_chunks(const double* time, int n, double scale_max, int nb, int span_cap, int chunk_cap, int* out,
                int capacity);
// fold_chunks into `out` (count + 1 offsets), sized by a bound on the count
// rather than by n: every chunk but the last ends after chunk_cap
// observations or at least a span after its first, so there are at most
// (t_last - t_first) / span + n / chunk_cap + 1 of them.
int fold_chunk_list(const double* time, int n, double scale_max, int nb, int span_cap, int chunk_cap,
                    std::vector<int>& out);
cudaError_t launch_fold(const FoldArgs& a, const FoldShape& shape, cudaStream_t stream);
// The walking fold with the tile scan and merge fused (FOLD_WALK shapes, no
// map or histogram output): the prefix rows stay in shared memory, every CTA
// scans its periods' tiles with groups of TILE threads into shared memory
// and merges them into m's records (s.cum, s.cum32, s.parts, s.keys,
// s.flags and m.parts, m.keys, m.flags unused). The same records as
// launch_fold + launch_scan_tiles + launch_merge.
cudaError_t launch_fold_scan(const FoldArgs& a, const FoldShape& shape, const ScanArgs& s, const MergeArgs& m,
                             cudaStream_t stream);
// Job launches (the batched search): jobs and their first CTA / period
// offsets (njobs + 1 entries, the last = total) live in device memory.
// A walking-fold job within limits. A job may write one period's raw
// histogram (hist_out, group 1) instead of prefix rows.
bool fold_job_ok(const FoldArgs& a, const FoldShape& shape);
// The scan and merge of a fused walking-fold job within limits.
bool fused_scan_ok(const FoldArgs& a, const ScanArgs& s, const MergeArgs& m);
// A staged-by-threads (FOLD_SMEM) fold job within limits, and the launch of
// many of them with one CTA size.
bool fold_smem_job_ok(const FoldArgs& a, const FoldShape& shape);
cudaError_t launch_fold_smem_jobs(const FoldArgs* jobs, const int* cta0, int njobs, int ctas, int threads, size_t smem,
                                  cudaStream_t stream);
// Walking-fold jobs of one CTA size and form (`threads`, `pair`, of their
// shapes).
cudaError_t launch_fold_jobs(const FoldArgs* jobs, const int* cta0, int njobs, int ctas, int threads, bool pair,
                             size_t smem, cudaStream_t stream);
// The same fold jobs by a persistent grid of one CTA per SM taking units
// from `counter` (device memory, zeroed by the launch).
cudaError_t launch_fold_steal(const FoldArgs* jobs, const int* cta0, int njobs, int units, int threads, bool pair,
                              size_t smem, unsigned int* counter, int sm_count, cudaStream_t stream);
// CTAs of a period's tile scan (one per tile); a scan job of n periods
// takes n times this many CTAs of launch_scan_jobs.
int scan_ctas_per_period(int nb);
cudaError_t launch_scan_jobs(const ScanArgs* jobs, const int* cta0, int njobs, int ctas, cudaStream_t stream);
cudaError_t launch_merge_jobs(const MergeArgs* jobs, const int* p0, int njobs, int total, cudaStream_t stream);
cudaError_t launch_scan_tiles(const ScanArgs& a, int periods, cudaStream_t stream);
cudaError_t launch_scan_all(const EventArgs& a, cudaStream_t stream);
cudaError_t launch_merge(const MergeArgs& a, cudaStream_t stream);
cudaError_t launch_box_map(const MapArgs& a, int periods, cudaStream_t stream);
cudaError_t launch_bin_fields(const double* v, const double* w, const int* starts, int nbins, double* vb, double* wb,
                              cudaStream_t stream);
// Job launches of the maps: jobs and offsets (njobs + 1) in device memory.
cudaError_t launch_box_map_jobs(const MapArgs* jobs, const int* p0, int njobs, int total, cudaStream_t stream);
cudaError_t launch_bin_fields_jobs(const BinJob* jobs, const int* b0, int njobs, int total, cudaStream_t stream);
cudaError_t launch_biweight(const BiweightArgs& a, int nblocks, size_t smem, cudaStream_t stream);
cudaError_t launch_rescore_rows(const RescoreArgs& a, cudaStream_t stream);
cudaError_t launch_count_rows(const RescoreArgs& a, cudaStream_t stream);
cudaError_t launch_map_features(const FeatJob* jobs, int njobs, int channels, int B, int T, float* x,
                                cudaStream_t stream);

}  // namespace fbls
