/* fbls_b200: B200 (sm_100a) implementation of the FBLS search hot path.
 *
 * C ABI. Plain pointers and sizes only; every host array is owned by the
 * caller and borrowed for the duration of the call. Device memory is owned by
 * the library (per context and per uploaded family) and never exposed.
 *
 * The reference (isakruas/fbls) has no FFI layer: its Rust host calls its
 * cuda-oxide kernels directly. The entry points below sit on the seams where
 * that host would call into a native library:
 *
 *   fbls_create / fbls_destroy   <- Gpu::new / Gpu::shared      src/search/scan.rs:51-77
 *   fbls_upload_ready            <- DeviceReady::upload         src/search/scan.rs:110-124
 *   fbls_scan_periods            <- scan_periods                src/search/scan.rs:363-408
 *   fbls_scan_bank               <- scan_bank (every period's   src/search/scan.rs:144-357
 *                                   winner at one nb)
 *   fbls_compare_search          <- compare_search              src/search/evidence.rs:693-1003
 *   fbls_compare_batch           <- the pipeline's evidence loop src/pipeline.rs:169-192
 *                                   (compare_search per peak)
 *
 * Host-side mirror (C++ restatements of the Rust host functions around the
 * path, for callers that do not have the Rust host):
 *
 *   fbls_period_grid             <- period_grid                 src/search/grid.rs:5-28
 *   fbls_family_state            <- family_state (prepared)     src/prep/curve.rs:541-569
 *   fbls_signal_search           <- signal_search               src/search/scan.rs:413-473
 *
 * Every call returns 0 on success or a nonzero status; fbls_last_error()
 * then holds the message. Messages that the reference raises keep its text:
 * "nonpositive template precision; inspect noise model" (scan.rs:336),
 * "one folded period exceeds max_fold_mib" (scan.rs:181).
 *
 * Threading: one context is used by one host thread at a time (the
 * reference keeps one context and stream per worker thread, scan.rs:47-64);
 * different contexts may run concurrently.
 */
#ifndef FBLS_B200_H
#define FBLS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FBLS_OK 0
#define FBLS_ERR_ARGUMENT 1
#define FBLS_ERR_CUDA 2
#define FBLS_ERR_PRECISION 3 /* nonpositive template precision */
#define FBLS_ERR_BUDGET 4    /* one folded period exceeds max_fold_mib */
#define FBLS_ERR_DATA 5      /* preparation errors (too few observations, ...) */

typedef struct fbls_ctx fbls_ctx;
typedef struct fbls_ready fbls_ready;

/* Template bank of one octave band; mirrors Bank, src/search/scan.rs:127-139.
 * durations (days, ascending) and rho have nd entries; ingress has ns. */
typedef struct {
    const double* durations;
    const double* rho;
    uint32_t nd;
    const double* ingress;
    uint32_t ns;
    uint32_t layers;
    double threshold;
    double shape_gate;
    uint32_t phase_oversample;
    uint32_t period_batch;
    double max_fold_mib;
    uint32_t prescan_factor;
    double prescan_fraction;
} fbls_bank;

/* One qualifying period; mirrors Row, src/search/scan.rs:17-23. */
typedef struct {
    double period;
    double epoch;
    double duration;
    double score;
    double depth;
} fbls_row;

/* Mirrors ScanStats, src/search/scan.rs:26-37. exact_tile_retries keeps the
 * reference's reported value (its flag word never carries the retry bit once
 * the f64 rescan has run, kernels.rs:796, :841-842); tile_rescans counts the
 * tiles whose f64 rescan actually ran. */
typedef struct {
    uint64_t periods;
    uint64_t prescan_survivors;
    uint64_t phase_bins;
    uint64_t batches;
    uint64_t templates_scanned;
    uint64_t exact_tile_retries;
    uint64_t tile_rescans;
    double seconds;
    double seconds_fold;
    double seconds_cumulative;
    double seconds_scan;
} fbls_scan_stats;

/* Search configuration fields read by the path; mirrors SearchConfig,
 * src/config.rs:6-88 (defaults there). stellar_radius_solar = NaN means None. */
typedef struct {
    double period_min;
    double period_max;
    double threshold;
    const double* ingress_fractions;
    uint32_t n_ingress;
    uint32_t shape_layers;
    uint32_t phase_oversample;
    double shape_gate_fraction;
    uint32_t prescan_factor;
    double prescan_fraction;
    double period_oversample;
    uint32_t period_batch;
    double max_fold_mib;
    double evidence_rtol;
    double planet_prior;
    double binary_prior;
    double planet_depth_scale;
    double binary_depth_scale;
    double diluted_binary_depth_scale;
    double stellar_radius_solar;
    double planet_radius_scale_rj;
    double target_flux_fraction;
    /* Scan precision: 0 = the reference's mixed mode (f32 pre-rank from
     * (hi, lo) pairs, f64 winner and rescans); 1 = f64 ranking throughout;
     * 2 = the f32 form (f32 ranking from the (hi, lo) pairs, no rescans, the
     * winner's score, depth and sums in f32: values within ~1e-6 of mode 1,
     * winners equal except at near ties). */
    uint32_t precision_mode;
} fbls_config;

/* Evidence row; mirrors EvidenceRow, src/search/evidence.rs:638-653. */
typedef struct {
    double period;
    double epoch;
    double duration;
    double snr;
    double depth;
    double planet_log_odds;
    double log_bf_planet_noise;
    double log_bf_binary_noise;
    double binary_secondary_ratio;
    double binary_secondary_phase;
    double binary_odd_even_ratio;
    double binary_period_days;
    double ingress_fraction;
    uint32_t selection_flags;
} fbls_evidence_row;

/* ---- context ---------------------------------------------------------- */

/* Replaces Gpu::new (scan.rs:66-77): device context, stream, workspace. */
fbls_ctx* fbls_create(int device, int* status);
void fbls_destroy(fbls_ctx* ctx);
/* Message of the last failed call on this context (never NULL). */
const char* fbls_last_error(const fbls_ctx* ctx);
/* Library version string. */
const char* fbls_version(void);

/* ---- boundary --------------------------------------------------------- */

/* Replaces DeviceReady::upload (scan.rs:110-124): uploads the prepared
 * family fields (times relative to origin, ascending; v; w) of n
 * observations. residual_energy is Ready::residual_energy (curve.rs:440). */
int fbls_upload_ready(fbls_ctx* ctx, const double* time, const double* v, const double* w, uint32_t n,
                      double baseline_norm, double origin, double residual_energy, fbls_ready** out);
/* Frees an uploaded family; before or after fbls_destroy of its context. */
void fbls_free_ready(fbls_ready* ready);

/* Replaces scan_periods (scan.rs:363-408): best template per period over
 * the bank, coarse prescan then full scan on survivors; writes the rows whose
 * score reaches bank->threshold (at most P) in period order. precision_mode
 * as in fbls_config. */
int fbls_scan_periods(fbls_ctx* ctx, const fbls_ready* ready, const double* periods, uint32_t P,
                      const fbls_bank* bank, uint32_t precision_mode, fbls_row* rows_out, uint32_t* n_rows,
                      fbls_scan_stats* stats);

/* Every period's winner at nb phase bins (one scan_bank pass, scan.rs:144-357):
 * records P x 9 (period, scale, phase, width, a, norm, d, ingress, rho),
 * score and depth P each, flags P (OR of the tile flag words). */
int fbls_scan_bank(fbls_ctx* ctx, const fbls_ready* ready, const double* periods, uint32_t P,
                   const fbls_bank* bank, uint32_t nb, uint32_t precision_mode, double* records, double* score,
                   double* depth, uint32_t* flags, fbls_scan_stats* stats);

/* Replaces compare_search (evidence.rs:693-1003) at one trial period.
 * durations/rho: the family's nd durations (days) and correlated-noise
 * factors, any order. Writes 0, 1 or 2 rows. */
int fbls_compare_search(fbls_ctx* ctx, const fbls_ready* ready, const double* durations, const double* rho,
                        uint32_t nd, double period, const fbls_config* cfg, fbls_evidence_row* rows_out,
                        uint32_t* n_rows);

/* One candidate of fbls_compare_batch: an uploaded family, one trial
 * period and the family's nd durations (days) and correlated-noise factors
 * (host arrays, any order). Outputs: rows[0 .. n_rows) (0, 1 or 2 rows, as
 * fbls_compare_search writes them) and the candidate's status. */
typedef struct {
    const fbls_ready* ready;
    double period;
    const double* durations;
    const double* rho;
    uint32_t nd;
    fbls_evidence_row rows[2];
    uint32_t n_rows;
    int status;
} fbls_evidence_job;

/* compare_search (evidence.rs:693-1003) for many candidates at once: the
 * pipeline's evidence loop (src/pipeline.rs:169-192, one compare_search per
 * peak, up to evidence_candidates of them) or several stars' peaks. Every
 * candidate's fold, prefix sums, screen, pilot and joint tiles run as shared
 * launches on the context's stream with one synchronisation; the rows are
 * those of one fbls_compare_search per candidate. Returns 0, or the first
 * failing candidate's status ("candidate i: " message); every candidate's
 * own status is in its record. */
int fbls_compare_batch(fbls_ctx* ctx, fbls_evidence_job* jobs, uint32_t count, const fbls_config* cfg);

/* ---- no device allocation ----------------------------------------------
 * No counterpart in the reference. For callers that cannot call cudaMalloc
 * (their device memory is owned by someone else: a framework's caching
 * allocator that must own every allocation, or a fixed per-process memory
 * partition). Same results as fbls_scan_bank (one scan_bank pass of every
 * period at nb bins), with every device buffer carved out of one file-scope
 * __device__ array of FBLS_STATIC_SCRATCH_BYTES that each GPU loading the
 * library holds until exit. All arrays are host arrays: time, v, w (n,
 * relative times ascending), periods (P), outputs as in fbls_scan_bank.
 * Inputs whose fields, chunk table and one period's intermediates do not fit
 * the array are rejected (FBLS_ERR_ARGUMENT with the message in error);
 * larger P is processed in batches that fit. Every call resolves the
 * array's address on its device (again after a cudaDeviceReset); the first
 * call on a device also loads the module there, so make it before any stream
 * capture. Calls share the array: calls that overlap on the GPU race.
 * Runs on the legacy default stream and returns after the results are on
 * the host. */
#define FBLS_STATIC_SCRATCH_BYTES (64u * 1024u * 1024u)
int fbls_scan_bank_static(int device, const double* time, const double* v, const double* w, uint32_t n,
                          double baseline_norm, const double* periods, uint32_t P, const fbls_bank* bank,
                          uint32_t nb, uint32_t precision_mode, double* records, double* score, double* depth,
                          uint32_t* flags, char* error, uint32_t error_len);

/* ---- instrumentation (no counterpart in the reference; its FBLS_PROFILE
 * synchronises after each kernel instead, scan.rs:152, :222-229) --------- */

/* Device time of the context's stream between two calls, by CUDA events
 * recorded on that stream (stop synchronises on its event). */
int fbls_timer_start(fbls_ctx* ctx);
int fbls_timer_stop(fbls_ctx* ctx, float* milliseconds);

/* Measured launch-shape tuning (no counterpart in the reference; written by
 * the autotuner, python -m fbls_b200.autotune, and read back from its table):
 * per nb class floor(log2(nb)) the largest fold period group (a power of two
 * up to 128; 0 = the built-in rule: the largest group up to 32 whose
 * histograms fit shared memory while every SM gets a CTA; a cap above 32
 * lets the walking fold give a period fewer than 32 lanes, down to 8), the
 * periods per launch (0 = 16,384), and
 * fold_steal: nonzero runs a batch's walking-fold jobs (fbls_search_batch
 * with workers 0) as one persistent grid of a CTA per SM that takes the next
 * (star, pass, period-group) unit from a counter, instead of a CTA per unit.
 * Per nb class, for the signal-search folds: fold_threads, the walking
 * fold's CTA size (128, 256, 512 or 1024; 0 = 1024; the period group is cut
 * to at least 8 lanes per period), and lockstep_min, the segment length from
 * which a CTA's lanes walk their observations in lockstep rather than each
 * its own window (0 = 11; at most 4096). fused_scan: nonzero has the
 * walking fold's CTAs scan and merge their own periods' tiles from the prefix
 * sums they keep in shared memory (no prefix rows or tile parts in device
 * memory), instead of the separate scan and merge kernels over prefix rows
 * the fold writes to device memory (the default, faster on B200).
 * map_lockstep_min: lockstep_min of the coarse maps' folds (their binned
 * families walk short segments), one value for every nb. fold_pair, per nb
 * class of the signal-search folds: nonzero walks two periods per lane, one
 * read of each staged observation serving both (CTAs of at most 512
 * threads; 512 when fold_threads is 0). map_threads and map_group_max: the
 * coarse maps' walking folds' CTA size (as fold_threads) and largest period
 * group (as fold_group_max, but a nonzero cap is taken whatever the SM count:
 * a map batch's launch holds every star's groups), one value for every nb.
 * batch_no_fill (0 or 1): in fbls_search_batch's job launches (workers 0),
 * which hold many passes (star, band, prescan or full scan) together, the
 * default cuts a pass's period groups until it has its share of CTAs
 * (ceil(SMs / passes of the launch session)); 1 never cuts them.
 * Process-wide; results do not depend on it, only the launch shapes do. */
typedef struct {
    uint32_t fold_group_max[32];
    uint32_t launch_periods;
    uint32_t fold_steal;
    uint32_t fold_threads[32];
    uint32_t lockstep_min[32];
    uint32_t fused_scan;
    uint32_t map_lockstep_min;
    uint32_t fold_pair[32];
    uint32_t map_threads;
    uint32_t map_group_max;
    uint32_t batch_no_fill;
} fbls_tuning;
int fbls_set_tuning(const fbls_tuning* tuning);
int fbls_get_tuning(fbls_tuning* tuning);

/* The precision study's bin forms (no counterpart in the reference): for
 * every observation of an uploaded family and every scale (nb / period), the
 * bin floor(t * scale) mod nb of the fold (one rounded f64 product,
 * kernels.rs:314-327) against a plain f32 product, a double-single product,
 * and the double-single product with an exact f64 fallback near integers.
 * counts (5): pairs, f32 mismatches, double-single mismatches, fallbacks
 * taken, mismatches after the fallback. Needs t * scale below 2^24. */
int fbls_precision_bins(fbls_ctx* ctx, const fbls_ready* ready, const double* scales, uint32_t P, uint32_t nb,
                        uint64_t* counts);

typedef struct {
    uint64_t launches;        /* every kernel this context launched */
    uint64_t fold_launches;   /* fold + prefix launches */
    double fold_ms;           /* their summed device time (timing enabled) */
    double fold_bytes;        /* algorithmic bytes: 24 n + 48 (2 nb + 1) per period */
    uint64_t scan_launches;   /* tile scan + merge launches */
    double scan_ms;
    double scan_bytes;        /* algorithmic bytes: 24 (2 nb + 1) + 84 tiles per period */
    uint64_t fold_updates;    /* observation x period bin updates */
    uint64_t rescore_launches; /* rescore_rows + count_rows launches */
    double rescore_ms;        /* their summed device time (timing enabled) */
    double detrend_ms;        /* biweight launches' device time (timing enabled) */
} fbls_counters;

/* Enables per-launch event timing of the fold, scan and rescoring kernels
 * (adds one event record per launch, no synchronisation). */
int fbls_set_kernel_timing(fbls_ctx* ctx, int enable);
/* Reads (and with reset != 0 clears) the context's counters. */
int fbls_read_counters(fbls_ctx* ctx, fbls_counters* out, int reset);

/* ---- host-side mirror ------------------------------------------------- */

/* period_grid (grid.rs:5-28). Returns the count; writes it when capacity
 * suffices (out may be NULL to query the count). Returns -1 when the count
 * is infinite (a zero minimum period or a zero step) or above 2^53, grids the
 * reference cannot allocate either. */
int64_t fbls_period_grid(double minimum, double maximum, double baseline, double minimum_duration,
                         double oversample, double* out, int64_t capacity);

/* family_state for a prepared curve (curve.rs:541-569 with
 * fit_segment_noise at bin 0, prepare_ready, correlated_noise_factors).
 * out arrays hold n_in entries; *n_out is the usable count. scalars_out:
 * baseline_norm, origin, residual_energy, inflation, segments. Status
 * FBLS_ERR_DATA with the reference's message on bad input, FBLS_ERR_ARGUMENT
 * ("null argument") for a null array. */
int fbls_family_state(const double* time, const double* flux, const double* sigma, uint32_t n_in,
                      const double* durations, uint32_t nd, int correlated, uint32_t* n_out, double* time_out,
                      double* v_out, double* w_out, double* scalars_out, double* rho_out, char* error,
                      uint32_t error_len);

/* signal_search (scan.rs:413-473) for one family: octave bands over the
 * family's grid. At most `capacity` rows are written to rows_out and
 * *n_rows is the number found (more than capacity: ask again with room for
 * all; the grid length always suffices); stats_out holds up to 64 bands.
 * Durations must be positive and finite (FBLS_ERR_ARGUMENT otherwise, as for
 * a period grid that is infinite or too large). */
int fbls_signal_search(fbls_ctx* ctx, const fbls_ready* ready, const double* durations, const double* rho,
                       uint32_t nd, const fbls_config* cfg, fbls_row* rows_out, uint32_t capacity,
                       uint32_t* n_rows, uint64_t* grid_len, fbls_scan_stats* stats_out, uint32_t* n_bands);

/* ---- proposal path (learned pruning of the search; no counterpart in the
 * reference) ------------------------------------------------------------- */

/* Coarse periodogram of an uploaded family, the proposal network's input:
 * out[i * nd + d] = best box score over all phases of period i (ascending)
 * and duration d (1 <= nd <= 8), the score of the reference's f64 ranking
 * (scan.rs template semantics: width below nb / 2, 3 .. n - 3 points, a > 0,
 * positive precision), 0 when none counts. Periods are folded in octave
 * groups at nb = max(8, ceil(oversample * longest period / shortest
 * duration)). bin_days > 0 first sums v and w over time bins of that width
 * (floor((t - t0) / bin_days)), at each bin's mean time, and maps the bins;
 * 0 maps the observations themselves. */
int fbls_coarse_map(fbls_ctx* ctx, const fbls_ready* ready, const double* periods, uint32_t P,
                    const double* durations, const double* rho, uint32_t nd, double oversample, double bin_days,
                    float* out);

/* One coarse map of a batch: inputs as fbls_coarse_map, out (P x nd floats,
 * caller-owned host memory) and the job's status. */
typedef struct {
    const fbls_ready* ready;
    const double* periods;
    uint32_t P;
    const double* durations;
    const double* rho;
    uint32_t nd;
    double oversample;
    double bin_days;
    float* out;
    int status;
} fbls_map_job;

/* Coarse maps of many uploaded families: on `workers` host threads with their
 * own streams (the contexts fbls_search_batch keeps), or with `workers` == 0
 * all together on the context's stream, every star's folds and box maps
 * packed into shared launches. The maps are the same either way. Returns 0
 * or the first failing job's status ("map i: " message). */
int fbls_coarse_map_batch(fbls_ctx* ctx, fbls_map_job* jobs, uint32_t count, uint32_t workers);

/* The proposal network's input for a batch of stars: every job's coarse map
 * (as fbls_coarse_map_batch with workers == 0; a job's `out` may be null) and
 * x (channels x count x T floats, channel-major; host memory, or device
 * memory of the context's device, which the features are copied to without
 * leaving the GPU; ready when the call returns): row i of channel c
 * holds (log1p(max(map, 0)) - mean) / (std + 1e-3) of the job's P map values
 * of duration c at positions [offsets[i], offsets[i] + P), with mean and
 * (population) std over those P values, and zeros elsewhere and for maps of
 * fewer than 8 periods. Every job needs nd == channels (1..8) and
 * offsets[i] + P <= T. Returns 0 or the first failing job's status ("map i: "
 * message). */
int fbls_coarse_features(fbls_ctx* ctx, fbls_map_job* jobs, uint32_t count, const uint32_t* offsets,
                         uint32_t channels, uint32_t T, float* x);

/* biweight_flatten_gpu (src/prep/curve.rs:256-329, kernel biweight
 * kernels.rs:1051-1110): for every observation of the ascending `time`, the
 * Tukey biweight location (tuning constant c, `iterations` reweightings from
 * the lower median) of 1 + relative_flux over the observations within
 * window / 2 of it in its gap-separated segment; out = (1 + relative_flux) /
 * location - 1. Medians are the windows' exact lower medians (bisection as
 * the reference). Device time adds to the counters' detrend_ms when timing is
 * on. Returns 0, FBLS_ERR_ARGUMENT or FBLS_ERR_CUDA. */
int fbls_biweight_flatten(fbls_ctx* ctx, const double* time, const double* relative_flux, uint32_t n, double window,
                          double gap, double c, uint32_t iterations, double* out);

/* fit_segment_noise (src/prep/curve.rs:89-198), host only: the diagonal noise
 * model of raw mission flux. Usable observations (finite, err > 0) in time
 * order; each group (sector label) divided by its lower median (flux / m - 1,
 * err / m); times relative to the first; with bin_minutes > 0,
 * inverse-variance means per (floor(t / width), group); the adjacent
 * differences within gap_days and one group give the error inflation (with
 * `err`) or a white level (err null). err and group may be null. Outputs hold
 * up to n_in values; scalars_out: origin, inflation, segments. Returns 0,
 * FBLS_ERR_ARGUMENT, or FBLS_ERR_DATA with the reference's message. */
int fbls_fit_segment_noise(const double* time, const double* flux, const double* err, const int64_t* group,
                           uint32_t n_in, double bin_minutes, double gap_days, uint32_t* n_out, double* time_out,
                           double* deficit_out, double* variance_out, int64_t* group_out, double* scalars_out,
                           char* error, uint32_t error_len);

/* segment_edges (curve.rs:332-345): each observation's distance to the
 * nearer edge of its segment (segments split where the time step exceeds
 * gap). detrending_windows (curve.rs:349-370): the distinct windows
 * round(clamp(factor x D, minimum, maximum) x 1e6) / 1e6 in increasing order
 * (windows_out, room for nd) and each duration's window index (family_out).
 * Host only; return 0 or FBLS_ERR_ARGUMENT. */
int fbls_segment_edges(const double* time, uint32_t n, double gap, double* out);
int fbls_detrending_windows(const double* durations, uint32_t nd, double minimum, double factor, double maximum,
                            double* windows_out, uint32_t* family_out, uint32_t* n_windows);

/* PrepConfig (src/prep/curve.rs:372-379, from SearchConfig, src/main.rs:134-143). */
typedef struct {
    double bin_minutes;
    double window_min;     /* days */
    double window_factor;  /* window = clamp(factor x duration, min, max) */
    double window_max;     /* days */
    double clip_sigma;     /* positive outliers above clip_sigma robust scales are dropped */
    double edge_trim;      /* observations within edge_trim windows of a segment edge are dropped */
} fbls_prep_config;

/* One detrended curve of prepare_families: caller-owned arrays (time, flux,
 * sigma: room for n observations; indices: room for nd), filled with the kept
 * observations (absolute times), the window, the count dropped and the
 * indices of the durations searched on it. */
typedef struct {
    double* time;
    double* flux;
    double* sigma;
    uint32_t n;
    double window_days;
    uint32_t clipped;
    uint32_t* indices;
    uint32_t n_indices;
} fbls_family_out;

/* prepare_families (src/prep/curve.rs:384-425): raw flux to one detrended
 * curve per detrending window (durations grouped by clamp(window_factor x D,
 * window_min, window_max) rounded to 1e-6 d), the biweight detrend on the
 * GPU. `out` has room for nd families; *n_families is the number filled, in
 * increasing window. */
int fbls_prepare_families(fbls_ctx* ctx, const double* time, const double* flux, const double* err,
                          const int64_t* group, uint32_t n, const double* durations, uint32_t nd,
                          const fbls_prep_config* cfg, fbls_family_out* out, uint32_t* n_families);

/* EventStats, src/search/events.rs:10-15. */
typedef struct {
    uint64_t templates_scanned;   /* nb x nd x shapes */
    uint64_t threshold_survivors; /* templates at or above threshold */
    int overflow;                 /* survivors exceeded capacity: no rows */
} fbls_event_stats;

/* single_event_search (src/search/events.rs:18-153): every template (phase,
 * duration, shape) above cfg->threshold at one trial period longer than the
 * observing baseline (baseline + 2 x longest duration + 1e-6 d), so nothing
 * folds; nb = max(8, ceil(phase_oversample x trial / shortest duration)).
 * Rows: period +inf, epoch, duration, score (the exact f64 score), depth
 * (a / q), ordered by (phase, duration, shape) — the reference appends them
 * in an arbitrary order. More than `capacity` survivors: no rows, overflow
 * set, status 0. */
int fbls_single_event_search(fbls_ctx* ctx, const fbls_ready* ready, const double* durations, const double* rho,
                             uint32_t nd, const fbls_config* cfg, uint32_t capacity, fbls_row* rows_out,
                             uint32_t* n_rows, fbls_event_stats* stats);

/* Peak-selection rescoring, replacing the kernels rescore_rows and
 * count_rows (src/search/kernels.rs:936-1042) that Rescorer::evaluate
 * (src/select/peaks.rs:148-252) launches. rows: R x 3 (period, epoch,
 * duration; days, epoch absolute). fbls_rescore_rows: per row the sums
 * (a = sum v, hp = sum w, norm = sum w) over the uploaded family's
 * observations with excluded[i] == 0 and |phase| <= duration / 2, where x =
 * ((t + origin) - epoch) / period + 0.5 and phase = (x - floor(x) - 0.5) *
 * period; sums: R x 3. fbls_count_rows: per row the observations of `time`
 * (absolute, ascending, n) in transit (phase from t - epoch) and, of those,
 * the ones with excluded[i] == 0; counts: R x 2. The sums are the reference's
 * bit for bit (same per-lane order and reduction tree). Returns 0,
 * FBLS_ERR_ARGUMENT or FBLS_ERR_CUDA. */
int fbls_rescore_rows(fbls_ctx* ctx, const fbls_ready* family, const uint8_t* excluded, const double* rows,
                      uint32_t R, double* sums);
int fbls_count_rows(fbls_ctx* ctx, const double* time, uint32_t n, const uint8_t* excluded, const double* rows,
                    uint32_t R, uint32_t* counts);

/* Proposal network kernels. Every pointer is device memory; `stream` is a
 * cudaStream_t (NULL: the legacy stream). Activations are f32 laid out
 * [channel][curve][position]. Returns 0, FBLS_ERR_ARGUMENT or FBLS_ERR_CUDA. */

/* C(m, n) = alpha sum_k A(m, k) B(k, n) + beta C(m, n) for `batch` problems,
 * X(i, j) = X[i * s_i + j * s_j + batch index * s_b]; the operands are
 * rounded to bf16 and multiplied on the tensor cores with f32 accumulation. */
int fbls_nn_gemm(const float* A, const float* B, float* C, int M, int N, int K, long long sam, long long sak,
                 long long sab, long long sbk, long long sbn, long long sbb, long long scm, long long scn,
                 long long scb, int batch, float alpha, float beta, void* stream);
/* Xcol[ci*KW + k][b][t] = X[ci][b][t + k - R] (0 outside), and its adjoint. */
int fbls_nn_im2col(const float* X, float* Xcol, int B, int Ci, int T, int KW, int R, void* stream);
int fbls_nn_col2im(const float* dXcol, float* dX, int B, int Ci, int T, int KW, int R, void* stream);
/* Z = maxpool_P(relu(Y + bias)) with the argmax offsets, and the backward
 * pass to dY (dbias accumulates). */
int fbls_nn_bias_relu_pool(const float* Y, const float* bias, float* Z, uint8_t* idx, int B, int C, int T, int P,
                           void* stream);
int fbls_nn_bias_relu_pool_bwd(const float* dZ, const float* Z, const uint8_t* idx, float* dY, float* dbias, int B,
                               int C, int T, int P, void* stream);
/* The same with GELU (x Phi(x)) in place of ReLU; the backward pass reads
 * the pre-activation Y and the bias. P = 1 is GELU without pooling. */
int fbls_nn_bias_gelu_pool(const float* Y, const float* bias, float* Z, uint8_t* idx, int B, int C, int T, int P,
                           void* stream);
int fbls_nn_bias_gelu_pool_bwd(const float* dZ, const float* Y, const uint8_t* idx, const float* bias, float* dY,
                               float* dbias, int B, int C, int T, int P, void* stream);
/* Head: logits[b][j] = mean over a group of G positions of (wh . Z[:, b, t] +
 * bh); with labels, the softmax cross-entropy per curve and d loss_mean /
 * d logits; and its backward pass (dwh, dbh accumulate). */
int fbls_nn_head(const float* Z, const float* wh, const float* bh, const int* labels, float* logits, float* loss,
                 float* dlogits, int B, int C, int T, int G, void* stream);
int fbls_nn_head_bwd(const float* Z, const float* wh, const float* dlogits, float* dZ, float* dwh, float* dbh, int B,
                     int C, int T, int G, void* stream);
/* Adam step t (>= 1) with bias correction over n parameters. */
int fbls_nn_adam(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2, float eps,
                 int t, void* stream);
/* AdamW step t (>= 1): Adam with the weight decay wd decoupled from the
 * gradient (w -= lr (m_hat / (sqrt(v_hat) + eps) + wd w)). */
int fbls_nn_adamw(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2, float eps,
                  float wd, int t, void* stream);

/* signal_search restricted to period ranges [lo, hi) given as n_ranges
 * pairs (no counterpart in the reference; the proposal path's pruned search):
 * the same octave bands, durations and nb as the full search (nb from each
 * octave's last grid period), scanning only the grid periods inside a range,
 * so its rows are exactly the full search's rows in those ranges. n_ranges = 0
 * is fbls_signal_search. */
int fbls_signal_search_ranges(fbls_ctx* ctx, const fbls_ready* ready, const double* durations, const double* rho,
                              uint32_t nd, const fbls_config* cfg, const double* ranges, uint32_t n_ranges,
                              fbls_row* rows_out, uint32_t capacity, uint32_t* n_rows, uint64_t* grid_len,
                              fbls_scan_stats* stats_out, uint32_t* n_bands);

/* ---- batched search (replaces the reference's per-device worker threads,
 * src/batch.rs:61-102, each running one star's search at a time) --------- */

/* One star of a batch. Inputs: an uploaded family (`ready`), or a prepared
 * family in host memory (time, v, w, n and its scalars) that the worker
 * uploads itself; the family's durations and rho; period_max overrides
 * cfg->period_max when finite (SearchConfig per star). Outputs: rows
 * (caller-owned, capacity of them; n_rows counts every row found, so
 * n_rows > capacity means the rows were cut short), the row count, grid
 * length, templates scanned and the star's status. */
typedef struct {
    const fbls_ready* ready;
    const double* time;
    const double* v;
    const double* w;
    uint32_t n;
    double baseline_norm;
    double origin;
    double residual_energy;
    const double* durations;
    const double* rho;
    uint32_t nd;
    double period_max;
    fbls_row* rows;
    uint32_t capacity;
    uint32_t n_rows;
    uint64_t grid_len;
    uint64_t templates;
    int status;
    /* optional: search only these period ranges (see fbls_signal_search_ranges) */
    const double* ranges;
    uint32_t n_ranges;
} fbls_star;

/* signal_search for every star of `stars` on the context's device. With
 * `workers` >= 1, host threads (up to 64, the caller's thread included) take
 * one star at a time, each with its own stream and workspace (kept in ctx for
 * later calls). With `workers` == 0 the stars are searched together on the
 * context's stream, in groups of up to 2^21 grid periods: each group's band
 * scans run as job launches covering every star of the group (a bank the
 * planner rejects fails the whole group). Results are the same as one
 * fbls_signal_search per star either way. Returns 0, or the status of the
 * first failing star (its message in fbls_last_error, prefixed "star i: ");
 * every star's own status is in its record. Do not share a context between
 * concurrent calls. */
int fbls_search_batch(fbls_ctx* ctx, fbls_star* stars, uint32_t count, const fbls_config* cfg, uint32_t workers);

#ifdef __cplusplus
}
#endif

#endif /* FBLS_B200_H */
