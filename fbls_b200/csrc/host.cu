// Host driver of the FBLS search path on one B200 and the search's C ABI
// (context, families, scan_bank / scan_periods / signal_search, evidence, the
// batch runner). The coarse maps are in host_maps.cu, the steps either side
// of the search in host_next.cu, the shared context and helpers in
// host_internal.h.
//
// Restates the reference's host logic around the kernels:
//   scan_bank      src/search/scan.rs:144-357 (bank factors, fold budget,
//                  batching, launch sequence, row decode, statistics)
//   scan_periods   src/search/scan.rs:363-408 (coarse prescan, survivors,
//                  full scan, threshold)
//   signal_search  src/search/scan.rs:413-473 (octave bands)
// The device work differs from the reference's: fold and prefix run as one
// kernel with the histograms in shared memory, and a signal search runs as
// two sessions (every band's first pass, then every band's survivor pass),
// each with one upload from page-locked memory, all launches back to back on
// one stream, one download and one synchronisation.
#include <tuple>

#include "common.cuh"
#include "evidence.h"
#include "host_internal.h"
#include "kernels.h"
#include "prep.h"

using namespace fbls;

namespace {

// Checks a family's host arrays; a rejection's message goes to `err`.
int check_family(std::string& err, const double* time, const double* v, const double* w, uint32_t n) {
    auto bad = [&](int status, const char* message) {
        err = message;
        return status;
    };
    if (!time || !v || !w) return bad(FBLS_ERR_ARGUMENT, "null argument");
    if (n < 6) return bad(FBLS_ERR_DATA, "at least six observations are required");
    for (uint32_t i = 1; i < n; i++)
        if (!(time[i] >= time[i - 1])) return bad(FBLS_ERR_ARGUMENT, "times must be ascending");
    if (!(time[0] >= 0.0)) return bad(FBLS_ERR_ARGUMENT, "times must be relative to the first observation");
    return FBLS_OK;
}

// Checks and uploads a prepared family into `r` (DeviceReady::upload,
// scan.rs:110-124): into a fresh allocation owned by `r` when `buf` is null,
// else into the reusable context buffer `buf` (no allocation once it is
// large enough, so a batch worker never synchronises the device on cudaFree).
int upload_family(fbls_ctx* ctx, DevBuf* buf, const double* time, const double* v, const double* w, uint32_t n,
                  double baseline_norm, double origin, double residual_energy, fbls_ready* r) {
    std::string err;
    const int rc = check_family(err, time, v, w, n);
    if (rc) return fail(ctx, rc, err);
    r->ctx = ctx;
    r->device = ctx->device;
    r->n = n;
    r->baseline_norm = baseline_norm;
    r->origin = origin;
    r->residual_energy = residual_energy;
    r->t_last = time[n - 1];
    r->time_host.assign(time, time + n);
    const size_t bytes = (size_t)n * sizeof(double);
    const size_t stride = fold_field_stride(n);
    cudaError_t e;
    if (buf) {
        e = ensure(*buf, 3 * stride * sizeof(double));
        r->time = static_cast<double*>(buf->ptr);
        r->owned = false;
    } else {
        e = cudaMalloc(&r->time, 3 * stride * sizeof(double));
        r->owned = true;
    }
    if (e != cudaSuccess) {
        r->time = nullptr;
        return cuda_fail(ctx, e, "upload_ready");
    }
    r->v = r->time + stride;
    r->w = r->v + stride;
    e = cudaMemsetAsync(r->time, 0, 3 * stride * sizeof(double), ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(r->time, time, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(r->v, v, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(r->w, w, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        if (r->owned) cudaFree(r->time);
        r->time = nullptr;
        return cuda_fail(ctx, e, "upload_ready");
    }
    return FBLS_OK;
}

// A pass's outputs, read in place from its session's page-locked download
// buffer (valid until that buffer serves another session).
struct BandOut {
    const double* records = nullptr;  // P x 9
    const double* score = nullptr;
    const double* depth = nullptr;
    const uint32_t* flags = nullptr;
};

// One scan_bank pass (scan.rs:144-357): every period's best template at nb
// bins. Planned on the host, then enqueued with the other passes of a session.
struct Pass {
    const fbls_ready* r = nullptr;  // the family this pass scans
    const double* periods = nullptr;
    uint32_t P = 0;
    const fbls_bank* bank = nullptr;
    uint32_t nb = 0;
    int mode = 1;  // ScanArgs::mixed: 1 the reference's mixed ranking, 0 f64, 2 the f32 form
    // plan
    uint64_t batch = 0, launch = 0;
    FoldShape shape{};
    std::vector<double> scales, host_bank;
    std::vector<int> chunks;
    size_t in_off = 0, in_scales = 0, in_periods = 0, in_bank = 0, in_chunks = 0, in_bytes = 0;
    size_t out_off = 0, out_score = 0, out_depth = 0, out_flags = 0, out_bytes = 0;
    size_t ev0 = 0, nlaunch = 0;
    BandOut out;
    fbls_scan_stats st{};
    bool bad = false;  // a template's precision came out nonpositive
    int fill_ctas = -1;  // the fold's groups are cut to give it this many CTAs (-1: one per SM; 0: no cut)
    std::string err;   // plan_pass's message when it rejects the pass
    int fail(int status, const char* message) {
        err = message;
        return status;
    }
};

// plan_pass over every pass (in parallel: the passes are independent);
// returns the first failure in pass order, its message in ctx.
int plan_passes(fbls_ctx* ctx, std::vector<Pass>& passes);

// Checks a pass and plans its batches, launches, fold shape and chunks
// (scan.rs:144-199 for the bank factors, the budget and the batch size). Reads
// ctx but writes only p (a rejection's message goes to p.err).
int plan_pass(const fbls_ctx* ctx, const fbls_ready* r, Pass& p) {
    const fbls_bank* bank = p.bank;
    const uint32_t nd = bank->nd, ns = bank->ns, layers = bank->layers, nb = p.nb;
    p.r = r;
    std::memset(&p.st, 0, sizeof(p.st));
    p.st.phase_bins = nb;
    p.st.periods = p.P;
    if (nd == 0 || nd > (uint32_t)MAX_DURATIONS || ns == 0 || ns > (uint32_t)MAX_SHAPES || layers == 0 ||
        layers > (uint32_t)MAX_LAYERS)
        return p.fail(FBLS_ERR_ARGUMENT, "bank size outside the supported range");
    if (nb < 2) return p.fail(FBLS_ERR_ARGUMENT, "nb must be at least 2");
    // Shape factors 1 - 2 ing l / (L - 1) (scan.rs:157-171).
    p.host_bank.assign(bank->durations, bank->durations + nd);
    p.host_bank.insert(p.host_bank.end(), bank->rho, bank->rho + nd);
    p.host_bank.insert(p.host_bank.end(), bank->ingress, bank->ingress + ns);
    for (uint32_t s = 0; s < ns; s++)
        for (uint32_t l = 0; l < layers; l++)
            p.host_bank.push_back(1.0 - 2.0 * bank->ingress[s] *
                                            (layers > 1 ? (double)l / (double)(layers - 1) : 0.0));
    const uint32_t tiles = (nb + TILE - 1) / TILE;
    const double per_period_bytes = (double)(NF * (4 * (size_t)nb + 2) * 8 + NF * (2 * (size_t)nb + 1) * 8);
    const uint64_t budget = (uint64_t)std::floor((bank->max_fold_mib * 1048576.0) / per_period_bytes);
    if (budget == 0) return p.fail(FBLS_ERR_BUDGET, "one folded period exceeds max_fold_mib");
    uint64_t batch = bank->period_batch;
    if (budget < batch) batch = budget;
    if (p.P < batch) batch = p.P;
    if (batch == 0) batch = 1;
    // The phase cell floor(t * scale) must fit u32 (kernels.rs:315), with room
    // for the fold's cell arithmetic (cell + 2 nb).
    double scale_max = 0.0;
    p.scales.resize(p.P);
    for (uint32_t i = 0; i < p.P; i++) {
        p.scales[i] = (double)nb / p.periods[i];
        if (!(p.scales[i] > 0.0) || !std::isfinite(p.scales[i]))
            return p.fail(FBLS_ERR_ARGUMENT, "periods must be positive and finite");
        if (p.scales[i] > scale_max) scale_max = p.scales[i];
    }
    if (std::floor(r->t_last * scale_max) >= 4294967295.0 - 2.0 * (double)nb - 2.0)
        return p.fail(FBLS_ERR_ARGUMENT, "phase cell exceeds 32 bits");
    // Periods per launch: whole batches of the reference's size, as many as
    // the fold budget holds in this path's buffers (cum, cum32 and tile parts;
    // the histograms never reach device memory), up to 16,384 (or the tuned
    // cap), so bands with
    // few bins fill the GPU with larger period groups. Statistics still count
    // the reference's batches.
    const size_t stride = 2 * (size_t)nb + 1;
    const double launch_period_bytes =
        (double)(NF * stride * (sizeof(double) + sizeof(float2)) +
                 tiles * (PART_STRIDE * sizeof(double) + sizeof(uint64_t) + sizeof(uint32_t)));
    uint64_t launch = (uint64_t)std::floor(bank->max_fold_mib * 1048576.0 / launch_period_bytes);
    launch = std::min<uint64_t>(launch, tuned_launch_periods());
    launch = std::max<uint64_t>(launch / batch, 1) * batch;
    if (launch > p.P) launch = p.P;
    p.batch = batch;
    p.launch = launch;
    p.shape = fold_group_shape((int)nb, (int)launch, ctx->sm_count, true, p.fill_ctas);
    const int count = fold_chunk_list(r->time_host.data(), (int)r->n, scale_max, (int)nb, p.shape.span_cap,
                                      p.shape.chunk_cap, p.chunks);
    if (count < 1) return p.fail(FBLS_ERR_ARGUMENT, "fold chunking failed");
    // Device input region: scales | periods | bank | chunks; output region:
    // records | score | depth | flags.
    p.in_scales = 0;
    p.in_periods = align256(p.P * sizeof(double));
    p.in_bank = p.in_periods + align256(p.P * sizeof(double));
    p.in_chunks = p.in_bank + align256(p.host_bank.size() * sizeof(double));
    p.in_bytes = p.in_chunks + align256(p.chunks.size() * sizeof(int));
    p.out_score = align256((size_t)p.P * RECORD_STRIDE * sizeof(double));
    p.out_depth = p.out_score + align256(p.P * sizeof(double));
    p.out_flags = p.out_depth + align256(p.P * sizeof(double));
    p.out_bytes = p.out_flags + align256(p.P * sizeof(uint32_t));
    p.nlaunch = (p.P + launch - 1) / launch;
    return FBLS_OK;
}

int plan_passes(fbls_ctx* ctx, std::vector<Pass>& passes) {
    std::vector<int> rc(passes.size(), FBLS_OK);
    parallel_for(passes.size(), [&](size_t i) { rc[i] = plan_pass(ctx, passes[i].r, passes[i]); });
    for (size_t i = 0; i < passes.size(); i++)
        if (rc[i]) return fail(ctx, rc[i], passes[i].err);
    return FBLS_OK;
}

// A pass whose fold also scans and merges: walking-fold shapes, when the
// tuning table asks for it (measured slower than the separate kernels on
// B200; it keeps no prefix rows or tile parts in device memory).
bool fused_scan(const Pass& p) { return p.shape.kind == FOLD_WALK && tuned_fused_scan(); }

// Kernel counters of one fold launch of n periods: algorithmic bytes are the
// observation stream once per period (24 B per observation) plus the prefix
// rows written and read back (unfused) or the tile parts written (fused).
void count_fold(fbls_ctx* ctx, int n, uint32_t nobs, uint32_t nb, bool fused) {
    const double stride = 2.0 * nb + 1.0, tiles = (double)((nb + TILE - 1) / TILE);
    ctx->counters.fold_updates += (uint64_t)n * nobs;
    if (fused) {
        ctx->counters.fold_bytes += (double)n * (24.0 * nobs + 84.0 * tiles);
        ctx->counters.scan_bytes += (double)n * 84.0 * tiles;
    } else {
        ctx->counters.fold_bytes += (double)n * (24.0 * nobs + 48.0 * stride);
        ctx->counters.scan_bytes += (double)n * (24.0 * stride + 84.0 * tiles);
    }
}

// Runs a session of planned passes on ctx->stream: one upload of every
// pass's inputs from page-locked memory, the fold / scan / merge launches of
// all passes back to back, one download of all outputs into `down` and a
// single synchronisation.
int run_session(fbls_ctx* ctx, std::vector<Pass>& passes, PinBuf& down_buf) {
    if (passes.empty()) return FBLS_OK;
    size_t in_total = 0, out_total = 0, launches = 0;
    size_t cum_max = 0, parts_max = 0, hist_max = 0;
    for (Pass& p : passes) {
        p.in_off = in_total;
        in_total += p.in_bytes;
        p.out_off = out_total;
        out_total += p.out_bytes;
        p.ev0 = launches;
        launches += p.nlaunch;
        const size_t stride = 2 * (size_t)p.nb + 1;
        const size_t tiles = (p.nb + TILE - 1) / TILE;
        if (!fused_scan(p)) {  // a fused pass keeps its rows and tile winners in shared memory
            cum_max = std::max(cum_max, (size_t)p.launch * NF * stride);
            parts_max = std::max(parts_max, (size_t)p.launch * tiles);
        }
        if (!p.shape.hist_in_smem) {
            const size_t blocks = (p.launch + p.shape.group - 1) / p.shape.group;
            hist_max = std::max(hist_max, blocks * p.shape.group * NF * (size_t)p.shape.row_stride);
        }
    }
    CK(ensure(ctx->pass_in, in_total), "workspace");
    CK(ensure(ctx->pass_out, out_total), "workspace");
    if (cum_max) {
        CK(ensure(ctx->cum, cum_max * sizeof(double)), "workspace");
        CK(ensure(ctx->cum32, cum_max * sizeof(float2)), "workspace");
    }
    if (parts_max) {
        CK(ensure(ctx->parts, parts_max * PART_STRIDE * sizeof(double)), "workspace");
        CK(ensure(ctx->keys, parts_max * sizeof(uint64_t)), "workspace");
        CK(ensure(ctx->tflags, parts_max * sizeof(uint32_t)), "workspace");
    }
    if (hist_max) CK(ensure(ctx->hist, hist_max * sizeof(double)), "workspace");
    CK(ensure(ctx->fault, sizeof(uint32_t)), "workspace");
    CK(ensure_pinned(ctx->pin_up, in_total), "pinned workspace");
    CK(ensure_pinned(down_buf, out_total + 256), "pinned workspace");
    const bool timing = ctx->profile || ctx->kernel_timing;
    if (timing) {
        while (ctx->pool.size() < 3 * launches) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e), "event");
            ctx->pool.push_back(e);
        }
    }
    unsigned char* up = static_cast<unsigned char*>(ctx->pin_up.ptr);
    for (Pass& p : passes) {
        unsigned char* b = up + p.in_off;
        std::memcpy(b + p.in_scales, p.scales.data(), p.P * sizeof(double));
        std::memcpy(b + p.in_periods, p.periods, p.P * sizeof(double));
        std::memcpy(b + p.in_bank, p.host_bank.data(), p.host_bank.size() * sizeof(double));
        std::memcpy(b + p.in_chunks, p.chunks.data(), p.chunks.size() * sizeof(int));
    }
    cudaStream_t s = ctx->stream;
    CK(cudaMemsetAsync(ctx->fault.ptr, 0, sizeof(uint32_t), s), "workspace");
    CK(cudaMemcpyAsync(ctx->pass_in.ptr, up, in_total, cudaMemcpyHostToDevice, s), "upload");
    unsigned char* din = static_cast<unsigned char*>(ctx->pass_in.ptr);
    unsigned char* dout = static_cast<unsigned char*>(ctx->pass_out.ptr);
    for (Pass& p : passes) {
        const fbls_ready* r = p.r;
        const uint32_t nb = p.nb, nd = p.bank->nd, ns = p.bank->ns, layers = p.bank->layers;
        const uint32_t tiles = (nb + TILE - 1) / TILE;
        const size_t stride = 2 * (size_t)nb + 1;
        const double* d_scales = reinterpret_cast<const double*>(din + p.in_off + p.in_scales);
        const double* d_periods = reinterpret_cast<const double*>(din + p.in_off + p.in_periods);
        const double* d_bank = reinterpret_cast<const double*>(din + p.in_off + p.in_bank);
        const int* d_chunks = reinterpret_cast<const int*>(din + p.in_off + p.in_chunks);
        double* d_records = reinterpret_cast<double*>(dout + p.out_off);
        double* d_score = reinterpret_cast<double*>(dout + p.out_off + p.out_score);
        double* d_depth = reinterpret_cast<double*>(dout + p.out_off + p.out_depth);
        uint32_t* d_flags = reinterpret_cast<uint32_t*>(dout + p.out_off + p.out_flags);
        size_t li = p.ev0;
        for (uint64_t cursor = 0; cursor < p.P; cursor += p.launch, li++) {
            const int n = (int)std::min<uint64_t>(p.P - cursor, p.launch);
            FoldArgs fa{};
            fa.time = r->time;
            fa.v = r->v;
            fa.w = r->w;
            fa.scales = d_scales + cursor;
            fa.n = (int)r->n;
            fa.nb = (int)nb;
            fa.periods = n;
            fa.group = p.shape.group;
            fa.cum = as<double>(ctx->cum);
            fa.cum32 = as<float2>(ctx->cum32);
            fa.hist_global = p.shape.hist_in_smem ? nullptr : as<double>(ctx->hist);
            fa.hist_out = nullptr;
            fa.chunks = d_chunks;
            fa.nchunks = (int)p.chunks.size() - 1;
            fa.stage_field = p.shape.stage_field;
            fa.window = p.shape.window;
            fa.row_stride = p.shape.row_stride;
            fa.fault = as<uint32_t>(ctx->fault);
            fa.rows32_only = p.mode == 2 ? 1 : 0;
            fa.lockstep_min = p.shape.lockstep_min;
            ScanArgs sa{};
            sa.cum = fa.cum;
            sa.cum32 = fa.cum32;
            sa.scales = fa.scales;
            sa.durations = d_bank;
            sa.rho = d_bank + nd;
            sa.ingress = d_bank + 2 * nd;
            sa.factors = d_bank + 2 * nd + ns;
            sa.baseline = r->baseline_norm;
            sa.gate = p.bank->shape_gate;
            sa.n = (double)r->n;
            sa.nb = (int)nb;
            sa.nd = (int)nd;
            sa.ns = (int)ns;
            sa.layers = (int)layers;
            sa.mixed = p.mode;
            sa.parts = as<double>(ctx->parts);
            sa.keys = as<uint64_t>(ctx->keys);
            sa.flags = as<uint32_t>(ctx->tflags);
            MergeArgs ma{};
            ma.parts = sa.parts;
            ma.keys = sa.keys;
            ma.flags = sa.flags;
            ma.periods_in = d_periods + cursor;
            ma.scales = fa.scales;
            ma.periods = n;
            ma.tiles = (int)tiles;
            ma.offset = (int)cursor;
            ma.records = d_records;
            ma.score = d_score;
            ma.depth = d_depth;
            ma.flags_out = d_flags;
            const bool fused = fused_scan(p);
            if (timing) CK(cudaEventRecord(ctx->pool[3 * li], s), "event");
            if (fused) {
                fa.cum = nullptr;
                fa.cum32 = nullptr;
                CK(launch_fold_scan(fa, p.shape, sa, ma, s), "fold_scan");
            } else {
                CK(launch_fold(fa, p.shape, s), "fold");
            }
            if (timing) CK(cudaEventRecord(ctx->pool[3 * li + 1], s), "event");
            if (!fused) {
                CK(launch_scan_tiles(sa, n, s), "scan_tiles");
                CK(launch_merge(ma, s), "merge");
            }
            if (timing) CK(cudaEventRecord(ctx->pool[3 * li + 2], s), "event");
            ctx->counters.launches += fused ? 1 : 3;
            ctx->counters.fold_launches += 1;
            ctx->counters.scan_launches += 1;
            count_fold(ctx, n, r->n, nb, fused);
            p.st.templates_scanned += (uint64_t)n * nd * ns * nb;
            p.st.batches += ((uint64_t)n + p.batch - 1) / p.batch;
        }
    }
    unsigned char* down = static_cast<unsigned char*>(down_buf.ptr);
    CK(cudaMemcpyAsync(down, dout, out_total, cudaMemcpyDeviceToHost, s), "download");
    CK(cudaMemcpyAsync(down + out_total, ctx->fault.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "download");
    CK(cudaStreamSynchronize(s), "scan_bank");
    uint32_t fault = 0;
    std::memcpy(&fault, down + out_total, sizeof(uint32_t));
    if (fault) return fail(ctx, FBLS_ERR_CUDA, "fold: staging copies did not complete");
    bool bad = false;
    for (Pass& p : passes) {
        const unsigned char* b = down + p.out_off;
        p.out.records = reinterpret_cast<const double*>(b);
        p.out.score = reinterpret_cast<const double*>(b + p.out_score);
        p.out.depth = reinterpret_cast<const double*>(b + p.out_depth);
        p.out.flags = reinterpret_cast<const uint32_t*>(b + p.out_flags);
        if (timing) {
            double t_fold = 0.0, t_scan = 0.0;
            for (size_t li = p.ev0; li < p.ev0 + p.nlaunch; li++) {
                float a = 0.f, c = 0.f;
                CK(cudaEventElapsedTime(&a, ctx->pool[3 * li], ctx->pool[3 * li + 1]), "event");
                CK(cudaEventElapsedTime(&c, ctx->pool[3 * li + 1], ctx->pool[3 * li + 2]), "event");
                t_fold += a;
                t_scan += c;
            }
            ctx->counters.fold_ms += t_fold;
            ctx->counters.scan_ms += t_scan;
            p.st.seconds_fold += t_fold * 1e-3;
            p.st.seconds_scan += t_scan * 1e-3;
        }
        for (uint32_t i = 0; i < p.P; i++) {
            p.bad = p.bad || (p.out.flags[i] & 2u);
            p.st.exact_tile_retries += (p.out.flags[i] & 1u) ? 1 : 0;
            p.st.tile_rescans += (p.out.flags[i] & 4u) ? 1 : 0;
        }
        bad = bad || p.bad;
    }
    if (bad) return fail(ctx, FBLS_ERR_PRECISION, "nonpositive template precision; inspect noise model");
    return FBLS_OK;
}

// The same session as run_session with every pass's launches packed into job
// launches: the (pass, launch) units are grouped into waves whose prefix-sum
// workspace fits WAVE_BYTES, and each wave is one fold launch (walking-fold
// units as jobs; other units on their own), one scan launch and one merge
// launch, whatever the number of passes and stars. Results are the same as
// run_session's, except that a pass with a nonpositive template precision is
// only marked (Pass::bad) for its caller, so the other stars of a batch keep
// their results.
constexpr size_t WAVE_BYTES = 1536ull << 20;

int run_session_fused(fbls_ctx* ctx, std::vector<Pass>& passes, PinBuf& down_buf) {
    if (passes.empty()) return FBLS_OK;
    struct Unit {
        int pass;
        uint64_t cursor;
        int n;
        size_t cum_off, parts_off, hist_off;  // elements within the wave's workspace
        bool walk;
        bool fused;  // a walking fold that scans its own tiles (no rows in device memory)
    };
    // A wave's walking-fold jobs run as one launch per CTA size and form: job range
    // [j0, j0 + njobs) with its CTA offsets at fc0 (njobs + 1 entries).
    struct FoldLaunch {
        int threads;
        bool pair;
        int j0, njobs, fc0, ctas;
        size_t smem;
    };
    struct Wave {
        std::vector<Unit> units;
        std::vector<FoldLaunch> folds;
        size_t cum = 0, parts = 0, hist = 0;
        int fold_jobs = 0, scan_units = 0, scan_ctas = 0, merge_total = 0;
        // in the job blob; the fold jobs' fused scans and merges at off_fscan
        // and off_fmerge, in fold-job order; the other units' scans and
        // merges at off_scan and off_merge
        size_t off_fold = 0, off_fcta = 0, off_fscan = 0, off_fmerge = 0, off_scan = 0, off_scta = 0, off_merge = 0,
               off_mp = 0;
    };
    size_t in_total = 0, out_total = 0;
    for (Pass& p : passes) {
        p.in_off = in_total;
        in_total += p.in_bytes;
        p.out_off = out_total;
        out_total += p.out_bytes;
    }
    std::vector<Wave> waves(1);
    size_t cum_max = 0, parts_max = 0, hist_max = 0;
    for (size_t pi = 0; pi < passes.size(); pi++) {
        Pass& p = passes[pi];
        const size_t stride = 2 * (size_t)p.nb + 1;
        const size_t tiles = (p.nb + TILE - 1) / TILE;
        for (uint64_t cursor = 0; cursor < p.P; cursor += p.launch) {
            const int n = (int)std::min<uint64_t>(p.P - cursor, p.launch);
            const bool walk = p.shape.kind == FOLD_WALK, fused = fused_scan(p);
            const size_t cum = fused ? 0 : (size_t)n * NF * stride, parts = fused ? 0 : (size_t)n * tiles;
            const size_t hist = walk ? 0 : ((n + p.shape.group - 1) / p.shape.group) * (size_t)p.shape.group * NF *
                                               (size_t)p.shape.row_stride;
            // A wave's device workspace (prefix rows and tile parts) stays within WAVE_BYTES.
            auto bytes = [](size_t c, size_t t) {
                return c * (sizeof(double) + sizeof(float2)) + t * (PART_STRIDE * sizeof(double) + 12);
            };
            if (!waves.back().units.empty() && bytes(waves.back().cum + cum, waves.back().parts + parts) > WAVE_BYTES)
                waves.emplace_back();
            Wave& w = waves.back();
            w.units.push_back({(int)pi, cursor, n, w.cum, w.parts, w.hist, walk, fused});
            w.cum += cum;
            w.parts += parts;
            w.hist += hist;
            if (walk) {
                w.fold_jobs++;
                FoldLaunch* fl = nullptr;
                for (FoldLaunch& f : w.folds)
                    if (f.threads == p.shape.threads && f.pair == p.shape.pair) fl = &f;
                if (!fl) {
                    w.folds.push_back({p.shape.threads, p.shape.pair, 0, 0, 0, 0, 0});
                    fl = &w.folds.back();
                }
                fl->njobs++;
                fl->ctas += (n + p.shape.group - 1) / p.shape.group;
                fl->smem = std::max(fl->smem, p.shape.smem);
            }
            if (!fused) {
                w.scan_units++;
                w.scan_ctas += n * scan_ctas_per_period((int)p.nb);
                w.merge_total += n;
            }
            p.st.templates_scanned += (uint64_t)n * p.bank->nd * p.bank->ns * p.nb;
            p.st.batches += ((uint64_t)n + p.batch - 1) / p.batch;
        }
    }
    // Job blob: per wave, fold jobs + CTA offsets, scan jobs + CTA offsets,
    // merge jobs + period offsets.
    size_t blob = 0;
    auto take = [&](size_t bytes) {
        const size_t at = blob;
        blob += align256(bytes);
        return at;
    };
    for (Wave& w : waves) {
        cum_max = std::max(cum_max, w.cum);
        parts_max = std::max(parts_max, w.parts);
        hist_max = std::max(hist_max, w.hist);
        const size_t nu = w.units.size();
        w.off_fold = take(std::max(1, w.fold_jobs) * sizeof(FoldArgs));
        int j0 = 0, fc0 = 0;
        for (FoldLaunch& f : w.folds) {
            f.j0 = j0;
            f.fc0 = fc0;
            j0 += f.njobs;
            fc0 += f.njobs + 1;
        }
        w.off_fcta = take((w.fold_jobs + w.folds.size() + 1) * sizeof(int));
        w.off_fscan = take(std::max(1, w.fold_jobs) * sizeof(ScanArgs));
        w.off_fmerge = take(std::max(1, w.fold_jobs) * sizeof(MergeArgs));
        w.off_scan = take(std::max(1, w.scan_units) * sizeof(ScanArgs));
        w.off_scta = take((w.scan_units + 1) * sizeof(int));
        w.off_merge = take(std::max(1, w.scan_units) * sizeof(MergeArgs));
        w.off_mp = take((w.scan_units + 1) * sizeof(int));
    }
    const size_t up_total = in_total + blob;
    CK(ensure(ctx->pass_in, up_total), "workspace");
    CK(ensure(ctx->pass_out, out_total), "workspace");
    if (cum_max) {
        CK(ensure(ctx->cum, cum_max * sizeof(double)), "workspace");
        CK(ensure(ctx->cum32, cum_max * sizeof(float2)), "workspace");
    }
    CK(ensure(ctx->parts, parts_max * PART_STRIDE * sizeof(double)), "workspace");
    CK(ensure(ctx->keys, parts_max * sizeof(uint64_t)), "workspace");
    CK(ensure(ctx->tflags, parts_max * sizeof(uint32_t)), "workspace");
    if (hist_max) CK(ensure(ctx->hist, hist_max * sizeof(double)), "workspace");
    CK(ensure(ctx->fault, sizeof(uint32_t)), "workspace");
    CK(ensure_pinned(ctx->pin_up, up_total), "pinned workspace");
    CK(ensure_pinned(down_buf, out_total + 256), "pinned workspace");
    unsigned char* up = static_cast<unsigned char*>(ctx->pin_up.ptr);
    unsigned char* din = static_cast<unsigned char*>(ctx->pass_in.ptr);
    unsigned char* dout = static_cast<unsigned char*>(ctx->pass_out.ptr);
    for (Pass& p : passes) {
        unsigned char* b = up + p.in_off;
        std::memcpy(b + p.in_scales, p.scales.data(), p.P * sizeof(double));
        std::memcpy(b + p.in_periods, p.periods, p.P * sizeof(double));
        std::memcpy(b + p.in_bank, p.host_bank.data(), p.host_bank.size() * sizeof(double));
        std::memcpy(b + p.in_chunks, p.chunks.data(), p.chunks.size() * sizeof(int));
    }
    // Jobs (device pointers into the buffers ensured above).
    for (Wave& w : waves) {
        FoldArgs* fj = reinterpret_cast<FoldArgs*>(up + in_total + w.off_fold);
        int* fc = reinterpret_cast<int*>(up + in_total + w.off_fcta);
        ScanArgs* fs = reinterpret_cast<ScanArgs*>(up + in_total + w.off_fscan);
        const ScanArgs* d_fs = reinterpret_cast<const ScanArgs*>(din + in_total + w.off_fscan);
        MergeArgs* fm = reinterpret_cast<MergeArgs*>(up + in_total + w.off_fmerge);
        const MergeArgs* d_fm = reinterpret_cast<const MergeArgs*>(din + in_total + w.off_fmerge);
        ScanArgs* sj = reinterpret_cast<ScanArgs*>(up + in_total + w.off_scan);
        int* sc = reinterpret_cast<int*>(up + in_total + w.off_scta);
        MergeArgs* mj = reinterpret_cast<MergeArgs*>(up + in_total + w.off_merge);
        int* mp = reinterpret_cast<int*>(up + in_total + w.off_mp);
        int scta = 0, mtot = 0, su = 0;
        std::vector<int> nf(w.folds.size(), 0), fcta(w.folds.size(), 0);  // per CTA size: jobs and CTAs so far
        for (size_t u = 0; u < w.units.size(); u++) {
            const Unit& un = w.units[u];
            Pass& p = passes[un.pass];
            const fbls_ready* r = p.r;
            const uint32_t nb = p.nb, nd = p.bank->nd, ns = p.bank->ns, layers = p.bank->layers;
            const int tiles = (int)((nb + TILE - 1) / TILE);
            const double* d_scales = reinterpret_cast<const double*>(din + p.in_off + p.in_scales);
            const double* d_periods = reinterpret_cast<const double*>(din + p.in_off + p.in_periods);
            const double* d_bank = reinterpret_cast<const double*>(din + p.in_off + p.in_bank);
            const int* d_chunks = reinterpret_cast<const int*>(din + p.in_off + p.in_chunks);
            FoldArgs fa{};
            fa.time = r->time;
            fa.v = r->v;
            fa.w = r->w;
            fa.scales = d_scales + un.cursor;
            fa.n = (int)r->n;
            fa.nb = (int)nb;
            fa.periods = un.n;
            fa.group = p.shape.group;
            fa.cum = un.fused ? nullptr : as<double>(ctx->cum) + un.cum_off;
            fa.cum32 = un.fused ? nullptr : as<float2>(ctx->cum32) + un.cum_off;
            fa.hist_global = un.walk ? nullptr : as<double>(ctx->hist) + un.hist_off;
            fa.hist_out = nullptr;
            fa.chunks = d_chunks;
            fa.nchunks = (int)p.chunks.size() - 1;
            fa.stage_field = p.shape.stage_field;
            fa.window = p.shape.window;
            fa.row_stride = p.shape.row_stride;
            fa.fault = as<uint32_t>(ctx->fault);
            fa.rows32_only = p.mode == 2 ? 1 : 0;
            fa.lockstep_min = p.shape.lockstep_min;
            ScanArgs sa{};
            sa.cum = fa.cum;
            sa.cum32 = fa.cum32;
            sa.scales = fa.scales;
            sa.durations = d_bank;
            sa.rho = d_bank + nd;
            sa.ingress = d_bank + 2 * nd;
            sa.factors = d_bank + 2 * nd + ns;
            sa.baseline = r->baseline_norm;
            sa.gate = p.bank->shape_gate;
            sa.n = (double)r->n;
            sa.nb = (int)nb;
            sa.nd = (int)nd;
            sa.ns = (int)ns;
            sa.layers = (int)layers;
            sa.mixed = p.mode;
            sa.parts = as<double>(ctx->parts) + un.parts_off * PART_STRIDE;
            sa.keys = as<uint64_t>(ctx->keys) + un.parts_off;
            sa.flags = as<uint32_t>(ctx->tflags) + un.parts_off;
            MergeArgs ma{};
            ma.parts = sa.parts;
            ma.keys = sa.keys;
            ma.flags = sa.flags;
            ma.periods_in = d_periods + un.cursor;
            ma.scales = fa.scales;
            ma.periods = un.n;
            ma.tiles = tiles;
            ma.offset = (int)un.cursor;
            ma.records = reinterpret_cast<double*>(dout + p.out_off);
            ma.score = reinterpret_cast<double*>(dout + p.out_off + p.out_score);
            ma.depth = reinterpret_cast<double*>(dout + p.out_off + p.out_depth);
            ma.flags_out = reinterpret_cast<uint32_t*>(dout + p.out_off + p.out_flags);
            if (un.walk) {
                size_t g = 0;
                while (w.folds[g].threads != p.shape.threads || w.folds[g].pair != p.shape.pair) g++;
                const FoldLaunch& fl = w.folds[g];
                const int j = fl.j0 + nf[g];
                if (un.fused) {
                    if (!fused_scan_ok(fa, sa, ma)) return fail(ctx, FBLS_ERR_ARGUMENT, "fold job outside limits");
                    fs[j] = sa;
                    fm[j] = ma;
                    fa.scan = d_fs + j;
                    fa.merge = d_fm + j;
                }
                if (!fold_job_ok(fa, p.shape)) return fail(ctx, FBLS_ERR_ARGUMENT, "fold job outside limits");
                fj[j] = fa;
                fc[fl.fc0 + nf[g]++] = fcta[g];
                fcta[g] += (un.n + p.shape.group - 1) / p.shape.group;
            }
            if (!un.fused) {
                sj[su] = sa;
                mj[su] = ma;
                mp[su] = mtot;
                mtot += un.n;
                sc[su++] = scta;
                scta += un.n * scan_ctas_per_period((int)nb);
            }
            ctx->counters.fold_launches += 1;
            ctx->counters.scan_launches += 1;
            count_fold(ctx, un.n, r->n, nb, un.fused);
        }
        for (size_t g = 0; g < w.folds.size(); g++) fc[w.folds[g].fc0 + nf[g]] = fcta[g];
        sc[su] = scta;
        mp[su] = mtot;
    }
    cudaStream_t s = ctx->stream;
    const bool timing = ctx->profile || ctx->kernel_timing;
    if (timing) {
        while (ctx->pool.size() < 3 * waves.size()) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e), "event");
            ctx->pool.push_back(e);
        }
    }
    CK(cudaMemsetAsync(ctx->fault.ptr, 0, sizeof(uint32_t), s), "workspace");
    CK(cudaMemcpyAsync(din, up, up_total, cudaMemcpyHostToDevice, s), "upload");
    for (size_t wi = 0; wi < waves.size(); wi++) {
        Wave& w = waves[wi];
        if (timing) CK(cudaEventRecord(ctx->pool[3 * wi], s), "event");
        for (const FoldLaunch& fl : w.folds) {
            const FoldArgs* jobs = reinterpret_cast<const FoldArgs*>(din + in_total + w.off_fold) + fl.j0;
            const int* cta0 = reinterpret_cast<const int*>(din + in_total + w.off_fcta) + fl.fc0;
            if (tuned_fold_steal()) {
                CK(ensure(ctx->steal, sizeof(unsigned int)), "workspace");
                CK(launch_fold_steal(jobs, cta0, fl.njobs, fl.ctas, fl.threads, fl.pair, fl.smem,
                                     as<unsigned int>(ctx->steal), ctx->sm_count, s),
                   "fold");
            } else {
                CK(launch_fold_jobs(jobs, cta0, fl.njobs, fl.ctas, fl.threads, fl.pair, fl.smem, s), "fold");
            }
            ctx->counters.launches += 1;
        }
        for (const Unit& un : w.units) {
            if (un.walk) continue;
            Pass& p = passes[un.pass];
            // A unit whose histograms do not fit shared memory: its own launch.
            const ScanArgs* sj = reinterpret_cast<const ScanArgs*>(up + in_total + w.off_scan);
            const ScanArgs& sa = sj[&un - &w.units[0]];
            FoldArgs fa{};
            fa.time = p.r->time;
            fa.v = p.r->v;
            fa.w = p.r->w;
            fa.scales = sa.scales;
            fa.n = (int)p.r->n;
            fa.nb = (int)p.nb;
            fa.periods = un.n;
            fa.group = p.shape.group;
            fa.cum = const_cast<double*>(sa.cum);
            fa.cum32 = const_cast<float2*>(sa.cum32);
            fa.hist_global = as<double>(ctx->hist) + un.hist_off;
            fa.chunks = reinterpret_cast<const int*>(din + p.in_off + p.in_chunks);
            fa.nchunks = (int)p.chunks.size() - 1;
            fa.stage_field = p.shape.stage_field;
            fa.window = p.shape.window;
            fa.row_stride = p.shape.row_stride;
            fa.fault = as<uint32_t>(ctx->fault);
            fa.rows32_only = p.mode == 2 ? 1 : 0;
            CK(launch_fold(fa, p.shape, s), "fold");
            ctx->counters.launches += 1;
        }
        if (timing) CK(cudaEventRecord(ctx->pool[3 * wi + 1], s), "event");
        if (w.scan_units) {
            CK(launch_scan_jobs(reinterpret_cast<const ScanArgs*>(din + in_total + w.off_scan),
                                reinterpret_cast<const int*>(din + in_total + w.off_scta), w.scan_units, w.scan_ctas,
                                s),
               "scan_tiles");
            ctx->counters.launches += 1;
        }
        if (w.scan_units) {
            CK(launch_merge_jobs(reinterpret_cast<const MergeArgs*>(din + in_total + w.off_merge),
                                 reinterpret_cast<const int*>(din + in_total + w.off_mp), w.scan_units, w.merge_total,
                                 s),
               "merge");
            ctx->counters.launches += 1;
        }
        if (timing) CK(cudaEventRecord(ctx->pool[3 * wi + 2], s), "event");
    }
    unsigned char* down = static_cast<unsigned char*>(down_buf.ptr);
    CK(cudaMemcpyAsync(down, dout, out_total, cudaMemcpyDeviceToHost, s), "download");
    CK(cudaMemcpyAsync(down + out_total, ctx->fault.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "download");
    CK(cudaStreamSynchronize(s), "scan_bank");
    uint32_t fault = 0;
    std::memcpy(&fault, down + out_total, sizeof(uint32_t));
    if (fault) return fail(ctx, FBLS_ERR_CUDA, "fold: staging copies did not complete");
    if (timing) {
        for (size_t wi = 0; wi < waves.size(); wi++) {
            float a = 0.f, c = 0.f;
            CK(cudaEventElapsedTime(&a, ctx->pool[3 * wi], ctx->pool[3 * wi + 1]), "event");
            CK(cudaEventElapsedTime(&c, ctx->pool[3 * wi + 1], ctx->pool[3 * wi + 2]), "event");
            ctx->counters.fold_ms += a;
            ctx->counters.scan_ms += c;
        }
    }
    for (Pass& p : passes) {
        const unsigned char* b = down + p.out_off;
        p.out.records = reinterpret_cast<const double*>(b);
        p.out.score = reinterpret_cast<const double*>(b + p.out_score);
        p.out.depth = reinterpret_cast<const double*>(b + p.out_depth);
        p.out.flags = reinterpret_cast<const uint32_t*>(b + p.out_flags);
        for (uint32_t i = 0; i < p.P; i++) {
            p.bad = p.bad || (p.out.flags[i] & 2u);
            p.st.exact_tile_retries += (p.out.flags[i] & 1u) ? 1 : 0;
            p.st.tile_rescans += (p.out.flags[i] & 4u) ? 1 : 0;
        }
    }
    return FBLS_OK;
}

void add_pass_stats(fbls_scan_stats& st, const Pass& p) {
    st.phase_bins = p.st.phase_bins;
    st.batches += p.st.batches;
    st.templates_scanned += p.st.templates_scanned;
    st.exact_tile_retries += p.st.exact_tile_retries;
    st.tile_rescans += p.st.tile_rescans;
    st.seconds_fold += p.st.seconds_fold;
    st.seconds_scan += p.st.seconds_scan;
}

// One scan_bank pass on its own (fbls_scan_bank).
int scan_bank(fbls_ctx* ctx, const fbls_ready* r, const double* periods, uint32_t P, const fbls_bank* bank, uint32_t nb,
              int mode, BandOut& out, fbls_scan_stats* stats) {
    std::vector<Pass> passes(1);
    Pass& p = passes[0];
    p.periods = periods;
    p.P = P;
    p.bank = bank;
    p.nb = nb;
    p.mode = mode;
    int rc = plan_pass(ctx, r, p);
    if (rc) return fail(ctx, rc, p.err);
    rc = run_session(ctx, passes, ctx->pin_down);
    out = p.out;
    if (stats) add_pass_stats(*stats, p);
    return rc;
}

// scan_periods (scan.rs:363-408) of several bands at once, of one star or of
// many: the first pass of every band (its coarse prescan, or its full scan
// when there is none) in one session, then the full scans of every band's
// survivors in a second one. Each band's rows are appended to its `rows`
// vector, band after band; each band's stats get its passes' counts and a
// share of the two sessions' wall time by templates scanned. `fused` runs the
// sessions as job launches (run_session_fused).
struct BandJob {
    const fbls_ready* r = nullptr;
    std::vector<fbls_row>* rows = nullptr;
    const double* periods = nullptr;
    uint32_t P = 0;
    double nb_period = 0.0;  // period that sets nb (0: the last of `periods`)
    const fbls_bank* bank = nullptr;
    fbls_scan_stats st{};
    uint64_t nb = 0;
    bool coarse = false;
    std::vector<double> survivors;
    int first = -1, second = -1;  // pass indices
    int status = FBLS_OK;         // fused sessions: FBLS_ERR_PRECISION when a pass of this band was marked bad
};

int scan_bands(fbls_ctx* ctx, std::vector<BandJob>& jobs, int mode, bool fused) {
    std::vector<Pass> first, second;
    auto session = [&](std::vector<Pass>& passes, PinBuf& down) {
        return fused ? run_session_fused(ctx, passes, down) : run_session(ctx, passes, down);
    };
    for (BandJob& j : jobs) {
        std::memset(&j.st, 0, sizeof(j.st));
        j.st.periods = j.P;
        if (j.P == 0 || j.bank->nd == 0) continue;
        double dmin = __builtin_huge_val();
        for (uint32_t i = 0; i < j.bank->nd; i++) dmin = rmin(dmin, j.bank->durations[i]);
        const double p_nb = j.nb_period > 0.0 ? j.nb_period : j.periods[j.P - 1];
        j.nb = as_u64(std::ceil((double)j.bank->phase_oversample * p_nb / dmin));
        if (j.nb < 8) j.nb = 8;
        if (j.nb > (1u << 24)) return fail(ctx, FBLS_ERR_ARGUMENT, "phase grid too large");
        j.coarse = j.bank->prescan_factor > 1 && j.nb / j.bank->prescan_factor >= 8;
        Pass p;
        p.r = j.r;
        p.periods = j.periods;
        p.P = j.P;
        p.bank = j.bank;
        p.nb = (uint32_t)(j.coarse ? j.nb / j.bank->prescan_factor : j.nb);
        p.mode = mode;
        j.first = (int)first.size();
        first.push_back(std::move(p));
    }
    // Job launches hold a session's passes together, so a pass's fold needs
    // only its share of the SMs (or, tuned, no cut at all).
    auto share = [&](std::vector<Pass>& passes) {
        if (!fused) return;
        const int n = (int)passes.size();
        const int ctas = tuned_batch_no_fill() ? 0 : std::max(1, (ctx->sm_count + n - 1) / std::max(n, 1));
        for (Pass& p : passes) p.fill_ctas = ctas;
    };
    share(first);
    int rc = plan_passes(ctx, first);
    if (rc) return rc;
    const double t0 = now_seconds();
    rc = session(first, ctx->pin_down);
    if (rc) return rc;
    const double t1 = now_seconds();
    for (BandJob& j : jobs) {
        if (j.first < 0) continue;
        add_pass_stats(j.st, first[j.first]);
        if (first[j.first].bad) {
            j.status = FBLS_ERR_PRECISION;
            continue;
        }
        if (!j.coarse) continue;
        const BandOut& band = first[j.first].out;
        const double cut = j.bank->prescan_fraction * j.bank->threshold;
        for (uint32_t i = 0; i < j.P; i++) {
            const double sc = band.score[i];
            if (std::isfinite(sc) && sc >= cut) j.survivors.push_back(band.records[(size_t)i * RECORD_STRIDE]);
        }
        j.st.prescan_survivors = j.survivors.size();
        if (j.survivors.empty()) continue;
        Pass p;
        p.r = j.r;
        p.periods = j.survivors.data();
        p.P = (uint32_t)j.survivors.size();
        p.bank = j.bank;
        p.nb = (uint32_t)j.nb;
        p.mode = mode;
        j.second = (int)second.size();
        second.push_back(std::move(p));
    }
    share(second);
    rc = plan_passes(ctx, second);
    if (rc) return rc;
    rc = session(second, ctx->pin_down2);
    if (rc) return rc;
    const double t2 = now_seconds();
    uint64_t tmpl_first = 0, tmpl_second = 0;
    for (const Pass& p : first) tmpl_first += p.st.templates_scanned;
    for (const Pass& p : second) tmpl_second += p.st.templates_scanned;
    for (BandJob& j : jobs) {
        if (j.first < 0) continue;
        if (j.second >= 0 && second[j.second].bad) j.status = FBLS_ERR_PRECISION;
        if (j.status) continue;
        j.st.seconds =
            (t1 - t0) * (double)first[j.first].st.templates_scanned / (double)std::max<uint64_t>(tmpl_first, 1);
        const Pass* full = nullptr;
        if (!j.coarse) {
            full = &first[j.first];
        } else if (j.second >= 0) {
            full = &second[j.second];
            add_pass_stats(j.st, *full);
            j.st.seconds +=
                (t2 - t1) * (double)full->st.templates_scanned / (double)std::max<uint64_t>(tmpl_second, 1);
        }
        if (!full) continue;
        for (uint32_t i = 0; i < full->P; i++) {
            const double sc = full->out.score[i];
            if (!(std::isfinite(sc) && sc >= j.bank->threshold)) continue;
            const double* rec = &full->out.records[(size_t)i * RECORD_STRIDE];
            fbls_row row;
            row.period = rec[0];
            row.epoch = (rec[2] + rec[3] / 2.0) / rec[1] + j.r->origin;
            row.duration = rec[3] / rec[1];
            row.score = sc;
            row.depth = full->out.depth[i];
            j.rows->push_back(row);
        }
    }
    return FBLS_OK;
}

// scan_periods (scan.rs:363-408). Rows are appended to `rows`.
int scan_periods(fbls_ctx* ctx, const fbls_ready* r, const double* periods, uint32_t P, const fbls_bank* bank,
                 int mode, std::vector<fbls_row>& rows, fbls_scan_stats* stats) {
    std::vector<BandJob> jobs(1);
    jobs[0].r = r;
    jobs[0].rows = &rows;
    jobs[0].periods = periods;
    jobs[0].P = P;
    jobs[0].bank = bank;
    int rc = scan_bands(ctx, jobs, mode, false);
    if (stats) *stats = jobs[0].st;
    return rc;
}


// The octave bands of signal_search (scan.rs:411-471) for one star: the grid
// periods of each octave [lo, 2 lo) (those inside the [lo, hi) `ranges` when
// any are given) with the durations below lo / 4, each band a BandJob over a
// bank of its own. Jobs are appended to `jobs` with their rows going to
// `rows`; they point into `sb`, which must outlive them. Touches no shared
// state (a rejection's message goes to `err`), so stars are planned in
// parallel.
struct StarBands {
    struct Band {
        std::vector<double> periods, durations, rho;
        double nb_period = 0.0;  // the octave's last grid period (sets nb)
        fbls_bank bank{};
    };
    std::vector<Band> bands;
    uint64_t grid_len = 0;
};

int plan_star_bands(std::string& err, const fbls_ready* ready, const double* durations, const double* rho,
                    uint32_t nd, const fbls_config* cfg, const double* ranges, uint32_t n_ranges, double budget_mib,
                    StarBands& sb, std::vector<BandJob>& jobs, std::vector<fbls_row>* rows) {
    sb.bands.clear();
    sb.grid_len = 0;
    if (nd == 0) {
        err = "no durations";
        return FBLS_ERR_ARGUMENT;
    }
    if (!durations || !rho || !cfg) {
        err = "null argument";
        return FBLS_ERR_ARGUMENT;
    }
    for (uint32_t i = 0; i < nd; i++)
        if (!(durations[i] > 0.0) || !std::isfinite(durations[i])) {
            err = "durations must be positive and finite";
            return FBLS_ERR_ARGUMENT;
        }
    auto kept = [&](double p) {
        if (!n_ranges) return true;
        for (uint32_t i = 0; i < n_ranges; i++)
            if (p >= ranges[2 * i] && p < ranges[2 * i + 1]) return true;
        return false;
    };
    // Durations sorted with rho carried along (scan.rs:418-424).
    std::vector<std::pair<double, double>> ds(nd);
    for (uint32_t i = 0; i < nd; i++) ds[i] = {durations[i], rho[i]};
    std::stable_sort(ds.begin(), ds.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    const double baseline = ready->t_last;
    const double maximum = rmin(cfg->period_max, baseline);
    const double minimum = rmax(cfg->period_min, 4.0 * ds[0].first * (1.0 + 1e-9));
    if (maximum <= minimum) return FBLS_OK;
    const int64_t count = period_grid(minimum, maximum, baseline, ds[0].first, cfg->period_oversample, nullptr, 0);
    if (count < 1) {
        err = "the period grid is infinite or too large";
        return FBLS_ERR_ARGUMENT;
    }
    std::vector<double> grid((size_t)count);
    period_grid(minimum, maximum, baseline, ds[0].first, cfg->period_oversample, grid.data(), count);
    sb.grid_len = (uint64_t)count;
    const double shape_gate = cfg->n_ingress > 0 && cfg->ingress_fractions[0] == 0.0
                                  ? cfg->shape_gate_fraction * cfg->threshold
                                  : 0.0;
    // Octave bands [lo, 2 lo) with the durations below lo / 4 (scan.rs:441-471);
    // every band is scanned by scan_periods, the bands together (scan_bands).
    // Octave k covers [los[k], los[k + 1] = 2 los[k]); one walk over the grid
    // hands every period to its octave, in grid order.
    std::vector<double> los;
    const double last = grid[grid.size() - 1];
    for (double lo = grid[0]; lo <= last; lo *= 2.0) los.push_back(lo);
    std::vector<StarBands::Band> octaves(los.size());
    size_t k = 0;
    for (double p : grid) {
        if (!(p >= los[0] && p < 2.0 * los.back())) continue;
        while (p >= 2.0 * los[k]) k++;
        while (p < los[k]) k--;
        octaves[k].nb_period = p;
        if (kept(p)) octaves[k].periods.push_back(p);
    }
    std::vector<StarBands::Band>& bands = sb.bands;
    for (size_t o = 0; o < octaves.size(); o++) {
        StarBands::Band& b = octaves[o];
        for (auto& d : ds)
            if (d.first < los[o] / 4.0) {
                b.durations.push_back(d.first);
                b.rho.push_back(d.second);
            }
        if (!b.periods.empty() && !b.durations.empty()) bands.push_back(std::move(b));
    }
    const size_t j0 = jobs.size();
    jobs.resize(j0 + bands.size());
    for (size_t i = 0; i < bands.size(); i++) {
        fbls_bank& bank = bands[i].bank;
        bank.durations = bands[i].durations.data();
        bank.rho = bands[i].rho.data();
        bank.nd = (uint32_t)bands[i].durations.size();
        bank.ingress = cfg->ingress_fractions;
        bank.ns = cfg->n_ingress;
        bank.layers = cfg->shape_layers;
        bank.threshold = cfg->threshold;
        bank.shape_gate = shape_gate;
        bank.phase_oversample = cfg->phase_oversample;
        bank.period_batch = cfg->period_batch;
        bank.max_fold_mib = budget_mib;
        bank.prescan_factor = cfg->prescan_factor;
        bank.prescan_fraction = cfg->prescan_fraction;
        BandJob& j = jobs[j0 + i];
        j.r = ready;
        j.rows = rows;
        j.periods = bands[i].periods.data();
        j.P = (uint32_t)bands[i].periods.size();
        j.nb_period = bands[i].nb_period;
        j.bank = &bank;
    }
    return FBLS_OK;
}


// fbls_search_batch with workers == 0: the stars are taken in groups of at
// most FUSED_GROUP_PERIODS grid periods (one star at least). The families of
// a group that are not uploaded yet go up together into ctx->family, and the
// bands of every star of the group are scanned by one scan_bands in fused
// sessions: one fold, one scan and one merge launch per wave, whatever the
// number of stars. Results are the same as one signal_search per star.
constexpr uint64_t FUSED_GROUP_PERIODS = 1u << 21;

int search_batch_fused(fbls_ctx* ctx, fbls_star* stars, uint32_t count, const fbls_config* cfg,
                       std::vector<std::string>& errors) {
    const double budget_mib = fold_budget_mib(cfg->max_fold_mib);
    if (cfg->precision_mode > 2) return fail(ctx, FBLS_ERR_ARGUMENT, "precision_mode must be 0, 1 or 2");
    const int mode = scan_mode(cfg->precision_mode);
    // A star's grid length, from the sizes alone (0 when its inputs are bad),
    // or with period ranges the grid lengths of the ranges: what the groups
    // are cut by.
    auto grid_estimate = [&](const fbls_star& s) -> uint64_t {
        if (!s.durations || !s.nd) return 0;
        const double t_last = s.ready ? s.ready->t_last : (s.time && s.n ? s.time[s.n - 1] : 0.0);
        double dmin = __builtin_huge_val();
        for (uint32_t i = 0; i < s.nd; i++) dmin = rmin(dmin, s.durations[i]);
        const double maximum = rmin(std::isfinite(s.period_max) ? s.period_max : cfg->period_max, t_last);
        const double minimum = rmax(cfg->period_min, 4.0 * dmin * (1.0 + 1e-9));
        if (!(maximum > minimum) || !(dmin > 0.0)) return 0;
        auto count = [&](double lo, double hi) -> uint64_t {
            if (!(hi > lo)) return 0;
            return (uint64_t)std::max<int64_t>(0, period_grid(lo, hi, t_last, dmin, cfg->period_oversample, nullptr, 0));
        };
        if (!s.n_ranges || !s.ranges) return count(minimum, maximum);
        uint64_t est = 0;
        for (uint32_t r = 0; r < s.n_ranges; r++)
            est += count(rmax(minimum, s.ranges[2 * r]), rmin(maximum, s.ranges[2 * r + 1]));
        return est;
    };
    uint32_t i0 = 0;
    while (i0 < count) {
        uint32_t i1 = i0;
        for (uint64_t est = 0; i1 < count && (i1 == i0 || est < FUSED_GROUP_PERIODS); i1++) est += grid_estimate(stars[i1]);
        const uint32_t g = i1 - i0;
        std::vector<fbls_ready> local(g);  // families uploaded for this group
        std::vector<uint8_t> upload(g, 0);  // bytes, not vector<bool>: set from the planning threads
        std::vector<StarBands> sbs(g);
        std::vector<std::vector<fbls_row>> rows(g);
        std::vector<std::vector<BandJob>> star_jobs(g);
        parallel_for(g, [&](size_t k) {
            fbls_star& s = stars[i0 + k];
            s.n_rows = 0;
            s.grid_len = 0;
            s.templates = 0;
            std::string& err = errors[i0 + k];
            const fbls_ready* r = s.ready;
            int rc = FBLS_OK;
            if (!s.durations || !s.rho || (s.n_ranges && !s.ranges)) {
                err = "null argument";
                rc = FBLS_ERR_ARGUMENT;
            }
            if (rc == FBLS_OK && !r) {
                rc = check_family(err, s.time, s.v, s.w, s.n);
                if (rc == FBLS_OK) {
                    fbls_ready& f = local[k];
                    f.ctx = ctx;
                    f.device = ctx->device;
                    f.n = s.n;
                    f.baseline_norm = s.baseline_norm;
                    f.origin = s.origin;
                    f.residual_energy = s.residual_energy;
                    f.t_last = s.time[s.n - 1];
                    f.time_host.assign(s.time, s.time + s.n);
                    f.owned = false;
                    upload[k] = 1;
                    r = &f;
                }
            }
            if (rc == FBLS_OK) {
                fbls_config c = *cfg;
                if (std::isfinite(s.period_max)) c.period_max = s.period_max;
                rc = plan_star_bands(err, r, s.durations, s.rho, s.nd, &c, s.ranges, s.n_ranges, budget_mib, sbs[k],
                                     star_jobs[k], &rows[k]);
                s.grid_len = sbs[k].grid_len;
            }
            s.status = rc;
        });
        std::vector<BandJob> jobs;
        std::vector<uint32_t> job_star;
        std::vector<std::pair<uint32_t, fbls_ready*>> uploads;
        for (uint32_t k = 0; k < g; k++) {
            if (upload[k]) uploads.push_back({i0 + k, &local[k]});
            for (BandJob& j : star_jobs[k]) {
                jobs.push_back(std::move(j));
                job_star.push_back(i0 + k);
            }
        }
        // The group's new families: one copy from page-locked staging, each at
        // a 256-byte aligned offset, zero-padded like upload_family's.
        if (!uploads.empty()) {
            std::vector<size_t> offs;
            size_t total = 0;
            for (auto& u : uploads) {
                offs.push_back(total);
                total += align256(3 * fold_field_stride(u.second->n) * sizeof(double));
            }
            CK(ensure(ctx->family, total), "workspace");
            CK(ensure_pinned(ctx->pin_up, total), "pinned workspace");
            unsigned char* host = static_cast<unsigned char*>(ctx->pin_up.ptr);
            parallel_for(uploads.size(), [&](size_t k) {
                const fbls_star& s = stars[uploads[k].first];
                fbls_ready* f = uploads[k].second;
                const size_t stride = fold_field_stride(f->n);
                double* h = reinterpret_cast<double*>(host + offs[k]);
                const size_t end = (k + 1 < uploads.size() ? offs[k + 1] : total) / sizeof(double);
                std::memset(h, 0, (end - offs[k] / sizeof(double)) * sizeof(double));
                std::memcpy(h, s.time, f->n * sizeof(double));
                std::memcpy(h + stride, s.v, f->n * sizeof(double));
                std::memcpy(h + 2 * stride, s.w, f->n * sizeof(double));
                f->time = reinterpret_cast<double*>(static_cast<unsigned char*>(ctx->family.ptr) + offs[k]);
                f->v = f->time + stride;
                f->w = f->v + stride;
            });
            CK(cudaMemcpyAsync(ctx->family.ptr, host, total, cudaMemcpyHostToDevice, ctx->stream), "upload_ready");
            CK(cudaStreamSynchronize(ctx->stream), "upload_ready");  // the sessions reuse the staging buffer
        }
        const int rc = scan_bands(ctx, jobs, mode, true);
        for (size_t j = 0; j < jobs.size(); j++) {
            fbls_star& s = stars[job_star[j]];
            if (s.status) continue;
            if (rc) {
                s.status = rc;
                errors[job_star[j]] = ctx->error;
            } else if (jobs[j].status) {
                s.status = jobs[j].status;
                errors[job_star[j]] = "nonpositive template precision; inspect noise model";
            } else {
                s.templates += jobs[j].st.templates_scanned;
            }
        }
        for (uint32_t i = i0; i < i1; i++) {
            fbls_star& s = stars[i];
            if (s.status) {
                s.templates = 0;
                continue;
            }
            const std::vector<fbls_row>& rr = rows[i - i0];  // filled by scan_bands
            if (s.rows) std::memcpy(s.rows, rr.data(), std::min<size_t>(rr.size(), s.capacity) * sizeof(fbls_row));
            s.n_rows = (uint32_t)rr.size();
        }
        i0 = i1;
    }
    return FBLS_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" {

const char* fbls_version(void) { return "fbls_b200 0.1 (sm_100a)"; }

fbls_ctx* fbls_create(int device, int* status) {
    fbls_ctx* ctx = new fbls_ctx();
    ctx->device = device;
    ctx->profile = std::getenv("FBLS_PROFILE") != nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    for (int i = 0; i < 4 && e == cudaSuccess; i++) e = cudaEventCreate(&ctx->ev[i]);
    for (int i = 0; i < 2 && e == cudaSuccess; i++) e = cudaEventCreate(&ctx->timer[i]);
    if (e != cudaSuccess) {
        if (status) *status = FBLS_ERR_CUDA;
        delete ctx;
        return nullptr;
    }
    if (status) *status = FBLS_OK;
    return ctx;
}

void fbls_destroy(fbls_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    DevBuf* bufs[] = {&ctx->cum,     &ctx->cum32,    &ctx->hist,     &ctx->parts, &ctx->keys,  &ctx->tflags,
                      &ctx->pass_in, &ctx->pass_out, &ctx->evidence, &ctx->fault, &ctx->family, &ctx->mapbin, &ctx->feat,
                      &ctx->rescore, &ctx->steal};
    for (DevBuf* b : bufs) release(*b);
    for (PinBuf* b : {&ctx->pin_up, &ctx->pin_down, &ctx->pin_down2})
        if (b->ptr) cudaFreeHost(b->ptr);
    for (fbls_ctx* w : ctx->workers) fbls_destroy(w);
    for (int i = 0; i < 4; i++)
        if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
    for (int i = 0; i < 2; i++)
        if (ctx->timer[i]) cudaEventDestroy(ctx->timer[i]);
    for (cudaEvent_t e : ctx->pool) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* fbls_last_error(const fbls_ctx* ctx) { return ctx ? ctx->error.c_str() : "null context"; }

int fbls_timer_start(fbls_ctx* ctx) {
    if (!ctx) return FBLS_ERR_ARGUMENT;
    CK(cudaSetDevice(ctx->device), "set device");
    CK(cudaEventRecord(ctx->timer[0], ctx->stream), "timer");
    return FBLS_OK;
}

int fbls_timer_stop(fbls_ctx* ctx, float* milliseconds) {
    if (!ctx || !milliseconds) return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    CK(cudaSetDevice(ctx->device), "set device");
    CK(cudaEventRecord(ctx->timer[1], ctx->stream), "timer");
    CK(cudaEventSynchronize(ctx->timer[1]), "timer");
    CK(cudaEventElapsedTime(milliseconds, ctx->timer[0], ctx->timer[1]), "timer");
    return FBLS_OK;
}

int fbls_set_kernel_timing(fbls_ctx* ctx, int enable) {
    if (!ctx) return FBLS_ERR_ARGUMENT;
    ctx->kernel_timing = enable != 0;
    return FBLS_OK;
}

int fbls_read_counters(fbls_ctx* ctx, fbls_counters* out, int reset) {
    if (!ctx || !out) return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    *out = ctx->counters;
    if (reset) std::memset(&ctx->counters, 0, sizeof(ctx->counters));
    return FBLS_OK;
}

int fbls_upload_ready(fbls_ctx* ctx, const double* time, const double* v, const double* w, uint32_t n,
                      double baseline_norm, double origin, double residual_energy, fbls_ready** out) {
    if (!ctx || !out) return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    CK(cudaSetDevice(ctx->device), "set device");
    fbls_ready* r = new fbls_ready();
    const int rc = upload_family(ctx, nullptr, time, v, w, n, baseline_norm, origin, residual_energy, r);
    if (rc) {
        delete r;
        return rc;
    }
    *out = r;
    return FBLS_OK;
}

void fbls_free_ready(fbls_ready* r) {
    if (!r) return;
    if (r->owned) {
        cudaSetDevice(r->device);
        cudaFree(r->time);
    }
    delete r;
}

int fbls_scan_bank(fbls_ctx* ctx, const fbls_ready* ready, const double* periods, uint32_t P, const fbls_bank* bank,
                   uint32_t nb, uint32_t precision_mode, double* records, double* score, double* depth,
                   uint32_t* flags, fbls_scan_stats* stats) {
    if (!ctx || !ready || !bank || (P && !periods)) return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    if (precision_mode > 2) return fail(ctx, FBLS_ERR_ARGUMENT, "precision_mode must be 0, 1 or 2");
    CK(cudaSetDevice(ctx->device), "set device");
    fbls_scan_stats st;
    std::memset(&st, 0, sizeof(st));
    st.periods = P;
    if (P == 0) {
        if (stats) *stats = st;
        return FBLS_OK;
    }
    BandOut band;
    int rc = scan_bank(ctx, ready, periods, P, bank, nb, scan_mode(precision_mode), band, &st);
    if (stats) *stats = st;
    if (rc && rc != FBLS_ERR_PRECISION) return rc;
    if (!band.records) return rc;
    if (records) std::memcpy(records, band.records, (size_t)P * RECORD_STRIDE * sizeof(double));
    if (score) std::memcpy(score, band.score, (size_t)P * sizeof(double));
    if (depth) std::memcpy(depth, band.depth, (size_t)P * sizeof(double));
    if (flags) std::memcpy(flags, band.flags, (size_t)P * sizeof(uint32_t));
    return rc;
}

int fbls_scan_periods(fbls_ctx* ctx, const fbls_ready* ready, const double* periods, uint32_t P,
                      const fbls_bank* bank, uint32_t precision_mode, fbls_row* rows_out, uint32_t* n_rows,
                      fbls_scan_stats* stats) {
    if (!ctx || !ready || !bank || !n_rows || (P && (!periods || !rows_out)))
        return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    if (precision_mode > 2) return fail(ctx, FBLS_ERR_ARGUMENT, "precision_mode must be 0, 1 or 2");
    CK(cudaSetDevice(ctx->device), "set device");
    std::vector<fbls_row> rows;
    int rc = scan_periods(ctx, ready, periods, P, bank, scan_mode(precision_mode), rows, stats);
    if (rc) return rc;
    std::memcpy(rows_out, rows.data(), rows.size() * sizeof(fbls_row));
    *n_rows = (uint32_t)rows.size();
    return FBLS_OK;
}

int64_t fbls_period_grid(double minimum, double maximum, double baseline, double minimum_duration, double oversample,
                         double* out, int64_t capacity) {
    return period_grid(minimum, maximum, baseline, minimum_duration, oversample, out, capacity);
}

int fbls_family_state(const double* time, const double* flux, const double* sigma, uint32_t n_in,
                      const double* durations, uint32_t nd, int correlated, uint32_t* n_out, double* time_out,
                      double* v_out, double* w_out, double* scalars_out, double* rho_out, char* error,
                      uint32_t error_len) {
    if (!time || !flux || !sigma || (nd && !durations) || !n_out || !time_out || !v_out || !w_out || !scalars_out ||
        (nd && !rho_out)) {
        if (error && error_len) {
            std::strncpy(error, "null argument", error_len - 1);
            error[error_len - 1] = '\0';
        }
        return FBLS_ERR_ARGUMENT;
    }
    PreparedFamily fam;
    std::string message;
    int rc = prepare_family(time, flux, sigma, n_in, durations, nd, correlated != 0, fam, message);
    if (rc) {
        if (error && error_len) {
            std::strncpy(error, message.c_str(), error_len - 1);
            error[error_len - 1] = '\0';
        }
        return FBLS_ERR_DATA;
    }
    const size_t n = fam.time.size();
    *n_out = (uint32_t)n;
    std::memcpy(time_out, fam.time.data(), n * sizeof(double));
    std::memcpy(v_out, fam.v.data(), n * sizeof(double));
    std::memcpy(w_out, fam.w.data(), n * sizeof(double));
    scalars_out[0] = fam.baseline_norm;
    scalars_out[1] = fam.origin;
    scalars_out[2] = fam.residual_energy;
    scalars_out[3] = fam.inflation;
    scalars_out[4] = (double)fam.segments;
    std::memcpy(rho_out, fam.rho.data(), nd * sizeof(double));
    return FBLS_OK;
}

int fbls_signal_search(fbls_ctx* ctx, const fbls_ready* ready, const double* durations, const double* rho,
                       uint32_t nd, const fbls_config* cfg, fbls_row* rows_out, uint32_t capacity,
                       uint32_t* n_rows, uint64_t* grid_len, fbls_scan_stats* stats_out, uint32_t* n_bands) {
    return fbls_signal_search_ranges(ctx, ready, durations, rho, nd, cfg, nullptr, 0, rows_out, capacity, n_rows,
                                     grid_len, stats_out, n_bands);
}

int fbls_signal_search_ranges(fbls_ctx* ctx, const fbls_ready* ready, const double* durations, const double* rho,
                              uint32_t nd, const fbls_config* cfg, const double* ranges, uint32_t n_ranges,
                              fbls_row* rows_out, uint32_t capacity, uint32_t* n_rows, uint64_t* grid_len,
                              fbls_scan_stats* stats_out, uint32_t* n_bands) {
    if (!ctx || !ready || !durations || !rho || !cfg || !n_rows || (n_ranges && !ranges))
        return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    if (cfg->precision_mode > 2) return fail(ctx, FBLS_ERR_ARGUMENT, "precision_mode must be 0, 1 or 2");
    CK(cudaSetDevice(ctx->device), "set device");
    StarBands sb;
    std::vector<BandJob> jobs;
    std::vector<fbls_row> rows;
    std::string err;
    int rc = plan_star_bands(err, ready, durations, rho, nd, cfg, ranges, n_ranges, fold_budget_mib(cfg->max_fold_mib),
                             sb, jobs, &rows);
    *n_rows = 0;
    if (grid_len) *grid_len = sb.grid_len;
    if (n_bands) *n_bands = 0;
    if (rc) return fail(ctx, rc, err);
    rc = scan_bands(ctx, jobs, scan_mode(cfg->precision_mode), false);
    if (rc) return rc;
    for (size_t i = 0; i < jobs.size() && stats_out && i < 64; i++) stats_out[i] = jobs[i].st;
    const uint32_t n_scanned = (uint32_t)jobs.size();
    // At most `capacity` rows are written; n_rows is the full count, so a
    // caller that sees n_rows > capacity can ask again with room for all.
    if (rows_out) std::memcpy(rows_out, rows.data(), std::min<size_t>(rows.size(), capacity) * sizeof(fbls_row));
    *n_rows = (uint32_t)rows.size();
    if (n_bands) *n_bands = n_scanned;
    return FBLS_OK;
}

int fbls_compare_search(fbls_ctx* ctx, const fbls_ready* ready, const double* durations, const double* rho,
                        uint32_t nd, double period, const fbls_config* cfg, fbls_evidence_row* rows_out,
                        uint32_t* n_rows) {
    if (!ctx || !ready || !durations || !rho || !cfg || !rows_out || !n_rows)
        return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    *n_rows = 0;
    fbls_evidence_job job{};
    job.ready = ready;
    job.period = period;
    job.durations = durations;
    job.rho = rho;
    job.nd = nd;
    const int rc = fbls_compare_batch(ctx, &job, 1, cfg);
    if (rc) return rc;
    for (uint32_t i = 0; i < job.n_rows; i++) rows_out[i] = job.rows[i];
    *n_rows = job.n_rows;
    return FBLS_OK;
}

int fbls_compare_batch(fbls_ctx* ctx, fbls_evidence_job* jobs, uint32_t count, const fbls_config* cfg) {
    if (!ctx || !cfg || (count && !jobs)) return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    if (count == 0) return FBLS_OK;
    CK(cudaSetDevice(ctx->device), "set device");
    std::vector<EvidenceCandidate> cands(count);
    for (uint32_t i = 0; i < count; i++) {
        fbls_evidence_job& J = jobs[i];
        J.n_rows = 0;
        J.status = FBLS_OK;
        EvidenceCandidate& E = cands[i];
        E.durations = J.durations;
        E.rho = J.rho;
        E.nd = J.nd;
        E.period = J.period;
        const fbls_ready* r = J.ready;
        if (r && r->device != ctx->device) {
            J.status = FBLS_ERR_ARGUMENT;
            return fail(ctx, FBLS_ERR_ARGUMENT,
                        "candidate " + std::to_string(i) + ": family uploaded to another device");
        }
        E.r = r ? EvidenceReady{r->time, r->v, r->w, r->n, r->baseline_norm, r->origin, r->residual_energy,
                                r->t_last, r->time_host.data()}
                : EvidenceReady{};
    }
    std::string message;
    uint64_t launched = 0;
    const int rc = compare_batch(ctx->stream, cands.data(), count, *cfg, message,
                                 [&](size_t bytes) -> void* {
                                     if (ensure(ctx->evidence, bytes) != cudaSuccess) return nullptr;
                                     return ctx->evidence.ptr;
                                 },
                                 ctx->sm_count, &launched);
    ctx->counters.launches += launched;
    if (rc) return fail(ctx, rc, message);
    int first = FBLS_OK;
    for (uint32_t i = 0; i < count; i++) {
        fbls_evidence_job& J = jobs[i];
        J.status = cands[i].status;
        J.n_rows = cands[i].n_rows;
        for (uint32_t k = 0; k < J.n_rows; k++) J.rows[k] = cands[i].rows[k];
        if (J.status && first == FBLS_OK) {
            first = J.status;
            fail(ctx, J.status, "candidate " + std::to_string(i) + ": " + cands[i].message);
        }
    }
    return first;
}

// Many stars on one device: `workers` host threads (the caller's included),
// each with its own context (stream, workspace and a reusable buffer for the
// star's observations), take stars from a shared counter and run
// signal_search on them, so one star's host work and small launches overlap
// the others' kernels. The reference runs one star per device worker thread
// (src/batch.rs:61-102) with one context per thread.
int fbls_search_batch(fbls_ctx* ctx, fbls_star* stars, uint32_t count, const fbls_config* cfg, uint32_t workers) {
    if (!ctx || (count && !stars) || !cfg) return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    if (count == 0) return FBLS_OK;
    CK(cudaSetDevice(ctx->device), "set device");
    if (workers == 0) {
        std::vector<std::string> errors(count);
        const int rc = search_batch_fused(ctx, stars, count, cfg, errors);
        if (rc) return rc;
        for (uint32_t i = 0; i < count; i++)
            if (stars[i].status) return fail(ctx, stars[i].status, "star " + std::to_string(i) + ": " + errors[i]);
        return FBLS_OK;
    }
    workers = std::min({workers, count, 64u});
    while (ctx->workers.size() < workers) {
        int status = FBLS_OK;
        fbls_ctx* w = fbls_create(ctx->device, &status);
        if (!w) return fail(ctx, status ? status : FBLS_ERR_CUDA, "batch worker context");
        ctx->workers.push_back(w);
    }
    for (uint32_t k = 0; k < workers; k++) ctx->workers[k]->kernel_timing = ctx->kernel_timing;
    std::atomic<uint32_t> next{0};
    std::vector<std::string> errors(count);
    auto work = [&](fbls_ctx* wc) {
        if (cudaSetDevice(wc->device) != cudaSuccess) return;
        for (;;) {
            const uint32_t i = next.fetch_add(1);
            if (i >= count) break;
            fbls_star& s = stars[i];
            s.n_rows = 0;
            s.grid_len = 0;
            s.templates = 0;
            fbls_ready local;
            const fbls_ready* r = s.ready;
            int rc = FBLS_OK;
            if (!r) {
                rc = upload_family(wc, &wc->family, s.time, s.v, s.w, s.n, s.baseline_norm, s.origin,
                                   s.residual_energy, &local);
                r = &local;
            }
            if (rc == FBLS_OK) {
                fbls_config c = *cfg;
                if (std::isfinite(s.period_max)) c.period_max = s.period_max;
                fbls_scan_stats st[64];
                uint32_t bands = 0;
                rc = fbls_signal_search_ranges(wc, r, s.durations, s.rho, s.nd, &c, s.ranges, s.n_ranges, s.rows,
                                               s.capacity, &s.n_rows, &s.grid_len, st, &bands);
                for (uint32_t b = 0; rc == FBLS_OK && b < bands && b < 64; b++) s.templates += st[b].templates_scanned;
            }
            s.status = rc;
            if (rc) errors[i] = wc->error;
        }
    };
    std::vector<std::thread> threads;
    for (uint32_t k = 1; k < workers; k++) threads.emplace_back(work, ctx->workers[k]);
    work(ctx->workers[0]);
    for (std::thread& t : threads) t.join();
    for (uint32_t k = 0; k < workers; k++) {
        ctx->counters.launches += ctx->workers[k]->counters.launches;
        ctx->counters.fold_launches += ctx->workers[k]->counters.fold_launches;
        ctx->counters.fold_ms += ctx->workers[k]->counters.fold_ms;
        ctx->counters.fold_bytes += ctx->workers[k]->counters.fold_bytes;
        ctx->counters.scan_launches += ctx->workers[k]->counters.scan_launches;
        ctx->counters.scan_ms += ctx->workers[k]->counters.scan_ms;
        ctx->counters.scan_bytes += ctx->workers[k]->counters.scan_bytes;
        ctx->counters.fold_updates += ctx->workers[k]->counters.fold_updates;
        std::memset(&ctx->workers[k]->counters, 0, sizeof(fbls_counters));
    }
    for (uint32_t i = 0; i < count; i++)
        if (stars[i].status) return fail(ctx, stars[i].status, "star " + std::to_string(i) + ": " + errors[i]);
    return FBLS_OK;
}
}  // extern "C"
