// Host driver of the FBLS search path on one B200 and the library's C ABI.
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
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/fbls_b200.h"
#include "common.cuh"
#include "evidence.h"
#include "kernels.h"
#include "prep.h"

using namespace fbls;

namespace {

struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};

struct PinBuf {  // page-locked host memory
    void* ptr = nullptr;
    size_t bytes = 0;
};

}  // namespace

struct fbls_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    std::string error;
    bool profile = false;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    bool kernel_timing = false;
    cudaEvent_t timer[2] = {nullptr, nullptr};
    std::vector<cudaEvent_t> pool;  // per-launch timing events
    fbls_counters counters{};
    // Workspace, grown on demand and reused across bands and calls.
    DevBuf cum, cum32, hist, parts, keys, tflags;  // per launch
    DevBuf pass_in, pass_out;  // per session: every pass's inputs and outputs
    DevBuf evidence, fault;
    DevBuf family;  // observations of the star a batch worker is searching
    DevBuf mapbin;  // time-binned observations of a coarse map
    DevBuf feat;    // the proposal network's input made from coarse maps
    DevBuf rescore; // peak-selection rescoring: rows, masks, times and results
    PinBuf pin_up, pin_down, pin_down2;  // staging of a session's upload and download (two sessions in flight)
    std::vector<fbls_ctx*> workers;  // fbls_search_batch worker contexts, kept for reuse
};

struct fbls_ready {
    fbls_ctx* ctx = nullptr;
    double* time = nullptr;  // n
    double* v = nullptr;     // n
    double* w = nullptr;     // n
    uint32_t n = 0;
    double baseline_norm = 0.0;
    double origin = 0.0;
    double residual_energy = 0.0;
    double t_last = 0.0;
    std::vector<double> time_host;  // for the fold's chunk boundaries
    bool owned = true;              // time/v/w allocated for this handle (else a context's buffer)
};

namespace {

int fail(fbls_ctx* ctx, int status, const std::string& message) {
    if (ctx) ctx->error = message;
    return status;
}

int cuda_fail(fbls_ctx* ctx, cudaError_t e, const char* where) {
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    return fail(ctx, FBLS_ERR_CUDA, m);
}

#define CK(call, where)                                   \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, where); \
    } while (0)

cudaError_t ensure(DevBuf& b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return cudaSuccess;
    if (b.ptr) {
        cudaError_t e = cudaFree(b.ptr);
        if (e != cudaSuccess) return e;
        b.ptr = nullptr;
        b.bytes = 0;
    }
    size_t want = bytes + bytes / 4;
    cudaError_t e = cudaMalloc(&b.ptr, want);
    if (e != cudaSuccess) return e;
    b.bytes = want;
    return cudaSuccess;
}

void release(DevBuf& b) {
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
}

template <typename T>
T* as(DevBuf& b) {
    return reinterpret_cast<T*>(b.ptr);
}

// Checks and uploads a prepared family into `r` (DeviceReady::upload,
// scan.rs:110-124): into a fresh allocation owned by `r` when `buf` is null,
// else into the reusable context buffer `buf` (no allocation once it is
// large enough, so a batch worker never synchronises the device on cudaFree).
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

int upload_family(fbls_ctx* ctx, DevBuf* buf, const double* time, const double* v, const double* w, uint32_t n,
                  double baseline_norm, double origin, double residual_energy, fbls_ready* r) {
    std::string err;
    const int rc = check_family(err, time, v, w, n);
    if (rc) return fail(ctx, rc, err);
    r->ctx = ctx;
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

// Fold budget in MiB: the configured value capped at half of the free device
// memory (Gpu::fold_budget_mib, scan.rs:93-98).
double fold_budget_mib(double configured) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return configured;
    double cap = (double)free_b / 1048576.0 / 2.0;
    return configured < cap ? configured : cap;
}

// A pass's outputs, read in place from its session's page-locked download
// buffer (valid until that buffer serves another session).
struct BandOut {
    const double* records = nullptr;  // P x 9
    const double* score = nullptr;
    const double* depth = nullptr;
    const uint32_t* flags = nullptr;
};

double now_seconds() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

cudaError_t ensure_pinned(PinBuf& b, size_t bytes) {
    if (bytes == 0) bytes = 256;
    if (b.bytes >= bytes) return cudaSuccess;
    if (b.ptr) {
        cudaError_t e = cudaFreeHost(b.ptr);
        if (e != cudaSuccess) return e;
        b.ptr = nullptr;
        b.bytes = 0;
    }
    size_t want = bytes + bytes / 4;
    cudaError_t e = cudaHostAlloc(&b.ptr, want, cudaHostAllocDefault);
    if (e != cudaSuccess) return e;
    b.bytes = want;
    return cudaSuccess;
}

// One scan_bank pass (scan.rs:144-357): every period's best template at nb
// bins. Planned on the host, then enqueued with the other passes of a session.
struct Pass {
    const fbls_ready* r = nullptr;  // the family this pass scans
    const double* periods = nullptr;
    uint32_t P = 0;
    const fbls_bank* bank = nullptr;
    uint32_t nb = 0;
    bool mixed = true;
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
    std::string err;   // plan_pass's message when it rejects the pass
    int fail(int status, const char* message) {
        err = message;
        return status;
    }
};

// Runs f(i) for i in [0, n) on up to 16 host threads, the caller's included.
// Fewer than PARALLEL_MIN items run on the caller's thread: a single star's
// few passes plan in milliseconds, and starting threads for them only adds
// the risk of waiting on a descheduled one when the host's cores are busy.
constexpr size_t PARALLEL_MIN = 32;
template <typename F>
void parallel_for(size_t n, F f) {
    const size_t threads = std::min<size_t>(n, std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
    if (threads <= 1 || n < PARALLEL_MIN) {
        for (size_t i = 0; i < n; i++) f(i);
        return;
    }
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t i; (i = next.fetch_add(1)) < n;) f(i);
    };
    std::vector<std::thread> pool;
    for (size_t k = 1; k < threads; k++) pool.emplace_back(work);
    work();
    for (std::thread& t : pool) t.join();
}

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
    // the histograms never reach device memory), up to 16,384, so bands with
    // few bins fill the GPU with larger period groups. Statistics still count
    // the reference's batches.
    const size_t stride = 2 * (size_t)nb + 1;
    const double launch_period_bytes =
        (double)(NF * stride * (sizeof(double) + sizeof(float2)) +
                 tiles * (PART_STRIDE * sizeof(double) + sizeof(uint64_t) + sizeof(uint32_t)));
    uint64_t launch = (uint64_t)std::floor(bank->max_fold_mib * 1048576.0 / launch_period_bytes);
    launch = std::min<uint64_t>(launch, 16384);
    launch = std::max<uint64_t>(launch / batch, 1) * batch;
    if (launch > p.P) launch = p.P;
    p.batch = batch;
    p.launch = launch;
    p.shape = fold_group_shape((int)nb, (int)launch, ctx->sm_count);
    p.chunks.resize((size_t)r->n + 2);
    const int count = fold_chunks(r->time_host.data(), (int)r->n, scale_max, (int)nb, p.shape.span_cap,
                                  p.shape.chunk_cap, p.chunks.data(), (int)p.chunks.size());
    if (count < 1) return p.fail(FBLS_ERR_ARGUMENT, "fold chunking failed");
    p.chunks.resize((size_t)count + 1);
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
        cum_max = std::max(cum_max, (size_t)p.launch * NF * stride);
        parts_max = std::max(parts_max, (size_t)p.launch * tiles);
        if (!p.shape.hist_in_smem) {
            const size_t blocks = (p.launch + p.shape.group - 1) / p.shape.group;
            hist_max = std::max(hist_max, blocks * p.shape.group * NF * (size_t)p.shape.row_stride);
        }
    }
    CK(ensure(ctx->pass_in, in_total), "workspace");
    CK(ensure(ctx->pass_out, out_total), "workspace");
    CK(ensure(ctx->cum, cum_max * sizeof(double)), "workspace");
    CK(ensure(ctx->cum32, cum_max * sizeof(float2)), "workspace");
    CK(ensure(ctx->parts, parts_max * PART_STRIDE * sizeof(double)), "workspace");
    CK(ensure(ctx->keys, parts_max * sizeof(uint64_t)), "workspace");
    CK(ensure(ctx->tflags, parts_max * sizeof(uint32_t)), "workspace");
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
            if (timing) CK(cudaEventRecord(ctx->pool[3 * li], s), "event");
            CK(launch_fold(fa, p.shape, s), "fold");
            if (timing) CK(cudaEventRecord(ctx->pool[3 * li + 1], s), "event");
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
            sa.mixed = p.mixed ? 1 : 0;
            sa.parts = as<double>(ctx->parts);
            sa.keys = as<uint64_t>(ctx->keys);
            sa.flags = as<uint32_t>(ctx->tflags);
            CK(launch_scan_tiles(sa, n, s), "scan_tiles");
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
            CK(launch_merge(ma, s), "merge");
            if (timing) CK(cudaEventRecord(ctx->pool[3 * li + 2], s), "event");
            ctx->counters.launches += 3;
            ctx->counters.fold_launches += 1;
            ctx->counters.scan_launches += 1;
            ctx->counters.fold_bytes += (double)n * (24.0 * r->n + 48.0 * (double)stride);
            ctx->counters.fold_updates += (uint64_t)n * r->n;
            ctx->counters.scan_bytes += (double)n * (24.0 * (double)stride + 84.0 * tiles);
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
    };
    struct Wave {
        std::vector<Unit> units;
        size_t cum = 0, parts = 0, hist = 0;
        int fold_jobs = 0, fold_ctas = 0, scan_ctas = 0, merge_total = 0;
        size_t smem = 0;
        size_t off_fold = 0, off_fcta = 0, off_scan = 0, off_scta = 0, off_merge = 0, off_mp = 0;  // in the job blob
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
            const size_t cum = (size_t)n * NF * stride, parts = (size_t)n * tiles;
            const bool walk = p.shape.kind == FOLD_WALK;
            const size_t hist = walk ? 0 : ((n + p.shape.group - 1) / p.shape.group) * (size_t)p.shape.group * NF *
                                               (size_t)p.shape.row_stride;
            if (!waves.back().units.empty() && (waves.back().cum + cum) * (sizeof(double) + sizeof(float2)) > WAVE_BYTES)
                waves.emplace_back();
            Wave& w = waves.back();
            w.units.push_back({(int)pi, cursor, n, w.cum, w.parts, w.hist, walk});
            w.cum += cum;
            w.parts += parts;
            w.hist += hist;
            if (walk) {
                w.fold_jobs++;
                w.fold_ctas += (n + p.shape.group - 1) / p.shape.group;
                w.smem = std::max(w.smem, p.shape.smem);
            }
            w.scan_ctas += n * (int)tiles;
            w.merge_total += n;
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
        w.off_fcta = take((w.fold_jobs + 1) * sizeof(int));
        w.off_scan = take(nu * sizeof(ScanArgs));
        w.off_scta = take((nu + 1) * sizeof(int));
        w.off_merge = take(nu * sizeof(MergeArgs));
        w.off_mp = take((nu + 1) * sizeof(int));
    }
    const size_t up_total = in_total + blob;
    CK(ensure(ctx->pass_in, up_total), "workspace");
    CK(ensure(ctx->pass_out, out_total), "workspace");
    CK(ensure(ctx->cum, cum_max * sizeof(double)), "workspace");
    CK(ensure(ctx->cum32, cum_max * sizeof(float2)), "workspace");
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
        ScanArgs* sj = reinterpret_cast<ScanArgs*>(up + in_total + w.off_scan);
        int* sc = reinterpret_cast<int*>(up + in_total + w.off_scta);
        MergeArgs* mj = reinterpret_cast<MergeArgs*>(up + in_total + w.off_merge);
        int* mp = reinterpret_cast<int*>(up + in_total + w.off_mp);
        int nf = 0, fcta = 0, scta = 0, mtot = 0;
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
            fa.cum = as<double>(ctx->cum) + un.cum_off;
            fa.cum32 = as<float2>(ctx->cum32) + un.cum_off;
            fa.hist_global = un.walk ? nullptr : as<double>(ctx->hist) + un.hist_off;
            fa.hist_out = nullptr;
            fa.chunks = d_chunks;
            fa.nchunks = (int)p.chunks.size() - 1;
            fa.stage_field = p.shape.stage_field;
            fa.window = p.shape.window;
            fa.row_stride = p.shape.row_stride;
            fa.fault = as<uint32_t>(ctx->fault);
            if (un.walk) {
                if (!fold_job_ok(fa, p.shape)) return fail(ctx, FBLS_ERR_ARGUMENT, "fold job outside limits");
                fj[nf] = fa;
                fc[nf++] = fcta;
                fcta += (un.n + p.shape.group - 1) / p.shape.group;
            }
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
            sa.mixed = p.mixed ? 1 : 0;
            sa.parts = as<double>(ctx->parts) + un.parts_off * PART_STRIDE;
            sa.keys = as<uint64_t>(ctx->keys) + un.parts_off;
            sa.flags = as<uint32_t>(ctx->tflags) + un.parts_off;
            sj[u] = sa;
            sc[u] = scta;
            scta += un.n * tiles;
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
            mj[u] = ma;
            mp[u] = mtot;
            mtot += un.n;
            ctx->counters.fold_launches += 1;
            ctx->counters.scan_launches += 1;
            ctx->counters.fold_bytes += (double)un.n * (24.0 * r->n + 48.0 * (2.0 * nb + 1.0));
            ctx->counters.fold_updates += (uint64_t)un.n * r->n;
            ctx->counters.scan_bytes += (double)un.n * (24.0 * (2.0 * nb + 1.0) + 84.0 * tiles);
        }
        fc[nf] = fcta;
        sc[w.units.size()] = scta;
        mp[w.units.size()] = mtot;
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
        if (w.fold_jobs)
            CK(launch_fold_jobs(reinterpret_cast<const FoldArgs*>(din + in_total + w.off_fold),
                                reinterpret_cast<const int*>(din + in_total + w.off_fcta), w.fold_jobs, w.fold_ctas,
                                w.smem, s),
               "fold");
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
            CK(launch_fold(fa, p.shape, s), "fold");
        }
        if (timing) CK(cudaEventRecord(ctx->pool[3 * wi + 1], s), "event");
        CK(launch_scan_jobs(reinterpret_cast<const ScanArgs*>(din + in_total + w.off_scan),
                            reinterpret_cast<const int*>(din + in_total + w.off_scta), (int)w.units.size(),
                            w.scan_ctas, s),
           "scan_tiles");
        CK(launch_merge_jobs(reinterpret_cast<const MergeArgs*>(din + in_total + w.off_merge),
                             reinterpret_cast<const int*>(din + in_total + w.off_mp), (int)w.units.size(),
                             w.merge_total, s),
           "merge");
        if (timing) CK(cudaEventRecord(ctx->pool[3 * wi + 2], s), "event");
        ctx->counters.launches += 3;
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
              bool mixed, BandOut& out, fbls_scan_stats* stats) {
    std::vector<Pass> passes(1);
    Pass& p = passes[0];
    p.periods = periods;
    p.P = P;
    p.bank = bank;
    p.nb = nb;
    p.mixed = mixed;
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

int scan_bands(fbls_ctx* ctx, std::vector<BandJob>& jobs, bool mixed, bool fused) {
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
        p.mixed = mixed;
        j.first = (int)first.size();
        first.push_back(std::move(p));
    }
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
        p.mixed = mixed;
        j.second = (int)second.size();
        second.push_back(std::move(p));
    }
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
                 bool mixed, std::vector<fbls_row>& rows, fbls_scan_stats* stats) {
    std::vector<BandJob> jobs(1);
    jobs[0].r = r;
    jobs[0].rows = &rows;
    jobs[0].periods = periods;
    jobs[0].P = P;
    jobs[0].bank = bank;
    int rc = scan_bands(ctx, jobs, mixed, false);
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
    const bool mixed = cfg->precision_mode == 0;
    // A star's grid length, from the sizes alone (0 when its inputs are bad):
    // what the groups are cut by.
    auto grid_estimate = [&](const fbls_star& s) -> uint64_t {
        if (!s.durations || !s.nd) return 0;
        const double t_last = s.ready ? s.ready->t_last : (s.time && s.n ? s.time[s.n - 1] : 0.0);
        double dmin = __builtin_huge_val();
        for (uint32_t i = 0; i < s.nd; i++) dmin = rmin(dmin, s.durations[i]);
        const double maximum = rmin(std::isfinite(s.period_max) ? s.period_max : cfg->period_max, t_last);
        const double minimum = rmax(cfg->period_min, 4.0 * dmin * (1.0 + 1e-9));
        if (!(maximum > minimum) || !(dmin > 0.0)) return 0;
        return (uint64_t)std::max<int64_t>(0, period_grid(minimum, maximum, t_last, dmin, cfg->period_oversample,
                                                          nullptr, 0));
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
        const int rc = scan_bands(ctx, jobs, mixed, true);
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


// A coarse map (fbls_coarse_map) planned on the host: its time bins when
// bin_days > 0 (observations whose floor((t - t0) / bin_days) agree, summed at
// their mean time) and its octave groups [lo, 2 lo), each folded at nb =
// max(8, ceil(oversample * (group's longest period) / shortest duration)) in
// launches of at most per_launch periods. plan_map writes only the plan, so
// the plans of a batch are made in parallel.
struct MapPlan {
    fbls_map_job* job = nullptr;
    int star = 0;             // index of the job in its batch
    bool need_out = true;     // job->out must be given (else only features are made)
    bool use_bins = false;
    fbls_ready bins;          // the binned family (use_bins); device fields set by run_maps
    std::vector<int> starts;  // nbins + 1 observation offsets of the bins
    struct Group {
        uint32_t i0 = 0, count = 0, nb = 0, per_launch = 0;
        FoldShape shape{};
        std::vector<int> chunks;
        size_t off_scales = 0, off_chunks = 0;
    };
    std::vector<Group> groups;
    size_t off_time = 0, off_starts = 0, in_bytes = 0;  // within the plan's upload region (bank at 0)
    size_t in_off = 0, out_off = 0, bin_off = 0;          // the plan's regions in its run
    std::string err;
    const fbls_ready* ready() const { return use_bins ? &bins : job->ready; }
};

int plan_map(const fbls_ctx* ctx, MapPlan& m) {
    const fbls_map_job& j = *m.job;
    auto bad = [&](int status, const char* message) {
        m.err = message;
        return status;
    };
    if (!j.ready || (j.P && !j.periods) || !j.durations || !j.rho || (m.need_out && !j.out))
        return bad(FBLS_ERR_ARGUMENT, "null argument");
    if (!(j.bin_days >= 0.0)) return bad(FBLS_ERR_ARGUMENT, "bin_days must not be negative");
    if (j.nd < 1 || j.nd > (uint32_t)MAP_MAX_DURATIONS) return bad(FBLS_ERR_ARGUMENT, "1 to 8 map durations");
    if (j.P == 0) return FBLS_OK;
    if (!(j.oversample > 0.0)) return bad(FBLS_ERR_ARGUMENT, "oversample must be positive");
    for (uint32_t i = 0; i < j.P; i++)
        if (!(j.periods[i] > 0.0) || !std::isfinite(j.periods[i]) || (i && !(j.periods[i] > j.periods[i - 1])))
            return bad(FBLS_ERR_ARGUMENT, "periods must be positive, finite and ascending");
    double dmin = __builtin_huge_val();
    for (uint32_t i = 0; i < j.nd; i++) {
        if (!(j.durations[i] > 0.0) || !(j.rho[i] > 0.0)) return bad(FBLS_ERR_ARGUMENT, "bad map duration");
        dmin = rmin(dmin, j.durations[i]);
    }
    const fbls_ready* family = j.ready;
    if (j.bin_days > 0.0) {
        const std::vector<double>& t = family->time_host;
        std::vector<double>& tb = m.bins.time_host;
        tb.clear();
        m.starts.clear();
        for (uint32_t i = 0; i < family->n;) {
            const double b = std::floor((t[i] - t[0]) / j.bin_days);
            uint32_t k = i;
            double sum = 0.0;
            while (k < family->n && std::floor((t[k] - t[0]) / j.bin_days) == b) sum += t[k++];
            m.starts.push_back((int)i);
            tb.push_back(sum / (double)(k - i));
            i = k;
        }
        m.starts.push_back((int)family->n);
        m.use_bins = true;
        m.bins.n = (uint32_t)tb.size();
        m.bins.baseline_norm = family->baseline_norm;
        m.bins.origin = family->origin;
        m.bins.residual_energy = family->residual_energy;
        m.bins.t_last = tb.back();
        m.bins.owned = false;
    }
    const fbls_ready* ready = m.ready();
    size_t in_bytes = align256(2 * j.nd * sizeof(double));
    if (m.use_bins) {
        m.off_time = in_bytes;
        in_bytes += align256(fold_field_stride(m.bins.n) * sizeof(double));
        m.off_starts = in_bytes;
        in_bytes += align256(m.starts.size() * sizeof(int));
    }
    m.groups.clear();
    for (uint32_t i0 = 0; i0 < j.P;) {
        uint32_t i1 = i0 + 1;
        while (i1 < j.P && j.periods[i1] < 2.0 * j.periods[i0]) i1++;
        MapPlan::Group g;
        g.i0 = i0;
        g.count = i1 - i0;
        const uint64_t nb = std::max<uint64_t>(8, as_u64(std::ceil(j.oversample * j.periods[i1 - 1] / dmin)));
        if (nb > (1u << 24)) return bad(FBLS_ERR_ARGUMENT, "phase grid too large");
        g.nb = (uint32_t)nb;
        const double scale_max = (double)nb / j.periods[i0];
        if (std::floor(ready->t_last * scale_max) >= 4294967295.0 - 2.0 * (double)nb - 2.0)
            return bad(FBLS_ERR_ARGUMENT, "phase cell exceeds 32 bits");
        const size_t stride = 2 * (size_t)nb + 1;
        g.per_launch = (uint32_t)std::max<size_t>(1, std::min<size_t>(16384, (512ull << 20) / (NF * stride * 12)));
        g.shape = fold_group_shape((int)nb, (int)std::min(g.count, g.per_launch), ctx->sm_count);
        g.chunks.resize((size_t)ready->n + 2);
        const int c = fold_chunks(ready->time_host.data(), (int)ready->n, scale_max, (int)nb, g.shape.span_cap,
                                  g.shape.chunk_cap, g.chunks.data(), (int)g.chunks.size());
        if (c < 1) return bad(FBLS_ERR_ARGUMENT, "fold chunking failed");
        g.chunks.resize((size_t)c + 1);
        g.off_scales = in_bytes;
        in_bytes += align256(g.count * sizeof(double));
        g.off_chunks = in_bytes;
        in_bytes += align256(g.chunks.size() * sizeof(int));
        m.groups.push_back(std::move(g));
        i0 = i1;
    }
    m.in_bytes = in_bytes;
    return FBLS_OK;
}

// Runs planned maps on ctx->stream: one upload, one launch for every star's
// bins, then waves of fold units (a group's launch of at most per_launch
// periods), each wave one fold launch of the walking folds as jobs, whose
// epilogue computes the box maps from the prefix rows in shared memory, and
// for any other fold (too many bins for the walking fold) its own launch,
// prefix rows in HBM (the wave's share under MAP_WAVE_BYTES) and a box-map
// launch;
// with `feat`, one k_map_features launch writing the maps' network input into
// feat->x (device); one download and one synchronisation; each map is copied
// to its job's out when there is one.
constexpr size_t MAP_WAVE_BYTES = 1536ull << 20;

struct MapFeatures {
    float* x = nullptr;  // device, channels x B x T, zeroed
    int channels = 0, B = 0, T = 0;
    const uint32_t* offsets = nullptr;  // per star
};

int run_maps(fbls_ctx* ctx, const std::vector<MapPlan*>& plans, const MapFeatures* feat) {
    if (plans.empty()) return FBLS_OK;
    struct Unit {
        MapPlan* m;
        const MapPlan::Group* g;
        uint32_t c0;
        int n;
        size_t cum_off, hist_off;
        bool walk;
    };
    struct Wave {
        std::vector<Unit> units;
        size_t cum = 0, hist = 0, smem = 0;
        int fold_jobs = 0, fold_ctas = 0, map_jobs = 0, map_total = 0;
        size_t off_fold = 0, off_fcta = 0, off_map = 0, off_mp = 0;
    };
    size_t in_total = 0, out_total = 0, bin_total = 0;
    int nbinned = 0, bin_total_bins = 0;
    std::vector<Wave> waves(1);
    for (MapPlan* m : plans) {
        m->in_off = in_total;
        in_total += m->in_bytes;
        m->out_off = out_total;
        out_total += align256((size_t)m->job->P * m->job->nd * sizeof(float));
        if (m->use_bins) {
            m->bin_off = bin_total;
            bin_total += align256(2 * fold_field_stride(m->bins.n) * sizeof(double));
            nbinned++;
            bin_total_bins += (int)m->bins.n;
        }
        for (const MapPlan::Group& g : m->groups) {
            const size_t stride = 2 * (size_t)g.nb + 1;
            for (uint32_t c0 = 0; c0 < g.count; c0 += g.per_launch) {
                const int n = (int)std::min(g.count - c0, g.per_launch);
                const bool walk = g.shape.kind == FOLD_WALK;  // box maps in the fold's epilogue: no prefix rows
                const size_t cum = walk ? 0 : (size_t)n * NF * stride;
                const size_t hist = walk ? 0 : ((n + g.shape.group - 1) / g.shape.group) * (size_t)g.shape.group *
                                                   NF * (size_t)g.shape.row_stride;
                if (!waves.back().units.empty() &&
                    (waves.back().cum + cum) * (sizeof(double) + sizeof(float2)) > MAP_WAVE_BYTES)
                    waves.emplace_back();
                Wave& w = waves.back();
                w.units.push_back({m, &g, c0, n, w.cum, w.hist, walk});
                w.cum += cum;
                w.hist += hist;
                if (walk) {
                    w.fold_jobs++;
                    w.fold_ctas += (n + g.shape.group - 1) / g.shape.group;
                    w.smem = std::max(w.smem, g.shape.smem);
                } else {
                    w.map_jobs++;
                    w.map_total += n;
                }
            }
        }
    }
    size_t blob = in_total;
    auto take = [&](size_t bytes) {
        const size_t at = blob;
        blob += align256(bytes);
        return at;
    };
    const size_t off_bins = take(std::max(1, nbinned) * sizeof(BinJob)), off_b0 = take((nbinned + 1) * sizeof(int));
    const size_t off_feat = take(plans.size() * sizeof(FeatJob));
    size_t cum_max = 0, hist_max = 0;
    for (Wave& w : waves) {
        cum_max = std::max(cum_max, w.cum);
        hist_max = std::max(hist_max, w.hist);
        w.off_fold = take(std::max(1, w.fold_jobs) * sizeof(FoldArgs));
        w.off_fcta = take((w.fold_jobs + 1) * sizeof(int));
        w.off_map = take(std::max(1, w.map_jobs) * sizeof(MapArgs));
        w.off_mp = take((w.map_jobs + 1) * sizeof(int));
    }
    CK(ensure(ctx->pass_in, blob), "workspace");
    CK(ensure(ctx->pass_out, out_total), "workspace");
    if (cum_max) {
        CK(ensure(ctx->cum, cum_max * sizeof(double)), "workspace");
        CK(ensure(ctx->cum32, cum_max * sizeof(float2)), "workspace");
    }
    if (hist_max) CK(ensure(ctx->hist, hist_max * sizeof(double)), "workspace");
    if (bin_total) CK(ensure(ctx->mapbin, bin_total), "workspace");
    CK(ensure(ctx->fault, sizeof(uint32_t)), "workspace");
    CK(ensure_pinned(ctx->pin_up, blob), "pinned workspace");
    CK(ensure_pinned(ctx->pin_down, out_total + 256), "pinned workspace");
    unsigned char* up = static_cast<unsigned char*>(ctx->pin_up.ptr);
    unsigned char* din = static_cast<unsigned char*>(ctx->pass_in.ptr);
    unsigned char* dout = static_cast<unsigned char*>(ctx->pass_out.ptr);
    unsigned char* dbin = static_cast<unsigned char*>(ctx->mapbin.ptr);
    BinJob* bj = reinterpret_cast<BinJob*>(up + off_bins);
    int* b0 = reinterpret_cast<int*>(up + off_b0);
    int nb_jobs = 0, nb_bins = 0;
    for (MapPlan* m : plans) {
        const fbls_map_job& j = *m->job;
        unsigned char* b = up + m->in_off;
        std::memcpy(b, j.durations, j.nd * sizeof(double));
        std::memcpy(b + j.nd * sizeof(double), j.rho, j.nd * sizeof(double));
        if (m->use_bins) {
            const size_t stride = fold_field_stride(m->bins.n);
            double* t = reinterpret_cast<double*>(b + m->off_time);
            std::memcpy(t, m->bins.time_host.data(), m->bins.n * sizeof(double));
            std::memset(t + m->bins.n, 0, (stride - m->bins.n) * sizeof(double));
            std::memcpy(b + m->off_starts, m->starts.data(), m->starts.size() * sizeof(int));
            m->bins.time = reinterpret_cast<double*>(din + m->in_off + m->off_time);
            m->bins.v = reinterpret_cast<double*>(dbin + m->bin_off);
            m->bins.w = m->bins.v + stride;
            bj[nb_jobs] = {j.ready->v, j.ready->w, reinterpret_cast<const int*>(din + m->in_off + m->off_starts),
                           (int)m->bins.n, m->bins.v, m->bins.w};
            b0[nb_jobs++] = nb_bins;
            nb_bins += (int)m->bins.n;
        }
        for (const MapPlan::Group& g : m->groups) {
            double* sc = reinterpret_cast<double*>(b + g.off_scales);
            for (uint32_t i = 0; i < g.count; i++) sc[i] = (double)g.nb / j.periods[g.i0 + i];
            std::memcpy(b + g.off_chunks, g.chunks.data(), g.chunks.size() * sizeof(int));
        }
    }
    b0[nb_jobs] = nb_bins;
    FeatJob* fjobs = reinterpret_cast<FeatJob*>(up + off_feat);
    bool any_out = false;
    for (size_t k = 0; k < plans.size(); k++) {
        const MapPlan* m = plans[k];
        any_out = any_out || m->job->out;
        fjobs[k] = {reinterpret_cast<const float*>(dout + m->out_off), (int)m->job->P, (int)m->job->nd, m->star,
                    feat ? (int)feat->offsets[m->star] : 0};
    }
    std::vector<FoldArgs> own;  // folds that are not walking folds: their own launches
    std::vector<const FoldShape*> own_shape;
    std::vector<size_t> own_wave;
    for (size_t wi = 0; wi < waves.size(); wi++) {
        Wave& w = waves[wi];
        FoldArgs* fj = reinterpret_cast<FoldArgs*>(up + w.off_fold);
        int* fc = reinterpret_cast<int*>(up + w.off_fcta);
        MapArgs* mj = reinterpret_cast<MapArgs*>(up + w.off_map);
        int* mp = reinterpret_cast<int*>(up + w.off_mp);
        int nf = 0, fcta = 0, nm = 0, mtot = 0;
        for (size_t u = 0; u < w.units.size(); u++) {
            const Unit& un = w.units[u];
            const MapPlan& m = *un.m;
            const MapPlan::Group& g = *un.g;
            const fbls_ready* r = m.ready();
            const unsigned char* b = din + m.in_off;
            FoldArgs fa{};
            fa.time = r->time;
            fa.v = r->v;
            fa.w = r->w;
            fa.scales = reinterpret_cast<const double*>(b + g.off_scales) + un.c0;
            fa.n = (int)r->n;
            fa.nb = (int)g.nb;
            fa.periods = un.n;
            fa.group = g.shape.group;
            fa.cum = un.walk ? nullptr : as<double>(ctx->cum) + un.cum_off;
            fa.cum32 = un.walk ? nullptr : as<float2>(ctx->cum32) + un.cum_off;
            fa.hist_global = un.walk ? nullptr : as<double>(ctx->hist) + un.hist_off;
            fa.hist_out = nullptr;
            fa.chunks = reinterpret_cast<const int*>(b + g.off_chunks);
            fa.nchunks = (int)g.chunks.size() - 1;
            fa.stage_field = g.shape.stage_field;
            fa.window = g.shape.window;
            fa.row_stride = g.shape.row_stride;
            fa.fault = as<uint32_t>(ctx->fault);
            float* out = reinterpret_cast<float*>(dout + m.out_off) + (size_t)(g.i0 + un.c0) * m.job->nd;
            if (un.walk) {
                fa.map_out = out;
                fa.map_durations = reinterpret_cast<const double*>(b);
                fa.map_rho = reinterpret_cast<const double*>(b) + m.job->nd;
                fa.map_nd = (int)m.job->nd;
                fa.map_baseline = r->baseline_norm;
                if (!fold_job_ok(fa, g.shape)) return fail(ctx, FBLS_ERR_ARGUMENT, "fold job outside limits");
                fj[nf] = fa;
                fc[nf++] = fcta;
                fcta += (un.n + g.shape.group - 1) / g.shape.group;
            } else {
                own.push_back(fa);
                own_shape.push_back(&g.shape);
                own_wave.push_back(wi);
            }
            if (!un.walk) {
                MapArgs ma{};
                ma.cum = fa.cum;
                ma.scales = fa.scales;
                ma.durations = reinterpret_cast<const double*>(b);
                ma.rho = reinterpret_cast<const double*>(b) + m.job->nd;
                ma.nd = (int)m.job->nd;
                ma.nb = (int)g.nb;
                ma.baseline = r->baseline_norm;
                ma.n = (double)r->n;
                ma.out = out;
                mj[nm] = ma;
                mp[nm++] = mtot;
                mtot += un.n;
            }
            ctx->counters.fold_updates += (uint64_t)un.n * r->n;
        }
        fc[nf] = fcta;
        mp[nm] = mtot;
    }
    cudaStream_t s = ctx->stream;
    CK(cudaMemsetAsync(ctx->fault.ptr, 0, sizeof(uint32_t), s), "workspace");
    if (bin_total) CK(cudaMemsetAsync(ctx->mapbin.ptr, 0, bin_total, s), "workspace");
    CK(cudaMemcpyAsync(din, up, blob, cudaMemcpyHostToDevice, s), "upload");
    if (nb_jobs) {
        CK(launch_bin_fields_jobs(reinterpret_cast<const BinJob*>(din + off_bins),
                                  reinterpret_cast<const int*>(din + off_b0), nb_jobs, nb_bins, s),
           "bins");
        ctx->counters.launches += 1;
    }
    size_t oi = 0;
    for (size_t wi = 0; wi < waves.size(); wi++) {
        const Wave& w = waves[wi];
        if (w.fold_jobs) {
            CK(launch_fold_jobs(reinterpret_cast<const FoldArgs*>(din + w.off_fold),
                                reinterpret_cast<const int*>(din + w.off_fcta), w.fold_jobs, w.fold_ctas, w.smem, s),
               "fold");
            ctx->counters.launches += 1;
        }
        for (; oi < own.size() && own_wave[oi] == wi; oi++) {
            CK(launch_fold(own[oi], *own_shape[oi], s), "fold");
            ctx->counters.launches += 1;
        }
        if (w.map_jobs) {
            CK(launch_box_map_jobs(reinterpret_cast<const MapArgs*>(din + w.off_map),
                                   reinterpret_cast<const int*>(din + w.off_mp), w.map_jobs, w.map_total, s),
               "box map");
            ctx->counters.launches += 1;
        }
    }
    if (feat) {
        CK(launch_map_features(reinterpret_cast<const FeatJob*>(din + off_feat), (int)plans.size(), feat->channels,
                               feat->B, feat->T, feat->x, s),
           "map features");
        ctx->counters.launches += 1;
    }
    unsigned char* down = static_cast<unsigned char*>(ctx->pin_down.ptr);
    if (any_out) CK(cudaMemcpyAsync(down, dout, out_total, cudaMemcpyDeviceToHost, s), "download");
    CK(cudaMemcpyAsync(down + out_total, ctx->fault.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "download");
    CK(cudaStreamSynchronize(s), "coarse map");
    uint32_t fault = 0;
    std::memcpy(&fault, down + out_total, sizeof(uint32_t));
    if (fault) return fail(ctx, FBLS_ERR_CUDA, "fold: staging copies did not complete");
    for (MapPlan* m : plans)
        if (m->job->out) std::memcpy(m->job->out, down + m->out_off, (size_t)m->job->P * m->job->nd * sizeof(float));
    return FBLS_OK;
}

// Plans (in parallel) and runs the maps of `jobs` on ctx, in runs of at most
// MAP_RUN_PERIODS periods; every job's status is set, a failing job's message
// goes to errors[i]. Returns a failure of the device work itself, else 0.
constexpr uint64_t MAP_RUN_PERIODS = 1u << 22;

int coarse_maps(fbls_ctx* ctx, fbls_map_job* jobs, uint32_t count, std::vector<std::string>& errors,
                const MapFeatures* feat = nullptr) {
    std::vector<MapPlan> plans(count);
    std::vector<int> rc(count, FBLS_OK);
    for (uint32_t i = 0; i < count; i++) {
        plans[i].job = &jobs[i];
        plans[i].star = (int)i;
        plans[i].need_out = feat == nullptr;
    }
    parallel_for(count, [&](size_t i) { rc[i] = plan_map(ctx, plans[i]); });
    std::vector<MapPlan*> run;
    uint64_t periods = 0;
    for (uint32_t i = 0; i <= count; i++) {
        if (i == count || (!run.empty() && periods + jobs[i].P > MAP_RUN_PERIODS)) {
            const int e = run_maps(ctx, run, feat);
            if (e) {
                for (MapPlan* m : run) {
                    m->job->status = e;
                    errors[m->job - jobs] = ctx->error;
                }
                return e;
            }
            run.clear();
            periods = 0;
            if (i == count) break;
        }
        jobs[i].status = rc[i];
        if (rc[i]) {
            errors[i] = plans[i].err;
            continue;
        }
        if (plans[i].groups.empty()) continue;
        run.push_back(&plans[i]);
        periods += jobs[i].P;
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
                      &ctx->rescore};
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
        if (r->ctx) cudaSetDevice(r->ctx->device);
        cudaFree(r->time);
    }
    delete r;
}

int fbls_scan_bank(fbls_ctx* ctx, const fbls_ready* ready, const double* periods, uint32_t P, const fbls_bank* bank,
                   uint32_t nb, uint32_t precision_mode, double* records, double* score, double* depth,
                   uint32_t* flags, fbls_scan_stats* stats) {
    if (!ctx || !ready || !bank || (P && !periods)) return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    CK(cudaSetDevice(ctx->device), "set device");
    fbls_scan_stats st;
    std::memset(&st, 0, sizeof(st));
    st.periods = P;
    if (P == 0) {
        if (stats) *stats = st;
        return FBLS_OK;
    }
    BandOut band;
    int rc = scan_bank(ctx, ready, periods, P, bank, nb, precision_mode == 0, band, &st);
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
    CK(cudaSetDevice(ctx->device), "set device");
    std::vector<fbls_row> rows;
    int rc = scan_periods(ctx, ready, periods, P, bank, precision_mode == 0, rows, stats);
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
    rc = scan_bands(ctx, jobs, cfg->precision_mode == 0, false);
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
    CK(cudaSetDevice(ctx->device), "set device");
    EvidenceReady er{ready->time, ready->v, ready->w, ready->n, ready->baseline_norm, ready->origin,
                     ready->residual_energy, ready->t_last, ready->time_host.data()};
    std::string message;
    int rc = compare_search(ctx->stream, ctx->evidence.ptr, ctx->evidence.bytes, er, durations, rho, nd, period, *cfg,
                            rows_out, n_rows, message, [&](size_t bytes) -> void* {
                                if (ensure(ctx->evidence, bytes) != cudaSuccess) return nullptr;
                                return ctx->evidence.ptr;
                            });
    if (rc) return fail(ctx, rc, message);
    return FBLS_OK;
}

// Coarse periodogram of a family for the proposal network (plan_map, then
// run_maps: the octave groups' folds and box maps as job launches).
int fbls_coarse_map(fbls_ctx* ctx, const fbls_ready* family, const double* periods, uint32_t P,
                    const double* durations, const double* rho, uint32_t nd, double oversample, double bin_days,
                    float* out) {
    if (!ctx) return FBLS_ERR_ARGUMENT;
    CK(cudaSetDevice(ctx->device), "set device");
    fbls_map_job job{family, periods, P, durations, rho, nd, oversample, bin_days, out, FBLS_OK};
    std::vector<std::string> errors(1);
    const int rc = coarse_maps(ctx, &job, 1, errors);
    if (rc) return rc;
    if (job.status) return fail(ctx, job.status, errors[0]);
    return FBLS_OK;
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

// single_event_search (events.rs:18-153): the durations sorted with their
// rho, one trial period baseline + 2 (longest duration) + 1e-6 d (longer than
// the data, so nothing wraps), nb = max(8, ceil(phase_oversample * trial /
// shortest duration)); the family folded at that period by the fold kernels,
// then k_scan_all keeps every template whose exact score reaches the
// threshold. Rows (period +inf, epoch, duration, score, depth) come out
// ordered by (phase, duration, shape); past `capacity` survivors the rows are
// dropped and `overflow` set, as the reference does.
int fbls_single_event_search(fbls_ctx* ctx, const fbls_ready* ready, const double* durations, const double* rho,
                             uint32_t nd, const fbls_config* cfg, uint32_t capacity, fbls_row* rows_out,
                             uint32_t* n_rows, fbls_event_stats* stats) {
    if (!ctx || !ready || !durations || !rho || !cfg || !n_rows || (capacity && !rows_out))
        return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    if (nd == 0 || nd > (uint32_t)MAX_DURATIONS) return fail(ctx, FBLS_ERR_ARGUMENT, "1 to 64 durations");
    if (cfg->n_ingress < 1 || cfg->n_ingress > (uint32_t)MAX_SHAPES || cfg->shape_layers < 1 ||
        cfg->shape_layers > (uint32_t)MAX_LAYERS)
        return fail(ctx, FBLS_ERR_ARGUMENT, "bank size outside the supported range");
    *n_rows = 0;
    CK(cudaSetDevice(ctx->device), "set device");
    std::vector<std::pair<double, double>> ds(nd);
    for (uint32_t i = 0; i < nd; i++) ds[i] = {durations[i], rho[i]};
    std::stable_sort(ds.begin(), ds.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    if (!(ds[0].first > 0.0)) return fail(ctx, FBLS_ERR_ARGUMENT, "durations must be positive");
    const double trial = ready->t_last + 2.0 * ds[nd - 1].first + 1e-6;
    const uint64_t nb64 = std::max<uint64_t>(8, as_u64(std::ceil((double)cfg->phase_oversample * trial / ds[0].first)));
    if (nb64 > (1u << 24)) return fail(ctx, FBLS_ERR_ARGUMENT, "phase grid too large");
    const int nb = (int)nb64;
    const double scale = (double)nb / trial;
    const uint32_t ns = cfg->n_ingress, layers = cfg->shape_layers;
    std::vector<double> bank;  // durations | rho | ingress | factors (scan.rs:157-171)
    for (auto& d : ds) bank.push_back(d.first);
    for (auto& d : ds) bank.push_back(d.second);
    bank.insert(bank.end(), cfg->ingress_fractions, cfg->ingress_fractions + ns);
    for (uint32_t si = 0; si < ns; si++)
        for (uint32_t l = 0; l < layers; l++)
            bank.push_back(1.0 - 2.0 * cfg->ingress_fractions[si] *
                                     (layers > 1 ? (double)l / (double)(layers - 1) : 0.0));
    const FoldShape shape = fold_group_shape(nb, 1, ctx->sm_count);
    std::vector<int> chunks((size_t)ready->n + 2);
    const int count = fold_chunks(ready->time_host.data(), (int)ready->n, scale, nb, shape.span_cap,
                                  shape.chunk_cap, chunks.data(), (int)chunks.size());
    if (count < 1) return fail(ctx, FBLS_ERR_ARGUMENT, "fold chunking failed");
    chunks.resize((size_t)count + 1);
    const size_t stride = 2 * (size_t)nb + 1;
    const size_t o_scale = 0, o_bank = 256, o_chunks = o_bank + align256(bank.size() * sizeof(double)),
                 in_total = o_chunks + align256(chunks.size() * sizeof(int));
    const size_t o_counter = 0, o_rec = 256, out_total = o_rec + align256((size_t)capacity * EVENT_RECORD * 8 + 8);
    CK(ensure(ctx->pass_in, in_total), "workspace");
    CK(ensure(ctx->pass_out, out_total), "workspace");
    CK(ensure(ctx->cum, NF * stride * sizeof(double)), "workspace");
    CK(ensure(ctx->cum32, NF * stride * sizeof(float2)), "workspace");
    if (!shape.hist_in_smem) CK(ensure(ctx->hist, (size_t)shape.group * NF * shape.row_stride * sizeof(double)),
                                "workspace");
    CK(ensure(ctx->fault, sizeof(uint32_t)), "workspace");
    CK(ensure_pinned(ctx->pin_up, in_total), "pinned workspace");
    unsigned char* up = static_cast<unsigned char*>(ctx->pin_up.ptr);
    std::memcpy(up + o_scale, &scale, sizeof(double));
    std::memcpy(up + o_bank, bank.data(), bank.size() * sizeof(double));
    std::memcpy(up + o_chunks, chunks.data(), chunks.size() * sizeof(int));
    unsigned char* din = static_cast<unsigned char*>(ctx->pass_in.ptr);
    unsigned char* dout = static_cast<unsigned char*>(ctx->pass_out.ptr);
    cudaStream_t s = ctx->stream;
    CK(cudaMemsetAsync(ctx->fault.ptr, 0, sizeof(uint32_t), s), "workspace");
    CK(cudaMemsetAsync(dout + o_counter, 0, sizeof(uint32_t), s), "workspace");
    CK(cudaMemcpyAsync(din, up, in_total, cudaMemcpyHostToDevice, s), "upload");
    FoldArgs fa{};
    fa.time = ready->time;
    fa.v = ready->v;
    fa.w = ready->w;
    fa.scales = reinterpret_cast<const double*>(din + o_scale);
    fa.n = (int)ready->n;
    fa.nb = nb;
    fa.periods = 1;
    fa.group = shape.group;
    fa.cum = as<double>(ctx->cum);
    fa.cum32 = as<float2>(ctx->cum32);
    fa.hist_global = shape.hist_in_smem ? nullptr : as<double>(ctx->hist);
    fa.chunks = reinterpret_cast<const int*>(din + o_chunks);
    fa.nchunks = count;
    fa.stage_field = shape.stage_field;
    fa.window = shape.window;
    fa.row_stride = shape.row_stride;
    fa.fault = as<uint32_t>(ctx->fault);
    const bool timing = ctx->profile || ctx->kernel_timing;
    if (timing) CK(cudaEventRecord(ctx->ev[0], s), "event");
    CK(launch_fold(fa, shape, s), "fold");
    if (timing) CK(cudaEventRecord(ctx->ev[1], s), "event");
    const double* d_bank = reinterpret_cast<const double*>(din + o_bank);
    EventArgs ea{};
    ea.cum = fa.cum;
    ea.durations = d_bank;
    ea.rho = d_bank + nd;
    ea.ingress = d_bank + 2 * nd;
    ea.factors = d_bank + 2 * nd + ns;
    ea.scale = scale;
    ea.baseline = ready->baseline_norm;
    ea.threshold = cfg->threshold;
    ea.n = (double)ready->n;
    ea.nb = nb;
    ea.nd = (int)nd;
    ea.ns = (int)ns;
    ea.layers = (int)layers;
    ea.capacity = capacity;
    ea.counter = reinterpret_cast<uint32_t*>(dout + o_counter);
    ea.records = reinterpret_cast<double*>(dout + o_rec);
    CK(launch_scan_all(ea, s), "scan_all");
    if (timing) CK(cudaEventRecord(ctx->ev[2], s), "event");
    ctx->counters.launches += 2;
    ctx->counters.fold_launches += 1;
    ctx->counters.scan_launches += 1;
    uint32_t found = 0, fault = 0;
    CK(cudaMemcpyAsync(&found, dout + o_counter, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "download");
    CK(cudaMemcpyAsync(&fault, ctx->fault.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "download");
    CK(cudaStreamSynchronize(s), "single_event_search");
    if (fault) return fail(ctx, FBLS_ERR_CUDA, "fold: staging copies did not complete");
    if (timing) {
        float f_ms = 0.f, s_ms = 0.f;
        CK(cudaEventElapsedTime(&f_ms, ctx->ev[0], ctx->ev[1]), "event");
        CK(cudaEventElapsedTime(&s_ms, ctx->ev[1], ctx->ev[2]), "event");
        ctx->counters.fold_ms += f_ms;
        ctx->counters.scan_ms += s_ms;
    }
    ctx->counters.fold_updates += ready->n;
    if (stats) {
        stats->templates_scanned = (uint64_t)nb * nd * ns;
        stats->threshold_survivors = found;
        stats->overflow = found > capacity ? 1 : 0;
    }
    if (found > capacity || found == 0) return FBLS_OK;
    std::vector<double> rec((size_t)found * EVENT_RECORD);
    CK(cudaMemcpyAsync(rec.data(), dout + o_rec, rec.size() * sizeof(double), cudaMemcpyDeviceToHost, s),
       "download");
    CK(cudaStreamSynchronize(s), "single_event_search");
    std::vector<uint32_t> order(found);
    for (uint32_t i = 0; i < found; i++) order[i] = i;
    auto key = [&](uint32_t i) {
        const double* r = &rec[(size_t)i * EVENT_RECORD];
        return std::make_tuple(r[0], r[4], r[5]);
    };
    std::sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return key(x) < key(y); });
    for (uint32_t m = 0; m < found; m++) {
        const double* r = &rec[(size_t)order[m] * EVENT_RECORD];
        fbls_row& row = rows_out[m];
        row.period = __builtin_huge_val();
        row.epoch = (r[0] + r[1] / 2.0) / scale + ready->origin;
        row.duration = r[1] / scale;
        row.score = r[2];
        row.depth = r[3];
    }
    *n_rows = found;
    return FBLS_OK;
}

// biweight_flatten_gpu (src/prep/curve.rs:256-329): window bounds per
// observation from the sorted times (segments split where the time step
// exceeds `gap`), blocks of up to 128 observations whose windows' union fits
// the shared-memory stage, one k_biweight launch. A window wider than the
// stage is read from global memory by a block of its own, so every window
// runs on the GPU (the reference sends a curve with one such window to its
// CPU implementation, which gives the same values).
int fbls_biweight_flatten(fbls_ctx* ctx, const double* time, const double* relative_flux, uint32_t n, double window,
                          double gap, double c, uint32_t iterations, double* out) {
    if (!ctx || (n && (!time || !relative_flux || !out))) return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    if (n == 0) return FBLS_OK;
    if (!(window >= 0.0) || !(gap >= 0.0)) return fail(ctx, FBLS_ERR_ARGUMENT, "window and gap must not be negative");
    for (uint32_t i = 1; i < n; i++)
        if (!(time[i] >= time[i - 1])) return fail(ctx, FBLS_ERR_ARGUMENT, "times must be ascending");
    CK(cudaSetDevice(ctx->device), "set device");
    std::vector<uint32_t> lo(n), hi(n);
    std::vector<std::pair<uint32_t, uint32_t>> segs;
    for (uint32_t start = 0, i = 1; i <= n; i++)
        if (i == n || time[i] - time[i - 1] > gap) {
            segs.push_back({start, i});
            start = i;
        }
    parallel_for(segs.size(), [&](size_t sgi) {
        const uint32_t a = segs[sgi].first, b = segs[sgi].second;
        const double* t0 = time + a;
        const double* t1 = time + b;
        for (uint32_t j = a; j < b; j++) {
            lo[j] = a + (uint32_t)(std::lower_bound(t0, t1, time[j] - window / 2.0) - t0);
            hi[j] = a + (uint32_t)(std::upper_bound(t0, t1, time[j] + window / 2.0) - t0);
        }
    });
    std::vector<uint32_t> blocks;
    size_t smem = 0;
    for (uint32_t first = 0; first < n;) {
        uint32_t count = 1;
        while (count < (uint32_t)BIWEIGHT_THREADS && first + count < n &&
               hi[first + count] - lo[first] <= (uint32_t)BIWEIGHT_STAGE)
            count++;
        const uint32_t ulo = lo[first], uhi = hi[first + count - 1];
        if (uhi - ulo <= (uint32_t)BIWEIGHT_STAGE) smem = std::max(smem, (size_t)(uhi - ulo) * sizeof(double));
        blocks.insert(blocks.end(), {first, count, ulo, uhi});
        first += count;
    }
    const size_t nblocks = blocks.size() / 4;
    const size_t o_flux = 0, o_lo = align256((size_t)n * 8), o_hi = o_lo + align256((size_t)n * 4),
                 o_blk = o_hi + align256((size_t)n * 4), o_out = o_blk + align256(blocks.size() * 4),
                 total = o_out + align256((size_t)n * 8);
    CK(ensure(ctx->pass_in, total), "workspace");
    CK(ensure_pinned(ctx->pin_up, o_out), "pinned workspace");
    unsigned char* up = static_cast<unsigned char*>(ctx->pin_up.ptr);
    double* fl = reinterpret_cast<double*>(up + o_flux);
    for (uint32_t i = 0; i < n; i++) fl[i] = 1.0 + relative_flux[i];
    std::memcpy(up + o_lo, lo.data(), (size_t)n * 4);
    std::memcpy(up + o_hi, hi.data(), (size_t)n * 4);
    std::memcpy(up + o_blk, blocks.data(), blocks.size() * 4);
    unsigned char* d = static_cast<unsigned char*>(ctx->pass_in.ptr);
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(d, up, o_out, cudaMemcpyHostToDevice, s), "upload");
    BiweightArgs a{};
    a.flux = reinterpret_cast<const double*>(d + o_flux);
    a.lo = reinterpret_cast<const uint32_t*>(d + o_lo);
    a.hi = reinterpret_cast<const uint32_t*>(d + o_hi);
    a.blocks = reinterpret_cast<const uint32_t*>(d + o_blk);
    a.c = c;
    a.iterations = (int)iterations;
    a.out = reinterpret_cast<double*>(d + o_out);
    const bool timing = ctx->profile || ctx->kernel_timing;
    if (timing) CK(cudaEventRecord(ctx->ev[0], s), "event");
    CK(launch_biweight(a, (int)nblocks, smem, s), "biweight");
    if (timing) CK(cudaEventRecord(ctx->ev[1], s), "event");
    ctx->counters.launches += 1;
    CK(cudaMemcpyAsync(out, d + o_out, (size_t)n * 8, cudaMemcpyDeviceToHost, s), "download");
    CK(cudaStreamSynchronize(s), "biweight");
    if (timing) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]), "event");
        ctx->counters.detrend_ms += ms;
    }
    return FBLS_OK;
}

// fit_segment_noise (src/prep/curve.rs:89-198) on the host: the diagonal
// noise model of raw flux. Outputs hold up to n_in values.
int fbls_fit_segment_noise(const double* time, const double* flux, const double* err, const int64_t* group,
                           uint32_t n_in, double bin_minutes, double gap_days, uint32_t* n_out, double* time_out,
                           double* deficit_out, double* variance_out, int64_t* group_out, double* scalars_out,
                           char* error, uint32_t error_len) {
    auto fail_msg = [&](int status, const std::string& message) {
        if (error && error_len) {
            std::strncpy(error, message.c_str(), error_len - 1);
            error[error_len - 1] = '\0';
        }
        return status;
    };
    if (!time || !flux || !n_out || !time_out || !deficit_out || !variance_out || !scalars_out)
        return fail_msg(FBLS_ERR_ARGUMENT, "null argument");
    DiagonalNoise d;
    std::string message;
    if (fit_segment_noise(time, flux, err, group, n_in, bin_minutes, gap_days, d, message))
        return fail_msg(FBLS_ERR_DATA, message);
    const size_t n = d.time.size();
    *n_out = (uint32_t)n;
    std::memcpy(time_out, d.time.data(), n * sizeof(double));
    std::memcpy(deficit_out, d.deficit.data(), n * sizeof(double));
    std::memcpy(variance_out, d.variance.data(), n * sizeof(double));
    if (group_out) std::memcpy(group_out, d.group.data(), n * sizeof(int64_t));
    scalars_out[0] = d.origin;
    scalars_out[1] = d.inflation;
    scalars_out[2] = (double)d.segments;
    return FBLS_OK;
}

// segment_edges and detrending_windows (curve.rs:332-370), host only.
int fbls_segment_edges(const double* time, uint32_t n, double gap, double* out) {
    if (n && (!time || !out)) return FBLS_ERR_ARGUMENT;
    const std::vector<double> e = segment_edges(std::vector<double>(time, time + n), gap);
    std::memcpy(out, e.data(), (size_t)n * sizeof(double));
    return FBLS_OK;
}

int fbls_detrending_windows(const double* durations, uint32_t nd, double minimum, double factor, double maximum,
                            double* windows_out, uint32_t* family_out, uint32_t* n_windows) {
    if (!n_windows || (nd && (!durations || !windows_out || !family_out))) return FBLS_ERR_ARGUMENT;
    const auto w = detrending_windows(durations, nd, minimum, factor, maximum);
    for (size_t k = 0; k < w.size(); k++) {
        windows_out[k] = w[k].first;
        for (uint32_t i : w[k].second) family_out[i] = (uint32_t)k;
    }
    *n_windows = (uint32_t)w.size();
    return FBLS_OK;
}

// prepare_families (src/prep/curve.rs:384-425): the noise model of the raw
// flux (groups, bins of cfg->bin_minutes, gap 0.75 d), then per detrending
// window the biweight detrend on the GPU (gap 0.5 d, c 5, 10 iterations) and
// the curve kept where the detrended flux is finite, at most clip_sigma
// robust scales above zero and at least edge_trim windows from a segment
// edge.
int fbls_prepare_families(fbls_ctx* ctx, const double* time, const double* flux, const double* err,
                          const int64_t* group, uint32_t n, const double* durations, uint32_t nd,
                          const fbls_prep_config* cfg, fbls_family_out* out, uint32_t* n_families) {
    if (!ctx || !time || !flux || !durations || !cfg || !out || !n_families)
        return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    *n_families = 0;
    DiagonalNoise d;
    std::string message;
    if (fit_segment_noise(time, flux, err, group, n, cfg->bin_minutes, 0.75, d, message))
        return fail(ctx, FBLS_ERR_DATA, message);
    const size_t m = d.time.size();
    std::vector<double> sigma(m), relative(m), flat(m);
    for (size_t i = 0; i < m; i++) {
        sigma[i] = std::sqrt(d.variance[i]);
        relative[i] = -d.deficit[i];
    }
    const std::vector<double> edge = segment_edges(d.time, 0.5);
    const auto windows = detrending_windows(durations, nd, cfg->window_min, cfg->window_factor, cfg->window_max);
    for (size_t k = 0; k < windows.size(); k++) {
        const double window = windows[k].first;
        const int rc = fbls_biweight_flatten(ctx, d.time.data(), relative.data(), (uint32_t)m, window, 0.5, 5.0, 10,
                                             flat.data());
        if (rc) return rc;
        const double scale = robust_scale(flat);
        fbls_family_out& f = out[k];
        if (!f.time || !f.flux || !f.sigma || !f.indices) return fail(ctx, FBLS_ERR_ARGUMENT, "null family buffer");
        uint32_t kept = 0;
        for (size_t i = 0; i < m; i++)
            if (std::isfinite(flat[i]) && flat[i] <= cfg->clip_sigma * scale && edge[i] >= cfg->edge_trim * window) {
                f.time[kept] = d.time[i] + d.origin;
                f.flux[kept] = flat[i];
                f.sigma[kept] = sigma[i];
                kept++;
            }
        f.n = kept;
        f.window_days = window;
        f.clipped = (uint32_t)(m - kept);
        f.n_indices = (uint32_t)windows[k].second.size();
        std::memcpy(f.indices, windows[k].second.data(), windows[k].second.size() * sizeof(uint32_t));
    }
    *n_families = (uint32_t)windows.size();
    return FBLS_OK;
}

// Peak-selection rescoring (src/select/peaks.rs:148-252 calls these): the
// rows' box sums over an uploaded family's observations outside `excluded`,
// and their in-transit counts over a time vector. Host arrays in and out;
// one upload, one launch, one download each.
int fbls_rescore_rows(fbls_ctx* ctx, const fbls_ready* family, const uint8_t* excluded, const double* rows,
                      uint32_t R, double* sums) {
    if (!ctx || !family || (family->n && !excluded) || (R && (!rows || !sums)))
        return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    if (R == 0) return FBLS_OK;
    CK(cudaSetDevice(ctx->device), "set device");
    const size_t o_rows = 0, o_sums = align256((size_t)R * 3 * sizeof(double)),
                 o_ex = o_sums + align256((size_t)R * 3 * sizeof(double)),
                 total = o_ex + align256((size_t)family->n + 1);
    CK(ensure(ctx->rescore, total), "workspace");
    unsigned char* d = static_cast<unsigned char*>(ctx->rescore.ptr);
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(d + o_rows, rows, (size_t)R * 3 * sizeof(double), cudaMemcpyHostToDevice, s), "upload");
    if (family->n) CK(cudaMemcpyAsync(d + o_ex, excluded, family->n, cudaMemcpyHostToDevice, s), "upload");
    RescoreArgs a{};
    a.time = family->time;
    a.v = family->v;
    a.w = family->w;
    a.excluded = d + o_ex;
    a.rows = reinterpret_cast<const double*>(d + o_rows);
    a.origin = family->origin;
    a.n = (int)family->n;
    a.R = (int)R;
    a.sums = reinterpret_cast<double*>(d + o_sums);
    const bool timing = ctx->profile || ctx->kernel_timing;
    if (timing) CK(cudaEventRecord(ctx->ev[0], s), "event");
    CK(launch_rescore_rows(a, s), "rescore_rows");
    if (timing) CK(cudaEventRecord(ctx->ev[1], s), "event");
    ctx->counters.launches += 1;
    ctx->counters.rescore_launches += 1;
    CK(cudaMemcpyAsync(sums, d + o_sums, (size_t)R * 3 * sizeof(double), cudaMemcpyDeviceToHost, s), "download");
    CK(cudaStreamSynchronize(s), "rescore_rows");
    if (timing) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]), "event");
        ctx->counters.rescore_ms += ms;
    }
    return FBLS_OK;
}

int fbls_count_rows(fbls_ctx* ctx, const double* time, uint32_t n, const uint8_t* excluded, const double* rows,
                    uint32_t R, uint32_t* counts) {
    if (!ctx || (n && (!time || !excluded)) || (R && (!rows || !counts)))
        return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    for (uint32_t i = 1; i < n; i++)
        if (!(time[i] >= time[i - 1])) return fail(ctx, FBLS_ERR_ARGUMENT, "times must be ascending");
    if (R == 0) return FBLS_OK;
    CK(cudaSetDevice(ctx->device), "set device");
    const size_t o_rows = 0, o_counts = align256((size_t)R * 3 * sizeof(double)),
                 o_time = o_counts + align256((size_t)R * 2 * sizeof(uint32_t)),
                 o_ex = o_time + align256((size_t)n * sizeof(double) + 8), total = o_ex + align256((size_t)n + 1);
    CK(ensure(ctx->rescore, total), "workspace");
    unsigned char* d = static_cast<unsigned char*>(ctx->rescore.ptr);
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(d + o_rows, rows, (size_t)R * 3 * sizeof(double), cudaMemcpyHostToDevice, s), "upload");
    if (n) {
        CK(cudaMemcpyAsync(d + o_time, time, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s), "upload");
        CK(cudaMemcpyAsync(d + o_ex, excluded, n, cudaMemcpyHostToDevice, s), "upload");
    }
    RescoreArgs a{};
    a.time = reinterpret_cast<const double*>(d + o_time);
    a.excluded = d + o_ex;
    a.rows = reinterpret_cast<const double*>(d + o_rows);
    a.n = (int)n;
    a.R = (int)R;
    a.counts = reinterpret_cast<uint32_t*>(d + o_counts);
    const bool timing = ctx->profile || ctx->kernel_timing;
    if (timing) CK(cudaEventRecord(ctx->ev[0], s), "event");
    CK(launch_count_rows(a, s), "count_rows");
    if (timing) CK(cudaEventRecord(ctx->ev[1], s), "event");
    ctx->counters.launches += 1;
    ctx->counters.rescore_launches += 1;
    CK(cudaMemcpyAsync(counts, d + o_counts, (size_t)R * 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
       "download");
    CK(cudaStreamSynchronize(s), "count_rows");
    if (timing) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]), "event");
        ctx->counters.rescore_ms += ms;
    }
    return FBLS_OK;
}

}  // extern "C"

extern "C" {

// Coarse maps of many uploaded families (the proposal path's first step for a
// batch of stars): on the batch worker contexts, or with workers == 0 planned
// in parallel and run together as job launches on ctx (coarse_maps).
int fbls_coarse_map_batch(fbls_ctx* ctx, fbls_map_job* jobs, uint32_t count, uint32_t workers) {
    if (!ctx || (count && !jobs)) return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    if (count == 0) return FBLS_OK;
    CK(cudaSetDevice(ctx->device), "set device");
    if (workers == 0) {
        std::vector<std::string> errors(count);
        const int rc = coarse_maps(ctx, jobs, count, errors);
        if (rc) return rc;
        for (uint32_t i = 0; i < count; i++)
            if (jobs[i].status) return fail(ctx, jobs[i].status, "map " + std::to_string(i) + ": " + errors[i]);
        return FBLS_OK;
    }
    workers = std::min({workers, count, 64u});
    while (ctx->workers.size() < workers) {
        int status = FBLS_OK;
        fbls_ctx* w = fbls_create(ctx->device, &status);
        if (!w) return fail(ctx, status ? status : FBLS_ERR_CUDA, "batch worker context");
        ctx->workers.push_back(w);
    }
    std::atomic<uint32_t> next{0};
    std::vector<std::string> errors(count);
    auto work = [&](fbls_ctx* wc) {
        if (cudaSetDevice(wc->device) != cudaSuccess) return;
        for (;;) {
            const uint32_t i = next.fetch_add(1);
            if (i >= count) break;
            fbls_map_job& j = jobs[i];
            j.status = fbls_coarse_map(wc, j.ready, j.periods, j.P, j.durations, j.rho, j.nd, j.oversample,
                                       j.bin_days, j.out);
            if (j.status) errors[i] = wc->error;
        }
    };
    std::vector<std::thread> threads;
    for (uint32_t k = 1; k < workers; k++) threads.emplace_back(work, ctx->workers[k]);
    work(ctx->workers[0]);
    for (std::thread& t : threads) t.join();
    for (uint32_t i = 0; i < count; i++)
        if (jobs[i].status) return fail(ctx, jobs[i].status, "map " + std::to_string(i) + ": " + errors[i]);
    return FBLS_OK;
}


// The proposal network's input for a batch of stars (coarse_maps with
// k_map_features): rows of x (channels x count x T) hold each map's
// standardised log1p channels at [offsets[i], offsets[i] + P_i).
int fbls_coarse_features(fbls_ctx* ctx, fbls_map_job* jobs, uint32_t count, const uint32_t* offsets,
                         uint32_t channels, uint32_t T, float* x) {
    if (!ctx || (count && (!jobs || !offsets || !x))) return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    if (channels < 1 || channels > (uint32_t)MAP_MAX_DURATIONS || T < 1)
        return fail(ctx, FBLS_ERR_ARGUMENT, "1 to 8 channels and T >= 1");
    if (count == 0) return FBLS_OK;
    for (uint32_t i = 0; i < count; i++)
        if (jobs[i].nd != channels || (uint64_t)offsets[i] + jobs[i].P > T)
            return fail(ctx, FBLS_ERR_ARGUMENT, "map " + std::to_string(i) + ": does not fit its feature row");
    CK(cudaSetDevice(ctx->device), "set device");
    const size_t bytes = (size_t)channels * count * T * sizeof(float);
    CK(ensure(ctx->feat, bytes), "workspace");
    CK(cudaMemsetAsync(ctx->feat.ptr, 0, bytes, ctx->stream), "workspace");
    MapFeatures feat;
    feat.x = as<float>(ctx->feat);
    feat.channels = (int)channels;
    feat.B = (int)count;
    feat.T = (int)T;
    feat.offsets = offsets;
    std::vector<std::string> errors(count);
    const int rc = coarse_maps(ctx, jobs, count, errors, &feat);
    if (rc) return rc;
    for (uint32_t i = 0; i < count; i++)
        if (jobs[i].status) return fail(ctx, jobs[i].status, "map " + std::to_string(i) + ": " + errors[i]);
    CK(cudaMemcpyAsync(x, ctx->feat.ptr, bytes, cudaMemcpyDeviceToHost, ctx->stream), "download");
    CK(cudaStreamSynchronize(ctx->stream), "map features");
    return FBLS_OK;
}

}  // extern "C"
