// Host driver of the FBLS search path on one B200 and the library's C ABI.
//
// Restates the reference's host logic around the kernels:
//   scan_bank      src/search/scan.rs:144-357 (bank factors, fold budget,
//                  batching, launch sequence, row decode, statistics)
//   scan_periods   src/search/scan.rs:363-408 (coarse prescan, survivors,
//                  full scan, threshold)
//   signal_search  src/search/scan.rs:413-473 (octave bands)
// The device work differs from the reference's: fold and prefix run as one
// kernel with the histograms in shared memory, all batches of a band are
// queued on one stream, and the band's records come back in one copy.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
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
    DevBuf bank, scales, periods, cum, cum32, hist, parts, keys, tflags, records, score, depth, rflags;
    DevBuf evidence, chunks, fault;
    DevBuf family;  // observations of the star a batch worker is searching
    std::vector<int> host_chunks;
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
int upload_family(fbls_ctx* ctx, DevBuf* buf, const double* time, const double* v, const double* w, uint32_t n,
                  double baseline_norm, double origin, double residual_energy, fbls_ready* r) {
    if (!time || !v || !w) return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    if (n < 6) return fail(ctx, FBLS_ERR_DATA, "at least six observations are required");
    for (uint32_t i = 1; i < n; i++)
        if (!(time[i] >= time[i - 1])) return fail(ctx, FBLS_ERR_ARGUMENT, "times must be ascending");
    if (!(time[0] >= 0.0)) return fail(ctx, FBLS_ERR_ARGUMENT, "times must be relative to the first observation");
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

struct BandOut {
    std::vector<double> records;  // P x 9
    std::vector<double> score;
    std::vector<double> depth;
    std::vector<uint32_t> flags;
};

// Fold shape for a launch of up to `periods` periods at nb bins, and the
// family's fold chunks for scales up to scale_max, uploaded to the device.
int plan_fold(fbls_ctx* ctx, const fbls_ready* r, double scale_max, int nb, int periods, FoldShape* shape,
              int* nchunks) {
    *shape = fold_group_shape(nb, periods, ctx->sm_count);
    std::vector<int>& h = ctx->host_chunks;
    h.resize((size_t)r->n + 2);
    const int count = fold_chunks(r->time_host.data(), (int)r->n, scale_max, nb, shape->span_cap, shape->chunk_cap,
                                  h.data(), (int)h.size());
    if (count < 1) return fail(ctx, FBLS_ERR_ARGUMENT, "fold chunking failed");
    CK(ensure(ctx->chunks, ((size_t)count + 1) * sizeof(int)), "workspace");
    CK(cudaMemcpyAsync(ctx->chunks.ptr, h.data(), ((size_t)count + 1) * sizeof(int), cudaMemcpyHostToDevice,
                       ctx->stream),
       "upload chunks");
    *nchunks = count;
    return FBLS_OK;
}

// One scan_bank pass (scan.rs:144-357) of `periods` at nb bins.
int scan_bank(fbls_ctx* ctx, const fbls_ready* r, const double* periods, uint32_t P, const fbls_bank* bank, uint32_t nb,
              bool mixed, BandOut& out, fbls_scan_stats* stats) {
    const uint32_t nd = bank->nd, ns = bank->ns, layers = bank->layers;
    if (stats) stats->phase_bins = nb;
    if (nd == 0 || nd > (uint32_t)MAX_DURATIONS || ns == 0 || ns > (uint32_t)MAX_SHAPES || layers == 0 ||
        layers > (uint32_t)MAX_LAYERS)
        return fail(ctx, FBLS_ERR_ARGUMENT, "bank size outside the supported range");
    if (nb < 2) return fail(ctx, FBLS_ERR_ARGUMENT, "nb must be at least 2");
    // Shape factors 1 - 2 ing l / (L - 1) (scan.rs:157-171).
    std::vector<double> host_bank;
    host_bank.insert(host_bank.end(), bank->durations, bank->durations + nd);
    host_bank.insert(host_bank.end(), bank->rho, bank->rho + nd);
    host_bank.insert(host_bank.end(), bank->ingress, bank->ingress + ns);
    for (uint32_t s = 0; s < ns; s++)
        for (uint32_t l = 0; l < layers; l++)
            host_bank.push_back(1.0 - 2.0 * bank->ingress[s] * (layers > 1 ? (double)l / (double)(layers - 1) : 0.0));
    const uint32_t tiles = (nb + TILE - 1) / TILE;
    const double per_period_bytes = (double)(NF * (4 * (size_t)nb + 2) * 8 + NF * (2 * (size_t)nb + 1) * 8);
    const uint64_t budget = (uint64_t)std::floor((bank->max_fold_mib * 1048576.0) / per_period_bytes);
    if (budget == 0) return fail(ctx, FBLS_ERR_BUDGET, "one folded period exceeds max_fold_mib");
    uint64_t batch = bank->period_batch;
    if (budget < batch) batch = budget;
    if (P < batch) batch = P;
    if (batch == 0) batch = 1;
    // The phase cell floor(t * scale) must fit u32 (kernels.rs:315), with room
    // for the fold's cell arithmetic (cell + 2 nb).
    double scale_max = 0.0;
    std::vector<double> scales(P);
    for (uint32_t i = 0; i < P; i++) {
        scales[i] = (double)nb / periods[i];
        if (!(scales[i] > 0.0) || !std::isfinite(scales[i]))
            return fail(ctx, FBLS_ERR_ARGUMENT, "periods must be positive and finite");
        if (scales[i] > scale_max) scale_max = scales[i];
    }
    if (std::floor(r->t_last * scale_max) >= 4294967295.0 - 2.0 * (double)nb - 2.0)
        return fail(ctx, FBLS_ERR_ARGUMENT, "phase cell exceeds 32 bits");

    const size_t stride = 2 * (size_t)nb + 1;
    // Periods per launch: whole batches of the reference's size, as many as
    // the fold budget holds in this path's buffers (cum, cum32 and tile parts;
    // the histograms never reach device memory), up to 16,384, so bands with
    // few bins fill the GPU with larger period groups. Statistics still count
    // the reference's batches.
    const double launch_period_bytes =
        (double)(NF * stride * (sizeof(double) + sizeof(float2)) +
                 tiles * (PART_STRIDE * sizeof(double) + sizeof(uint64_t) + sizeof(uint32_t)));
    uint64_t launch = (uint64_t)std::floor(bank->max_fold_mib * 1048576.0 / launch_period_bytes);
    launch = std::min<uint64_t>(launch, 16384);
    launch = std::max<uint64_t>(launch / batch, 1) * batch;
    if (launch > P) launch = P;
    CK(ensure(ctx->bank, host_bank.size() * sizeof(double)), "workspace");
    CK(ensure(ctx->scales, (size_t)P * sizeof(double)), "workspace");
    CK(ensure(ctx->periods, (size_t)P * sizeof(double)), "workspace");
    CK(ensure(ctx->cum, launch * NF * stride * sizeof(double)), "workspace");
    CK(ensure(ctx->cum32, launch * NF * stride * sizeof(float2)), "workspace");
    CK(ensure(ctx->parts, launch * tiles * PART_STRIDE * sizeof(double)), "workspace");
    CK(ensure(ctx->keys, launch * tiles * sizeof(uint64_t)), "workspace");
    CK(ensure(ctx->tflags, launch * tiles * sizeof(uint32_t)), "workspace");
    CK(ensure(ctx->records, (size_t)P * RECORD_STRIDE * sizeof(double)), "workspace");
    CK(ensure(ctx->score, (size_t)P * sizeof(double)), "workspace");
    CK(ensure(ctx->depth, (size_t)P * sizeof(double)), "workspace");
    CK(ensure(ctx->rflags, (size_t)P * sizeof(uint32_t)), "workspace");
    CK(ensure(ctx->fault, sizeof(uint32_t)), "workspace");
    FoldShape shape;
    int nchunks = 0;
    {
        int rc = plan_fold(ctx, r, scale_max, (int)nb, (int)launch, &shape, &nchunks);
        if (rc) return rc;
    }
    if (!shape.hist_in_smem) {
        const size_t blocks = (launch + shape.group - 1) / shape.group;
        CK(ensure(ctx->hist, blocks * shape.group * NF * (size_t)shape.row_stride * sizeof(double)), "workspace");
    }

    cudaStream_t s = ctx->stream;
    CK(cudaMemsetAsync(ctx->fault.ptr, 0, sizeof(uint32_t), s), "workspace");
    CK(cudaMemcpyAsync(ctx->bank.ptr, host_bank.data(), host_bank.size() * sizeof(double), cudaMemcpyHostToDevice, s),
       "upload bank");
    CK(cudaMemcpyAsync(ctx->scales.ptr, scales.data(), (size_t)P * sizeof(double), cudaMemcpyHostToDevice, s),
       "upload scales");
    CK(cudaMemcpyAsync(ctx->periods.ptr, periods, (size_t)P * sizeof(double), cudaMemcpyHostToDevice, s),
       "upload periods");
    const double* d_bank = as<double>(ctx->bank);

    const bool timing = ctx->profile || ctx->kernel_timing;
    const uint64_t nbatches = (P + launch - 1) / launch;
    if (timing) {
        while (ctx->pool.size() < 3 * nbatches) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e), "event");
            ctx->pool.push_back(e);
        }
    }
    uint64_t bi = 0;
    for (uint64_t cursor = 0; cursor < P; cursor += launch, bi++) {
        const int p = (int)((P - cursor) < launch ? (P - cursor) : launch);
        FoldArgs fa;
        fa.time = r->time;
        fa.v = r->v;
        fa.w = r->w;
        fa.scales = as<double>(ctx->scales) + cursor;
        fa.n = (int)r->n;
        fa.nb = (int)nb;
        fa.periods = p;
        fa.group = 1;
        fa.cum = as<double>(ctx->cum);
        fa.cum32 = as<float2>(ctx->cum32);
        if (timing) CK(cudaEventRecord(ctx->pool[3 * bi], s), "event");
        fa.group = shape.group;
        fa.hist_global = shape.hist_in_smem ? nullptr : as<double>(ctx->hist);
        fa.hist_out = nullptr;
        fa.chunks = as<int>(ctx->chunks);
        fa.nchunks = nchunks;
        fa.stage_field = shape.stage_field;
        fa.window = shape.window;
        fa.row_stride = shape.row_stride;
        fa.fault = as<uint32_t>(ctx->fault);
        CK(launch_fold(fa, shape, s), "fold");
        ctx->counters.launches += 1;
        ctx->counters.fold_launches += 1;
        ctx->counters.fold_bytes += (double)p * (24.0 * r->n + 48.0 * (double)stride);
        ctx->counters.fold_updates += (uint64_t)p * r->n;
        if (timing) CK(cudaEventRecord(ctx->pool[3 * bi + 1], s), "event");
        ScanArgs sa;
        sa.cum = as<double>(ctx->cum);
        sa.cum32 = as<float2>(ctx->cum32);
        sa.scales = fa.scales;
        sa.durations = d_bank;
        sa.rho = d_bank + nd;
        sa.ingress = d_bank + 2 * nd;
        sa.factors = d_bank + 2 * nd + ns;
        sa.baseline = r->baseline_norm;
        sa.gate = bank->shape_gate;
        sa.n = (double)r->n;
        sa.nb = (int)nb;
        sa.nd = (int)nd;
        sa.ns = (int)ns;
        sa.layers = (int)layers;
        sa.mixed = mixed ? 1 : 0;
        sa.parts = as<double>(ctx->parts);
        sa.keys = as<uint64_t>(ctx->keys);
        sa.flags = as<uint32_t>(ctx->tflags);
        CK(launch_scan_tiles(sa, p, s), "scan_tiles");
        MergeArgs ma;
        ma.parts = sa.parts;
        ma.keys = sa.keys;
        ma.flags = sa.flags;
        ma.periods_in = as<double>(ctx->periods) + cursor;
        ma.scales = fa.scales;
        ma.periods = p;
        ma.tiles = (int)tiles;
        ma.offset = (int)cursor;
        ma.records = as<double>(ctx->records);
        ma.score = as<double>(ctx->score);
        ma.depth = as<double>(ctx->depth);
        ma.flags_out = as<uint32_t>(ctx->rflags);
        CK(launch_merge(ma, s), "merge");
        if (timing) CK(cudaEventRecord(ctx->pool[3 * bi + 2], s), "event");
        ctx->counters.launches += 2;
        ctx->counters.scan_launches += 1;
        ctx->counters.scan_bytes += (double)p * (24.0 * (double)stride + 84.0 * tiles);
        if (stats) {
            stats->templates_scanned += (uint64_t)p * nd * ns * nb;
            stats->batches += ((uint64_t)p + batch - 1) / batch;
        }
    }
    out.records.resize((size_t)P * RECORD_STRIDE);
    out.score.resize(P);
    out.depth.resize(P);
    out.flags.resize(P);
    CK(cudaMemcpyAsync(out.records.data(), ctx->records.ptr, out.records.size() * sizeof(double),
                       cudaMemcpyDeviceToHost, s),
       "download records");
    CK(cudaMemcpyAsync(out.score.data(), ctx->score.ptr, P * sizeof(double), cudaMemcpyDeviceToHost, s), "download");
    CK(cudaMemcpyAsync(out.depth.data(), ctx->depth.ptr, P * sizeof(double), cudaMemcpyDeviceToHost, s), "download");
    CK(cudaMemcpyAsync(out.flags.data(), ctx->rflags.ptr, P * sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
       "download");
    uint32_t fault = 0;
    CK(cudaMemcpyAsync(&fault, ctx->fault.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "download");
    CK(cudaStreamSynchronize(s), "scan_bank");
    if (fault) return fail(ctx, FBLS_ERR_CUDA, "fold: staging copies did not complete");
    double t_fold = 0.0, t_scan = 0.0;
    if (timing) {
        for (uint64_t b = 0; b < nbatches; b++) {
            float a = 0.f, c = 0.f;
            CK(cudaEventElapsedTime(&a, ctx->pool[3 * b], ctx->pool[3 * b + 1]), "event");
            CK(cudaEventElapsedTime(&c, ctx->pool[3 * b + 1], ctx->pool[3 * b + 2]), "event");
            t_fold += a;
            t_scan += c;
        }
        ctx->counters.fold_ms += t_fold;
        ctx->counters.scan_ms += t_scan;
    }
    uint64_t rescans = 0, retries = 0;
    bool bad = false;
    for (uint32_t i = 0; i < P; i++) {
        bad = bad || (out.flags[i] & 2u);
        retries += (out.flags[i] & 1u) ? 1 : 0;
        rescans += (out.flags[i] & 4u) ? 1 : 0;
    }
    if (stats) {
        stats->exact_tile_retries += retries;
        stats->tile_rescans += rescans;
        stats->seconds_fold += t_fold * 1e-3;
        stats->seconds_scan += t_scan * 1e-3;
    }
    if (bad) return fail(ctx, FBLS_ERR_PRECISION, "nonpositive template precision; inspect noise model");
    return FBLS_OK;
}

double now_seconds() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

// scan_periods (scan.rs:363-408). Rows are appended to `rows`.
int scan_periods(fbls_ctx* ctx, const fbls_ready* r, const double* periods, uint32_t P, const fbls_bank* bank,
                 bool mixed, std::vector<fbls_row>& rows, fbls_scan_stats* stats) {
    const double start = now_seconds();
    fbls_scan_stats st;
    std::memset(&st, 0, sizeof(st));
    st.periods = P;
    if (P == 0 || bank->nd == 0) {
        if (stats) *stats = st;
        return FBLS_OK;
    }
    double dmin = __builtin_huge_val();
    for (uint32_t i = 0; i < bank->nd; i++) dmin = rmin(dmin, bank->durations[i]);
    uint64_t nb = as_u64(std::ceil((double)bank->phase_oversample * periods[P - 1] / dmin));
    if (nb < 8) nb = 8;
    if (nb > (1u << 24)) return fail(ctx, FBLS_ERR_ARGUMENT, "phase grid too large");
    std::vector<double> survivors(periods, periods + P);
    BandOut band;
    if (bank->prescan_factor > 1 && nb / bank->prescan_factor >= 8) {
        int rc = scan_bank(ctx, r, periods, P, bank, (uint32_t)(nb / bank->prescan_factor), mixed, band, &st);
        if (rc) return rc;
        survivors.clear();
        const double cut = bank->prescan_fraction * bank->threshold;
        for (uint32_t i = 0; i < P; i++) {
            double sc = band.score[i];
            if (std::isfinite(sc) && sc >= cut) survivors.push_back(band.records[(size_t)i * RECORD_STRIDE]);
        }
        st.prescan_survivors = survivors.size();
    }
    if (!survivors.empty()) {
        int rc = scan_bank(ctx, r, survivors.data(), (uint32_t)survivors.size(), bank, (uint32_t)nb, mixed, band, &st);
        if (rc) return rc;
        for (size_t i = 0; i < survivors.size(); i++) {
            double sc = band.score[i];
            if (!(std::isfinite(sc) && sc >= bank->threshold)) continue;
            const double* rec = &band.records[i * RECORD_STRIDE];
            fbls_row row;
            row.period = rec[0];
            row.epoch = (rec[2] + rec[3] / 2.0) / rec[1] + r->origin;
            row.duration = rec[3] / rec[1];
            row.score = sc;
            row.depth = band.depth[i];
            rows.push_back(row);
        }
    }
    st.seconds = now_seconds() - start;
    if (stats) *stats = st;
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
    DevBuf* bufs[] = {&ctx->bank,  &ctx->scales,  &ctx->periods, &ctx->cum,   &ctx->cum32,  &ctx->hist,    &ctx->parts,
                      &ctx->keys,  &ctx->tflags,  &ctx->records, &ctx->score, &ctx->depth,  &ctx->rflags,  &ctx->evidence,
                      &ctx->chunks, &ctx->fault,  &ctx->family};
    for (DevBuf* b : bufs) release(*b);
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
    if (records) std::memcpy(records, band.records.data(), band.records.size() * sizeof(double));
    if (score) std::memcpy(score, band.score.data(), band.score.size() * sizeof(double));
    if (depth) std::memcpy(depth, band.depth.data(), band.depth.size() * sizeof(double));
    if (flags) std::memcpy(flags, band.flags.data(), band.flags.size() * sizeof(uint32_t));
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
    if (!ctx || !ready || !durations || !rho || !cfg || !n_rows) return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    if (nd == 0) return fail(ctx, FBLS_ERR_ARGUMENT, "no durations");
    CK(cudaSetDevice(ctx->device), "set device");
    // Durations sorted with rho carried along (scan.rs:418-424).
    std::vector<std::pair<double, double>> ds(nd);
    for (uint32_t i = 0; i < nd; i++) ds[i] = {durations[i], rho[i]};
    std::stable_sort(ds.begin(), ds.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    const double baseline = ready->t_last;
    const double maximum = rmin(cfg->period_max, baseline);
    const double minimum = rmax(cfg->period_min, 4.0 * ds[0].first * (1.0 + 1e-9));
    *n_rows = 0;
    if (grid_len) *grid_len = 0;
    if (n_bands) *n_bands = 0;
    if (maximum <= minimum) return FBLS_OK;
    const int64_t count = period_grid(minimum, maximum, baseline, ds[0].first, cfg->period_oversample, nullptr, 0);
    std::vector<double> grid((size_t)count);
    period_grid(minimum, maximum, baseline, ds[0].first, cfg->period_oversample, grid.data(), count);
    if (grid_len) *grid_len = (uint64_t)count;
    const double shape_gate = cfg->n_ingress > 0 && cfg->ingress_fractions[0] == 0.0
                                  ? cfg->shape_gate_fraction * cfg->threshold
                                  : 0.0;
    std::vector<fbls_row> rows;
    uint32_t bands = 0;
    double lo = grid[0];
    const double last = grid[grid.size() - 1];
    while (lo <= last) {
        const double hi = lo * 2.0;
        std::vector<double> selected;
        for (double p : grid)
            if (p >= lo && p < hi) selected.push_back(p);
        std::vector<double> bd, br;
        for (auto& d : ds)
            if (d.first < lo / 4.0) {
                bd.push_back(d.first);
                br.push_back(d.second);
            }
        if (!selected.empty() && !bd.empty()) {
            fbls_bank bank;
            bank.durations = bd.data();
            bank.rho = br.data();
            bank.nd = (uint32_t)bd.size();
            bank.ingress = cfg->ingress_fractions;
            bank.ns = cfg->n_ingress;
            bank.layers = cfg->shape_layers;
            bank.threshold = cfg->threshold;
            bank.shape_gate = shape_gate;
            bank.phase_oversample = cfg->phase_oversample;
            bank.period_batch = cfg->period_batch;
            bank.max_fold_mib = fold_budget_mib(cfg->max_fold_mib);
            bank.prescan_factor = cfg->prescan_factor;
            bank.prescan_fraction = cfg->prescan_fraction;
            fbls_scan_stats st;
            int rc = scan_periods(ctx, ready, selected.data(), (uint32_t)selected.size(), &bank,
                                  cfg->precision_mode == 0, rows, &st);
            if (rc) return rc;
            if (stats_out && bands < 64) stats_out[bands] = st;
            bands++;
        }
        lo = hi;
    }
    if (rows.size() > capacity) return fail(ctx, FBLS_ERR_ARGUMENT, "row capacity too small");
    std::memcpy(rows_out, rows.data(), rows.size() * sizeof(fbls_row));
    *n_rows = (uint32_t)rows.size();
    if (n_bands) *n_bands = bands;
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

// Many stars on one device: `workers` host threads (the caller's included),
// each with its own context (stream, workspace and a reusable buffer for the
// star's observations), take stars from a shared counter and run
// signal_search on them, so one star's host work and small launches overlap
// the others' kernels. The reference runs one star per device worker thread
// (src/batch.rs:61-102) with one context per thread.
int fbls_search_batch(fbls_ctx* ctx, fbls_star* stars, uint32_t count, const fbls_config* cfg, uint32_t workers) {
    if (!ctx || (count && !stars) || !cfg) return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    if (count == 0) return FBLS_OK;
    workers = std::max(1u, std::min({workers, count, 64u}));
    CK(cudaSetDevice(ctx->device), "set device");
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
                rc = fbls_signal_search(wc, r, s.durations, s.rho, s.nd, &c, s.rows, s.capacity, &s.n_rows,
                                        &s.grid_len, st, &bands);
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
