// C ABI of the steps either side of the search: the single-event scan
// (src/search/events.rs), the biweight detrend and the raw-mode preparation
// (src/prep/curve.rs), and the peak-selection rescoring (src/select/peaks.rs
// with kernels.rs:936-1042).
#include <tuple>

#include "common.cuh"
#include "host_internal.h"
#include "kernels.h"
#include "prep.h"

using namespace fbls;

extern "C" {

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
