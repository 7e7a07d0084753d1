// Host side of the proposal path's coarse maps (the learned pruning of the
// search; no counterpart in the reference): per-star plans made on host
// threads, job launches of the folds (with the box-map epilogue) and the
// features, and the C ABI entry points fbls_coarse_map, fbls_coarse_map_batch
// and fbls_coarse_features.
#include "common.cuh"
#include "host_internal.h"
#include "kernels.h"

using namespace fbls;

namespace {
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
        g.shape = fold_map_shape((int)nb, (int)std::min(g.count, g.per_launch), ctx->sm_count);
        const int c = fold_chunk_list(ready->time_host.data(), (int)ready->n, scale_max, (int)nb, g.shape.span_cap,
                                      g.shape.chunk_cap, g.chunks);
        if (c < 1) return bad(FBLS_ERR_ARGUMENT, "fold chunking failed");
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
        int fold_jobs = 0, fold_ctas = 0, map_jobs = 0, map_total = 0, fold_threads = 0;
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
                // one CTA size per wave's job launch
                if (!waves.back().units.empty() &&
                    ((waves.back().cum + cum) * (sizeof(double) + sizeof(float2)) > MAP_WAVE_BYTES ||
                     (walk && waves.back().fold_threads && waves.back().fold_threads != g.shape.threads)))
                    waves.emplace_back();
                Wave& w = waves.back();
                w.units.push_back({m, &g, c0, n, w.cum, w.hist, walk});
                w.cum += cum;
                w.hist += hist;
                if (walk) {
                    w.fold_jobs++;
                    w.fold_threads = g.shape.threads;
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
            fa.lockstep_min = g.shape.lockstep_min;
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
                                reinterpret_cast<const int*>(din + w.off_fcta), w.fold_jobs, w.fold_ctas,
                                w.fold_threads, false, w.smem, s),
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

extern "C" {

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
    // x is host or device memory (unified addressing tells the copy which).
    CK(cudaMemcpyAsync(x, ctx->feat.ptr, bytes, cudaMemcpyDefault, ctx->stream), "copy features");
    CK(cudaStreamSynchronize(ctx->stream), "map features");
    return FBLS_OK;
}

}  // extern "C"
