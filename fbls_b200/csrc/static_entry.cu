// fbls_scan_bank_static: the scan_bank pass (fold, prefix sums, tile scan,
// merge) without any device allocation.
//
// Some callers cannot call cudaMalloc: their device memory belongs to someone
// else (a framework's caching allocator that must own every allocation, or a
// fixed per-process memory partition), so they cannot create a context with
// its own workspace. This entry point keeps all of its device storage in one
// file-scope __device__ array of FBLS_STATIC_SCRATCH_BYTES, which every GPU
// that loads the library holds until the process exits. The caller passes
// host inputs and host outputs; the data is copied into the array, folded
// and scanned in batches of periods that fit it, and the results are copied
// back.
//
// Set-up: every call, with its device current, resolves the array's device
// address (cudaGetSymbolAddress) and checks the result. The address is not
// kept between calls: after cudaDeviceReset the module is loaded again and
// the array may sit elsewhere. The first call on a device also loads the
// library's module there, so make that call before any stream capture. In
// host code the array's name is only a host-side stand-in, never a device
// address.
//
// Every call shares the one array and overwrites it: calls that overlap on
// the GPU (from several host threads, or on several streams) race. Nothing in
// the array needs to start at zero: every region a kernel uses is written
// earlier in the same call (the fold zeroes its own histograms; its bulk
// copies also read the one padding slot past each field, which it ignores).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fbls_b200.h"
#include "common.cuh"
#include "kernels.h"

namespace fbls {

static __device__ __align__(256) unsigned char g_fbls_scratch[FBLS_STATIC_SCRATCH_BYTES];

namespace {

constexpr int MAX_DEVICES = 64;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

int report(char* error, uint32_t error_len, int status, const std::string& message) {
    if (error && error_len) {
        std::strncpy(error, message.c_str(), error_len - 1);
        error[error_len - 1] = '\0';
    }
    return status;
}

}  // namespace

}  // namespace fbls

using namespace fbls;

extern "C" int fbls_scan_bank_static(int device, const double* time, const double* v, const double* w, uint32_t n,
                                     double baseline_norm, const double* periods, uint32_t P, const fbls_bank* bank,
                                     uint32_t nb, uint32_t precision_mode, double* records, double* score,
                                     double* depth, uint32_t* flags, char* error, uint32_t error_len) {
    if (!time || !v || !w || !bank || (P && (!periods || !records || !score || !depth || !flags)))
        return report(error, error_len, FBLS_ERR_ARGUMENT, "null argument");
    if (device < 0 || device >= MAX_DEVICES) return report(error, error_len, FBLS_ERR_ARGUMENT, "bad device");
    if (precision_mode > 2) return report(error, error_len, FBLS_ERR_ARGUMENT, "precision_mode must be 0, 1 or 2");
    if (P == 0) return FBLS_OK;
    if (n < 6) return report(error, error_len, FBLS_ERR_DATA, "at least six observations are required");
    const uint32_t nd = bank->nd, ns = bank->ns, layers = bank->layers;
    if (nd == 0 || nd > (uint32_t)MAX_DURATIONS || ns == 0 || ns > (uint32_t)MAX_SHAPES || layers == 0 ||
        layers > (uint32_t)MAX_LAYERS || nb < 8)
        return report(error, error_len, FBLS_ERR_ARGUMENT, "bank size outside the supported range");
    if (!bank->durations || !bank->rho || !bank->ingress)
        return report(error, error_len, FBLS_ERR_ARGUMENT, "null argument");
    for (uint32_t i = 0; i < nd; i++)
        if (!(bank->durations[i] > 0.0) || !std::isfinite(bank->durations[i]) || !std::isfinite(bank->rho[i]))
            return report(error, error_len, FBLS_ERR_ARGUMENT, "durations must be positive and finite");
    for (uint32_t i = 1; i < n; i++)
        if (!(time[i] >= time[i - 1])) return report(error, error_len, FBLS_ERR_ARGUMENT, "times must be ascending");
    if (!(time[0] >= 0.0))
        return report(error, error_len, FBLS_ERR_ARGUMENT, "times must be relative to the first observation");
    std::vector<double> scales(P);
    double scale_max = 0.0;
    for (uint32_t i = 0; i < P; i++) {
        scales[i] = (double)nb / periods[i];
        if (!(scales[i] > 0.0) || !std::isfinite(scales[i]))
            return report(error, error_len, FBLS_ERR_ARGUMENT, "periods must be positive and finite");
        scale_max = std::max(scale_max, scales[i]);
    }
    if (std::floor(time[n - 1] * scale_max) >= 4294967295.0 - 2.0 * (double)nb - 2.0)
        return report(error, error_len, FBLS_ERR_ARGUMENT, "phase cell exceeds 32 bits");

    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return report(error, error_len, FBLS_ERR_CUDA, cudaGetErrorString(e));
    void* symbol = nullptr;
    e = cudaGetSymbolAddress(&symbol, g_fbls_scratch);
    if (e != cudaSuccess)
        return report(error, error_len, FBLS_ERR_CUDA, std::string("static scratch address: ") + cudaGetErrorString(e));
    unsigned char* const base = static_cast<unsigned char*>(symbol);
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return report(error, error_len, FBLS_ERR_CUDA, cudaGetErrorString(e));

    // Fixed part of the array: fields, bank constants, fold chunks.
    std::vector<double> host_bank;
    host_bank.insert(host_bank.end(), bank->durations, bank->durations + nd);
    host_bank.insert(host_bank.end(), bank->rho, bank->rho + nd);
    host_bank.insert(host_bank.end(), bank->ingress, bank->ingress + ns);
    for (uint32_t s = 0; s < ns; s++)
        for (uint32_t l = 0; l < layers; l++)
            host_bank.push_back(1.0 - 2.0 * bank->ingress[s] * (layers > 1 ? (double)l / (double)(layers - 1) : 0.0));
    const size_t fstride = fold_field_stride(n);
    const size_t fields_bytes = align256(3 * sizeof(double) * fstride) + align256(sizeof(uint32_t));
    const size_t bank_bytes = align256(sizeof(double) * host_bank.size());
    const size_t chunk_bytes = align256(sizeof(int) * ((size_t)n + 2));
    const size_t fixed = fields_bytes + bank_bytes + chunk_bytes;
    const uint32_t tiles = (nb + TILE - 1) / TILE;
    const size_t stride = 2 * (size_t)nb + 1;
    // Per period of a batch: scales, periods, cum, cum32, parts, keys, tile
    // flags, records, score, depth, flags, plus 3 row_stride doubles of fold
    // scratch when the histogram does not fit shared memory (the fold's CTAs
    // take `group` periods each, so the scratch covers group x ceil(batch /
    // group) periods: group - 1 more are budgeted); 256 bytes of alignment
    // slack per region. The batch is the largest that fits with the fold
    // shape it is launched with.
    const size_t slack = 12 * 256;
    auto per_period_of = [&](const FoldShape& sh) {
        return 2 * sizeof(double) + NF * stride * (sizeof(double) + sizeof(float2)) +
               tiles * (PART_STRIDE * sizeof(double) + sizeof(uint64_t) + sizeof(uint32_t)) +
               RECORD_STRIDE * sizeof(double) + 2 * sizeof(double) + sizeof(uint32_t) +
               (sh.hist_in_smem ? 0 : (size_t)NF * sh.row_stride * sizeof(double));
    };
    auto hist_extra_of = [&](const FoldShape& sh) {
        return sh.hist_in_smem ? (size_t)0 : (size_t)(sh.group - 1) * NF * sh.row_stride * sizeof(double);
    };
    size_t batch = P;
    FoldShape shape{};
    for (;;) {
        shape = fold_group_shape((int)nb, (int)batch, sms);
        const size_t need = fixed + slack + hist_extra_of(shape);
        const size_t per_period = per_period_of(shape);
        const size_t fit = need + per_period > FBLS_STATIC_SCRATCH_BYTES
                               ? 0
                               : (FBLS_STATIC_SCRATCH_BYTES - need) / per_period;
        if (fit == 0)
            return report(error, error_len, FBLS_ERR_ARGUMENT,
                          "input exceeds the static scratch of fbls_scan_bank_static (" +
                              std::to_string((unsigned long long)FBLS_STATIC_SCRATCH_BYTES) + " bytes)");
        if (batch <= fit) break;
        batch = fit;  // strictly smaller: the loop ends
    }
    const size_t hist_periods = ((batch + shape.group - 1) / shape.group) * (size_t)shape.group;
    std::vector<int> chunks((size_t)n + 2);
    const int nchunks = fold_chunks(time, (int)n, scale_max, (int)nb, shape.span_cap, shape.chunk_cap, chunks.data(),
                                    (int)chunks.size());
    if (nchunks < 1) return report(error, error_len, FBLS_ERR_ARGUMENT, "fold chunking failed");

    unsigned char* at = base;
    auto take = [&](size_t bytes) {
        unsigned char* p = at;
        at += align256(bytes);
        return p;
    };
    double* d_time = reinterpret_cast<double*>(take(3 * sizeof(double) * fstride));
    double* d_v = d_time + fstride;
    double* d_w = d_v + fstride;
    uint32_t* d_fault = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t)));
    double* d_bank = reinterpret_cast<double*>(take(sizeof(double) * host_bank.size()));
    int* d_chunks = reinterpret_cast<int*>(take(sizeof(int) * ((size_t)nchunks + 1)));
    double* d_scales = reinterpret_cast<double*>(take(sizeof(double) * batch));
    double* d_periods = reinterpret_cast<double*>(take(sizeof(double) * batch));
    double* d_cum = reinterpret_cast<double*>(take(NF * stride * sizeof(double) * batch));
    float2* d_cum32 = reinterpret_cast<float2*>(take(NF * stride * sizeof(float2) * batch));
    double* d_parts = reinterpret_cast<double*>(take(tiles * PART_STRIDE * sizeof(double) * batch));
    uint64_t* d_keys = reinterpret_cast<uint64_t*>(take(tiles * sizeof(uint64_t) * batch));
    uint32_t* d_tflags = reinterpret_cast<uint32_t*>(take(tiles * sizeof(uint32_t) * batch));
    double* d_records = reinterpret_cast<double*>(take(RECORD_STRIDE * sizeof(double) * batch));
    double* d_score = reinterpret_cast<double*>(take(sizeof(double) * batch));
    double* d_depth = reinterpret_cast<double*>(take(sizeof(double) * batch));
    uint32_t* d_rflags = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * batch));
    double* d_hist = shape.hist_in_smem ? nullptr
                                        : reinterpret_cast<double*>(
                                              take((size_t)NF * shape.row_stride * sizeof(double) * hist_periods));
    if ((size_t)(at - base) > FBLS_STATIC_SCRATCH_BYTES)
        return report(error, error_len, FBLS_ERR_ARGUMENT, "input exceeds the static scratch");

    const cudaStream_t s = 0;
    auto ok = [&](cudaError_t err, const char* where) {
        if (err != cudaSuccess) report(error, error_len, FBLS_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(err));
        return err == cudaSuccess;
    };
    if (!ok(cudaMemsetAsync(d_fault, 0, sizeof(uint32_t), s), "clear fault") ||
        !ok(cudaMemcpyAsync(d_time, time, sizeof(double) * n, cudaMemcpyHostToDevice, s), "upload time") ||
        !ok(cudaMemcpyAsync(d_v, v, sizeof(double) * n, cudaMemcpyHostToDevice, s), "upload v") ||
        !ok(cudaMemcpyAsync(d_w, w, sizeof(double) * n, cudaMemcpyHostToDevice, s), "upload w") ||
        !ok(cudaMemcpyAsync(d_bank, host_bank.data(), sizeof(double) * host_bank.size(), cudaMemcpyHostToDevice, s),
            "upload bank") ||
        !ok(cudaMemcpyAsync(d_chunks, chunks.data(), sizeof(int) * ((size_t)nchunks + 1), cudaMemcpyHostToDevice, s),
            "upload chunks"))
        return FBLS_ERR_CUDA;

    bool bad = false;
    for (size_t cursor = 0; cursor < P; cursor += batch) {
        const int p = (int)std::min(batch, (size_t)P - cursor);
        if (!ok(cudaMemcpyAsync(d_scales, scales.data() + cursor, sizeof(double) * p, cudaMemcpyHostToDevice, s),
                "upload scales") ||
            !ok(cudaMemcpyAsync(d_periods, periods + cursor, sizeof(double) * p, cudaMemcpyHostToDevice, s),
                "upload periods"))
            return FBLS_ERR_CUDA;
        FoldArgs fa{};
        fa.time = d_time;
        fa.v = d_v;
        fa.w = d_w;
        fa.scales = d_scales;
        fa.n = (int)n;
        fa.nb = (int)nb;
        fa.periods = p;
        fa.group = shape.group;
        fa.cum = d_cum;
        fa.cum32 = d_cum32;
        fa.hist_global = d_hist;
        fa.hist_out = nullptr;
        fa.chunks = d_chunks;
        fa.nchunks = nchunks;
        fa.stage_field = shape.stage_field;
        fa.window = shape.window;
        fa.row_stride = shape.row_stride;
        fa.fault = d_fault;
        fa.rows32_only = precision_mode == 2 ? 1 : 0;
        if (!ok(launch_fold(fa, shape, s), "fold")) return FBLS_ERR_CUDA;
        ScanArgs sa{};
        sa.cum = d_cum;
        sa.cum32 = d_cum32;
        sa.scales = d_scales;
        sa.durations = d_bank;
        sa.rho = d_bank + nd;
        sa.ingress = d_bank + 2 * nd;
        sa.factors = d_bank + 2 * nd + ns;
        sa.baseline = baseline_norm;
        sa.gate = bank->shape_gate;
        sa.n = (double)n;
        sa.nb = (int)nb;
        sa.nd = (int)nd;
        sa.ns = (int)ns;
        sa.layers = (int)layers;
        sa.mixed = precision_mode == 0 ? 1 : precision_mode == 1 ? 0 : 2;
        sa.parts = d_parts;
        sa.keys = d_keys;
        sa.flags = d_tflags;
        if (!ok(launch_scan_tiles(sa, p, s), "scan_tiles")) return FBLS_ERR_CUDA;
        MergeArgs ma{};
        ma.parts = d_parts;
        ma.keys = d_keys;
        ma.flags = d_tflags;
        ma.periods_in = d_periods;
        ma.scales = d_scales;
        ma.periods = p;
        ma.tiles = (int)tiles;
        ma.offset = 0;
        ma.records = d_records;
        ma.score = d_score;
        ma.depth = d_depth;
        ma.flags_out = d_rflags;
        if (!ok(launch_merge(ma, s), "merge")) return FBLS_ERR_CUDA;
        if (!ok(cudaMemcpyAsync(records + cursor * RECORD_STRIDE, d_records, RECORD_STRIDE * sizeof(double) * p,
                                cudaMemcpyDeviceToHost, s),
                "download records") ||
            !ok(cudaMemcpyAsync(score + cursor, d_score, sizeof(double) * p, cudaMemcpyDeviceToHost, s),
                "download score") ||
            !ok(cudaMemcpyAsync(depth + cursor, d_depth, sizeof(double) * p, cudaMemcpyDeviceToHost, s),
                "download depth") ||
            !ok(cudaMemcpyAsync(flags + cursor, d_rflags, sizeof(uint32_t) * p, cudaMemcpyDeviceToHost, s),
                "download flags") ||
            !ok(cudaStreamSynchronize(s), "scan"))
            return FBLS_ERR_CUDA;
        for (int i = 0; i < p; i++) bad = bad || (flags[cursor + i] & 2u);
    }
    uint32_t fault = 0;
    if (!ok(cudaMemcpy(&fault, d_fault, sizeof(uint32_t), cudaMemcpyDeviceToHost), "download fault"))
        return FBLS_ERR_CUDA;
    if (fault) return report(error, error_len, FBLS_ERR_CUDA, "fold: staging copies did not complete");
    if (bad) return report(error, error_len, FBLS_ERR_PRECISION, "nonpositive template precision; inspect noise model");
    return FBLS_OK;
}
