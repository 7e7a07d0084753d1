// Bin-index forms of the precision study on sm_100a (and, at the end, the C
// entry points of the launch-shape tuning table): the fold's bin
// floor(t * scale) mod nb (src/search/kernels.rs:314-327, one rounded f64
// product) against two cheaper forms, on the device, for every observation
// of an uploaded family at a sample of scales:
//   * a plain f32 product of the rounded inputs;
//   * a double-single product (t and scale split into f32 (hi, lo) pairs;
//     the hi product and its exact error from an f32 fma, plus the two cross
//     terms), whose floor is taken from the unevaluated sum; and
//   * the double-single form with an exact fallback: where the double-single
//     value lies within a bound of an integer (|value| 2^-36 + 2^-40, well
//     above the form's error of about |value| 2^-46 and the f64 product's
//     |value| 2^-53), the bin comes from the f64 product instead.
// The fold itself keeps the f64 product: it is exact by definition and the
// fold is bound by its shared-memory pipe, not by f64 multiplies.
#include "common.cuh"
#include "host_internal.h"
#include "kernels.h"

namespace fbls {

namespace {

__device__ __forceinline__ uint32_t bin_f64(double t, double scale, uint32_t nb) {
    return (uint32_t)((uint64_t)floor(__dmul_rn(t, scale)) % nb);
}

__global__ void __launch_bounds__(256) k_bin_forms(const double* __restrict__ time, int n,
                                                   const double* __restrict__ scales, int P, uint32_t nb,
                                                   unsigned long long* __restrict__ counts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long pairs = 0, f32_miss = 0, ds_miss = 0, fallbacks = 0, after = 0;
    if (i < n) {
        const double t = time[i];
        const float th = __double2float_rn(t);
        const float tl = __double2float_rn(__dsub_rn(t, (double)th));
        for (int p = 0; p < P; p++) {
            const double s = scales[p];
            const uint32_t ref = bin_f64(t, s, nb);
            const float sh = __double2float_rn(s);
            const float sl = __double2float_rn(__dsub_rn(s, (double)sh));
            // plain f32 product
            const uint32_t b32 = (uint32_t)((uint64_t)floorf(__fmul_rn(th, sh)) % nb);
            // double-single product: hi + lo
            const float hi = __fmul_rn(th, sh);
            const float err = __fmaf_rn(th, sh, -hi);
            const float lo = __fadd_rn(err, __fadd_rn(__fmul_rn(th, sl), __fmul_rn(tl, sh)));
            const float base = floorf(hi);
            const float frac = __fadd_rn(__fsub_rn(hi, base), lo);  // hi - base is exact below 2^23
            const float step = frac < 0.0f ? -1.0f : (frac >= 1.0f ? 1.0f : 0.0f);
            const uint32_t bds = (uint32_t)((uint64_t)(base + step) % nb);
            const float bound = __fadd_rn(__fmul_rn(fabsf(hi), 0x1p-36f), 0x1p-40f);
            const bool near = fabsf(frac) < bound || fabsf(__fsub_rn(frac, 1.0f)) < bound;
            const uint32_t bfb = near ? ref : bds;
            pairs++;
            f32_miss += b32 != ref;
            ds_miss += bds != ref;
            fallbacks += near;
            after += bfb != ref;
        }
    }
    // Warp totals, one atomic per warp and counter.
    for (int off = 16; off > 0; off >>= 1) {
        pairs += __shfl_xor_sync(0xffffffffu, pairs, off);
        f32_miss += __shfl_xor_sync(0xffffffffu, f32_miss, off);
        ds_miss += __shfl_xor_sync(0xffffffffu, ds_miss, off);
        fallbacks += __shfl_xor_sync(0xffffffffu, fallbacks, off);
        after += __shfl_xor_sync(0xffffffffu, after, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(counts + 0, pairs);
        atomicAdd(counts + 1, f32_miss);
        atomicAdd(counts + 2, ds_miss);
        atomicAdd(counts + 3, fallbacks);
        atomicAdd(counts + 4, after);
    }
}

}  // namespace

}  // namespace fbls

using namespace fbls;

extern "C" int fbls_precision_bins(fbls_ctx* ctx, const fbls_ready* ready, const double* scales, uint32_t P,
                                   uint32_t nb, uint64_t* counts) {
    if (!ctx || !ready || !counts || (P && !scales)) return fail(ctx, FBLS_ERR_ARGUMENT, "null argument");
    if (nb < 1) return fail(ctx, FBLS_ERR_ARGUMENT, "nb must be positive");
    for (uint32_t p = 0; p < P; p++)
        if (!(scales[p] > 0.0) || !std::isfinite(scales[p]) ||
            !(ready->t_last * scales[p] < 16777216.0))  // the f32 forms' cells stay below 2^24
            return fail(ctx, FBLS_ERR_ARGUMENT, "scales must be positive with t * scale below 2^24");
    CK(cudaSetDevice(ctx->device), "set device");
    for (int k = 0; k < 5; k++) counts[k] = 0;
    if (P == 0 || ready->n == 0) return FBLS_OK;
    const size_t bytes = align256(P * sizeof(double)) + 5 * sizeof(unsigned long long);
    CK(ensure(ctx->rescore, bytes), "workspace");
    double* d_scales = as<double>(ctx->rescore);
    unsigned long long* d_counts =
        reinterpret_cast<unsigned long long*>(static_cast<unsigned char*>(ctx->rescore.ptr) + align256(P * sizeof(double)));
    const cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(d_scales, scales, P * sizeof(double), cudaMemcpyHostToDevice, s), "upload scales");
    CK(cudaMemsetAsync(d_counts, 0, 5 * sizeof(unsigned long long), s), "clear counts");
    k_bin_forms<<<(ready->n + 255) / 256, 256, 0, s>>>(ready->time, (int)ready->n, d_scales, (int)P, nb, d_counts);
    CK(cudaGetLastError(), "bin forms");
    ctx->counters.launches++;
    unsigned long long host[5];
    CK(cudaMemcpyAsync(host, d_counts, sizeof(host), cudaMemcpyDeviceToHost, s), "download counts");
    CK(cudaStreamSynchronize(s), "bin forms");
    for (int k = 0; k < 5; k++) counts[k] = host[k];
    return FBLS_OK;
}

static bool cta_size_ok(uint32_t th) { return th == 0 || th == 128 || th == 256 || th == 512 || th == 1024; }

static bool group_cap_ok(uint32_t g) { return g <= (uint32_t)WALK_MAX_GROUP && (g & (g - 1)) == 0; }

extern "C" int fbls_set_tuning(const fbls_tuning* tuning) {
    if (!tuning) return FBLS_ERR_ARGUMENT;
    FoldTuning t{};
    for (int c = 0; c < 32; c++) {
        const uint32_t g = tuning->fold_group_max[c], th = tuning->fold_threads[c], l = tuning->lockstep_min[c];
        if (!group_cap_ok(g) || !cta_size_ok(th)) return FBLS_ERR_ARGUMENT;
        if (l > 4096) return FBLS_ERR_ARGUMENT;
        t.group_cap[c] = g;
        t.threads[c] = th;
        t.lockstep_min[c] = l;
        if (tuning->fold_pair[c] > 1) return FBLS_ERR_ARGUMENT;
        t.pair[c] = tuning->fold_pair[c];
    }
    t.launch_periods = tuning->launch_periods;
    t.steal = tuning->fold_steal;
    t.fused_scan = tuning->fused_scan;
    if (tuning->map_lockstep_min > 4096) return FBLS_ERR_ARGUMENT;
    t.map_lockstep_min = tuning->map_lockstep_min;
    if (!cta_size_ok(tuning->map_threads) || !group_cap_ok(tuning->map_group_max)) return FBLS_ERR_ARGUMENT;
    t.map_threads = tuning->map_threads;
    t.map_group_max = tuning->map_group_max;
    if (tuning->batch_no_fill > 1) return FBLS_ERR_ARGUMENT;
    t.batch_no_fill = tuning->batch_no_fill;
    set_fold_tuning(t);
    return FBLS_OK;
}

extern "C" int fbls_get_tuning(fbls_tuning* tuning) {
    if (!tuning) return FBLS_ERR_ARGUMENT;
    FoldTuning t{};
    get_fold_tuning(&t);
    for (int c = 0; c < 32; c++) {
        tuning->fold_group_max[c] = t.group_cap[c];
        tuning->fold_threads[c] = t.threads[c];
        tuning->lockstep_min[c] = t.lockstep_min[c];
        tuning->fold_pair[c] = t.pair[c];
    }
    tuning->launch_periods = t.launch_periods;
    tuning->fold_steal = t.steal;
    tuning->fused_scan = t.fused_scan;
    tuning->map_lockstep_min = t.map_lockstep_min;
    tuning->map_threads = t.map_threads;
    tuning->map_group_max = t.map_group_max;
    tuning->batch_no_fill = t.batch_no_fill;
    return FBLS_OK;
}
