// Kernels of the proposal path (the learned pruning of the search): the coarse
// periodogram that feeds the proposal network.
//
// k_box_map: for each period of a launch and each duration of a small bank,
// the best box score over every phase, (a / rho) / sqrt(norm - hp^2 / c)
// with hp = norm = the template's weight sum, in f64 from the doubled prefix
// sums the fold writes; a template counts when its width is below nb / 2,
// it holds 3 .. n - 3 observations, a > 0 and the precision is positive, as in
// the scan's f64 pass (src/search/kernels.rs:428-455, :679-700). 0 when no
// template of the duration counts. One CTA of 256 threads per period; the job
// form (k_box_map_jobs) covers the periods of many folds, of many stars, in
// one launch.
#include "common.cuh"
#include "kernels.h"

namespace fbls {

namespace {
constexpr int MAP_THREADS = 256;
}

__device__ __forceinline__ void box_map_period(const MapArgs& a, const int f) {
    __shared__ double s_best[MAP_MAX_DURATIONS][MAP_THREADS / 32];
    const int tid = threadIdx.x;
    const int nb = a.nb;
    const int nd = a.nd;
    const size_t stride = 2 * (size_t)nb + 1;
    const double* rv = a.cum + (size_t)f * NF * stride + F_V * stride;
    const double* rw = a.cum + (size_t)f * NF * stride + F_W * stride;
    const double* rn = a.cum + (size_t)f * NF * stride + F_N * stride;
    const double scale = a.scales[f];
    const uint32_t half = (uint32_t)(nb / 2);
    uint32_t width[MAP_MAX_DURATIONS];
    bool ok[MAP_MAX_DURATIONS];
    double best[MAP_MAX_DURATIONS];
#pragma unroll
    for (int d = 0; d < MAP_MAX_DURATIONS; d++) {
        const uint32_t raw = d < nd ? template_width(a.durations[d], scale) : 1u;
        width[d] = min(raw, half);
        ok[d] = d < nd && raw < half;
        best[d] = 0.0;
    }
    for (int j = tid; j < nb; j += MAP_THREADS) {
#pragma unroll
        for (int d = 0; d < MAP_MAX_DURATIONS; d++) {
            if (!ok[d]) continue;
            const uint32_t k = width[d];
            const double count = __dsub_rn(rn[j + k], rn[j]);
            if (!(count >= 3.0 && count <= a.n - 3.0)) continue;
            const double av = __dsub_rn(rv[j + k], rv[j]);
            if (!(av > 0.0)) continue;
            const double w = __dsub_rn(rw[j + k], rw[j]);
            const double q = __dsub_rn(w, __ddiv_rn(__dmul_rn(w, w), a.baseline));
            if (!(q > 0.0)) continue;
            const double s = __ddiv_rn(__ddiv_rn(av, a.rho[d]), __dsqrt_rn(rmax(q, 1e-300)));
            if (s > best[d]) best[d] = s;
        }
    }
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int d = 0; d < MAP_MAX_DURATIONS; d++) {
        double v = best[d];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
        if (lane == 0) s_best[d][warp] = v;
    }
    __syncthreads();
    if (tid < nd) {
        double v = s_best[tid][0];
        for (int w = 1; w < MAP_THREADS / 32; w++) v = fmax(v, s_best[tid][w]);
        a.out[(size_t)f * nd + tid] = (float)v;
    }
}

__global__ void __launch_bounds__(MAP_THREADS) k_box_map(MapArgs a) { box_map_period(a, blockIdx.x); }

// Job j covers the CTAs [p0[j], p0[j + 1]), one per period of its fold.
__global__ void __launch_bounds__(MAP_THREADS) k_box_map_jobs(const MapArgs* __restrict__ jobs,
                                                              const int* __restrict__ p0, int njobs) {
    const int c = blockIdx.x;
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (p0[mid] <= c) lo = mid;
        else hi = mid - 1;
    }
    const MapArgs a = jobs[lo];
    box_map_period(a, c - p0[lo]);
}

// Sums of v and w over runs of observations (the time bins of a coarse map):
// bin b covers observations [starts[b], starts[b + 1]).
__global__ void k_bin_fields(const double* v, const double* w, const int* starts, int nbins, double* vb,
                             double* wb) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbins; b += gridDim.x * blockDim.x) {
        double sv = 0.0, sw = 0.0;
        for (int i = starts[b]; i < starts[b + 1]; i++) {
            sv += v[i];
            sw += w[i];
        }
        vb[b] = sv;
        wb[b] = sw;
    }
}

// The bins of many stars: job j covers the global bin indices [b0[j], b0[j + 1]).
__global__ void k_bin_fields_jobs(const BinJob* __restrict__ jobs, const int* __restrict__ b0, int njobs, int total) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        int lo = 0, hi = njobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (b0[mid] <= g) lo = mid;
            else hi = mid - 1;
        }
        const BinJob& j = jobs[lo];
        const int b = g - b0[lo];
        double sv = 0.0, sw = 0.0;
        for (int i = j.starts[b]; i < j.starts[b + 1]; i++) {
            sv += j.v[i];
            sw += j.w[i];
        }
        j.vb[b] = sv;
        j.wb[b] = sw;
    }
}

cudaError_t launch_bin_fields_jobs(const BinJob* jobs, const int* b0, int njobs, int total, cudaStream_t stream) {
    if (njobs < 1 || total < 1) return cudaErrorInvalidValue;
    const int blocks = (total + 255) / 256;
    k_bin_fields_jobs<<<blocks < 4096 ? blocks : 4096, 256, 0, stream>>>(jobs, b0, njobs, total);
    return cudaGetLastError();
}

cudaError_t launch_box_map_jobs(const MapArgs* jobs, const int* p0, int njobs, int total, cudaStream_t stream) {
    if (njobs < 1 || total < 1) return cudaErrorInvalidValue;
    k_box_map_jobs<<<total, MAP_THREADS, 0, stream>>>(jobs, p0, njobs);
    return cudaGetLastError();
}

// Network input of the proposal path: for map job j (star jobs[j].star) and
// channel (duration) c, f_t = log1p(max(map[t][c], 0)) over the job's P
// periods, standardised by its mean and (population) standard deviation + 1e-3,
// written to x[c][star][offset + t] (x is C x B x T, zeroed beforehand). Jobs
// with fewer than 8 periods are left at zero. One CTA per (job, channel).
__global__ void __launch_bounds__(256) k_map_features(const FeatJob* __restrict__ jobs, int B, int T,
                                                      float* __restrict__ x) {
    __shared__ double s_sum[2][8];
    const FeatJob j = jobs[blockIdx.x];
    const int c = blockIdx.y;
    if (j.P < 8 || c >= j.nd) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float* m = j.map;
    double sum = 0.0;
    for (int t = tid; t < j.P; t += blockDim.x) sum += (double)log1pf(fmaxf(m[(size_t)t * j.nd + c], 0.f));
    for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
    if (lane == 0) s_sum[0][warp] = sum;
    __syncthreads();
    double mu = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) mu += s_sum[0][w];
    mu /= (double)j.P;
    double var = 0.0;
    for (int t = tid; t < j.P; t += blockDim.x) {
        const double d = (double)log1pf(fmaxf(m[(size_t)t * j.nd + c], 0.f)) - mu;
        var += d * d;
    }
    for (int off = 16; off > 0; off >>= 1) var += __shfl_xor_sync(0xffffffffu, var, off);
    if (lane == 0) s_sum[1][warp] = var;
    __syncthreads();
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += s_sum[1][w];
    const double sd = sqrt(v / (double)j.P) + 1e-3;
    float* out = x + ((size_t)c * B + j.star) * T + j.offset;
    for (int t = tid; t < j.P; t += blockDim.x)
        out[t] = (float)(((double)log1pf(fmaxf(m[(size_t)t * j.nd + c], 0.f)) - mu) / sd);
}

cudaError_t launch_map_features(const FeatJob* jobs, int njobs, int channels, int B, int T, float* x,
                                cudaStream_t stream) {
    if (njobs < 1 || channels < 1 || channels > MAP_MAX_DURATIONS || B < 1 || T < 1) return cudaErrorInvalidValue;
    k_map_features<<<dim3(njobs, channels), 256, 0, stream>>>(jobs, B, T, x);
    return cudaGetLastError();
}

cudaError_t launch_bin_fields(const double* v, const double* w, const int* starts, int nbins, double* vb, double* wb,
                              cudaStream_t stream) {
    if (nbins < 1) return cudaErrorInvalidValue;
    const int blocks = (nbins + 255) / 256;
    k_bin_fields<<<blocks < 4096 ? blocks : 4096, 256, 0, stream>>>(v, w, starts, nbins, vb, wb);
    return cudaGetLastError();
}

cudaError_t launch_box_map(const MapArgs& a, int periods, cudaStream_t stream) {
    if (a.nd < 1 || a.nd > MAP_MAX_DURATIONS || a.nb < 2 || periods < 1) return cudaErrorInvalidValue;
    k_box_map<<<periods, MAP_THREADS, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace fbls
