// Biweight detrending on sm_100a (the raw-mode preparation's hot step):
// per observation the Tukey biweight location of the flux in a sliding time
// window, iterated from the window's lower median, and the relative residual
// flux / location - 1 (src/search/kernels.rs:1051-1110 with window_median
// :333-377; host side src/prep/curve.rs:256-329).
//
// One thread per observation, blocks of up to 128 consecutive observations;
// a block's union of windows is staged in shared memory when it fits
// BIWEIGHT_STAGE doubles (200 KB; the reference's stage is 4096 doubles and
// wider windows go to its CPU path), else the block is a single observation
// reading its window from global memory. Every median is the window's exact
// lower median, found as the reference does it: bisection on the value range
// (at most 64 halvings), then the smallest value at or above the bound; the
// weighted sums run over the window in order. All arithmetic rounds as the
// reference's (no contraction), so the output is the reference's bit for bit.

#include "common.cuh"
#include "kernels.h"

namespace fbls {

namespace {

// Lower median (the k-th smallest, k = (W - 1) / 2) of x[a..e) or of
// |x[j] - center| (window_median, kernels.rs:333-377).
template <typename Load>
__device__ double window_median(Load x, int a, int e, int k, double center, bool absolute) {
    auto value = [&](int j) {
        const double v = x(j);
        return absolute ? fabs(__dsub_rn(v, center)) : v;
    };
    double vlo = __builtin_huge_val(), vhi = -__builtin_huge_val();
    for (int j = a; j < e; j++) {
        const double v = value(j);
        vlo = fmin(vlo, v);
        vhi = fmax(vhi, v);
    }
    for (int it = 0; it < 64 && vhi > vlo; it++) {
        const double mid = __dmul_rn(0.5, __dadd_rn(vlo, vhi));
        if (mid <= vlo || mid >= vhi) break;
        int below = 0;
        for (int j = a; j < e; j++) below += value(j) < mid ? 1 : 0;
        if (below <= k)
            vlo = mid;
        else
            vhi = mid;
    }
    double best = __builtin_huge_val();
    for (int j = a; j < e; j++) {
        const double v = value(j);
        if (v >= vlo && v < best) best = v;
    }
    return best;
}

template <typename Load>
__device__ double biweight_point(Load x, int a, int e, int p, double c, int iterations) {
    const int k = (e - a - 1) / 2;
    double location = window_median(x, a, e, k, 0.0, false);
    for (int n = 0; n < iterations; n++) {
        const double loc = location;
        const double scale = fmax(__dmul_rn(c, window_median(x, a, e, k, loc, true)), 1e-12);
        double total = 0.0, acc = 0.0;
        for (int j = a; j < e; j++) {
            const double v = x(j);
            const double u = __ddiv_rn(__dsub_rn(v, loc), scale);
            if (fabs(u) < 1.0) {
                const double one = __dsub_rn(1.0, __dmul_rn(u, u));
                const double wt = __dmul_rn(one, one);
                total = __dadd_rn(total, wt);
                acc = __dadd_rn(acc, __dmul_rn(wt, v));
            }
        }
        if (total > 0.0) location = __ddiv_rn(acc, total);
    }
    return __dsub_rn(__ddiv_rn(x(p), location), 1.0);
}

__global__ void __launch_bounds__(BIWEIGHT_THREADS) k_biweight(BiweightArgs args) {
    extern __shared__ __align__(16) double win[];
    const int4 blk = reinterpret_cast<const int4*>(args.blocks)[blockIdx.x];  // first, count, ulo, uhi
    const int first = blk.x, count = blk.y, ulo = blk.z, uhi = blk.w;
    const bool staged = uhi - ulo <= BIWEIGHT_STAGE;
    if (staged)
        for (int q = threadIdx.x; q < uhi - ulo; q += blockDim.x) win[q] = args.flux[ulo + q];
    __syncthreads();
    if ((int)threadIdx.x >= count) return;
    const int p = first + threadIdx.x;
    const int a = (int)args.lo[p], e = (int)args.hi[p];
    double r;
    if (staged) {
        auto x = [&](int j) { return win[j - ulo]; };
        r = biweight_point(x, a, e, p, args.c, args.iterations);
    } else {
        const double* f = args.flux;
        auto x = [&](int j) { return f[j]; };
        r = biweight_point(x, a, e, p, args.c, args.iterations);
    }
    args.out[p] = r;
}

}  // namespace

cudaError_t launch_biweight(const BiweightArgs& a, int nblocks, size_t smem, cudaStream_t stream) {
    if (nblocks < 1 || smem > BIWEIGHT_STAGE * sizeof(double) || !a.flux || !a.lo || !a.hi || !a.blocks || !a.out)
        return cudaErrorInvalidValue;
    // The limit belongs to the module loaded in the current context; a context
    // made again after cudaDeviceReset reloads the module without it, so it is
    // set at every launch (a host-side attribute write, no device work).
    cudaError_t e = cudaFuncSetAttribute(k_biweight, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(BIWEIGHT_STAGE * sizeof(double)));
    if (e != cudaSuccess) return e;
    k_biweight<<<nblocks, BIWEIGHT_THREADS, smem, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace fbls
