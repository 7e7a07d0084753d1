// Fold, doubled prefix sums, tile scan and merge of the FBLS signal scan on
// sm_100a. Semantics follow src/search/kernels.rs; the layout of the work on
// the GPU is this project's own:
//
//  * the fold and prefix sums are in fold.cu;
//  * k_scan_tiles: one CTA of TILE lanes per (tile, period), the reference's
//    two-pass f32 pre-rank / f64 rescan (kernels.rs:610-845).
//  * k_merge: best tile per period (kernels.rs:1115-1155).
#include "common.cuh"
#include "kernels.h"
#include "scan_tile.cuh"

namespace fbls {

// ---------------------------------------------------------------------------
// Tile scan (kernels.rs:610-845): scan_tile (scan_tile.cuh) over the fold's
// global rows, one CTA of TILE threads per (tile, period). (A warp form with
// four lanes per thread and no barriers measured slower on B200: 128
// registers leave 16 warps per SM; the group form keeps 32 at 64 registers.)
// ---------------------------------------------------------------------------

__device__ __forceinline__ void scan_tile_cta(const ScanArgs& a, const int tile, const int f, const int tiles) {
    __shared__ TileScratch sc;
    GlobalRows rows;
    rows.stride = 2 * (size_t)a.nb + 1;
    rows.r64 = a.cum ? a.cum + (size_t)f * NF * rows.stride : nullptr;
    rows.r32 = a.cum32 + (size_t)f * NF * rows.stride;
    const size_t idx = (size_t)f * tiles + tile;
    scan_tile(a, rows, CtaGroup{}, sc, tile, a.scales[f], a.parts + idx * PART_STRIDE, a.keys + idx, a.flags + idx);
}

// Eight CTAs per SM (64 registers): the f32 pass keeps its state in registers;
// the few spills are on the f64 rescan and winner paths.
__global__ void __launch_bounds__(TILE, 8) k_scan_tiles(ScanArgs a) {
    scan_tile_cta(a, blockIdx.x, blockIdx.y, gridDim.x);
}

// Many scans in one launch: CTA c is tile (c - cta0[j]) % tiles of period
// (c - cta0[j]) / tiles of job j, where cta0[j] <= c < cta0[j + 1].
__global__ void __launch_bounds__(TILE, 8) k_scan_jobs(const ScanArgs* __restrict__ jobs,
                                                       const int* __restrict__ cta0, int njobs) {
    int lo = 0, hi = njobs - 1;
    const int c = blockIdx.x;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (cta0[mid] <= c)
            lo = mid;
        else
            hi = mid - 1;
    }
    const ScanArgs& a = jobs[lo];
    const int tiles = (a.nb + TILE - 1) / TILE;
    const int local = c - cta0[lo];
    scan_tile_cta(a, local % tiles, local / tiles, tiles);
}

// Best tile per period by (score, lowest key) (kernels.rs:1115-1155). Writes
// records at `offset` so one buffer collects a whole band; flags are ORed.
__device__ __forceinline__ void merge_period(const MergeArgs& a, const int f) {
    const size_t idx = (size_t)f * a.tiles;
    merge_tiles(a.parts + idx * PART_STRIDE, a.keys + idx, a.flags + idx, a.tiles, a, f);
}

// ---------------------------------------------------------------------------
// Launchers.
// ---------------------------------------------------------------------------

// Single-event scan (kernels.rs:851-921): one thread per phase j of the
// single trial period; for every duration whose box is usable (width below
// nb / 2, 3 .. n - 3 observations) and every shape, the exact f64 score
// (a / rho) / sqrt(norm - hp^2 / c); a template reaching the threshold takes
// a slot from the counter. The host orders the records by (j, duration,
// shape), so the output does not depend on the order of the appends.
__global__ void __launch_bounds__(TILE) k_scan_all(EventArgs a) {
    const uint32_t nb = (uint32_t)a.nb;
    const uint32_t j = blockIdx.x * TILE + threadIdx.x;
    if (j >= nb) return;
    GlobalRows rows;
    rows.stride = 2 * (size_t)nb + 1;
    rows.r64 = a.cum;
    rows.r32 = nullptr;
    const uint32_t half = nb / 2;
    for (int di = 0; di < a.nd; di++) {
        const uint32_t raw = template_width(a.durations[di], a.scale);
        const uint32_t k = raw < half ? raw : half;
        const double r = a.rho[di];
        const double count = rows.i64(F_N, j, k);
        const double w = rows.i64(F_W, j, k);
        const double av = rows.i64(F_V, j, k);
        if (!(raw < half && count >= 3.0 && count <= a.n - 3.0)) continue;
        for (int si = 0; si < a.ns; si++) {
            double aa, hp, norm;
            shape_sums64(rows, j, k, av, w, w, a.ingress[si], a.factors, si, a.layers, aa, hp, norm);
            const double q = __dsub_rn(norm, __ddiv_rn(__dmul_rn(hp, hp), a.baseline));
            if (!(aa > 0.0 && q > 0.0)) continue;
            const double score = __ddiv_rn(__ddiv_rn(aa, r), __dsqrt_rn(q));
            if (score >= a.threshold) {
                const uint32_t slot = atomicAdd(a.counter, 1u);
                if (slot < a.capacity) {
                    double* rec = a.records + (size_t)slot * EVENT_RECORD;
                    rec[0] = (double)j;
                    rec[1] = (double)k;
                    rec[2] = score;
                    rec[3] = __ddiv_rn(aa, q);
                    rec[4] = (double)di;
                    rec[5] = (double)si;
                }
            }
        }
    }
}

cudaError_t launch_scan_all(const EventArgs& a, cudaStream_t stream) {
    if (a.nb < 2 || a.nd < 1 || a.nd > MAX_DURATIONS || a.ns < 1 || a.ns > MAX_SHAPES || a.layers < 1 ||
        a.layers > MAX_LAYERS || !a.cum || !a.counter || (a.capacity && !a.records))
        return cudaErrorInvalidValue;
    k_scan_all<<<(a.nb + TILE - 1) / TILE, TILE, 0, stream>>>(a);
    return cudaGetLastError();
}

int scan_ctas_per_period(int nb) { return (nb + TILE - 1) / TILE; }

cudaError_t launch_scan_tiles(const ScanArgs& a, int periods, cudaStream_t stream) {
    dim3 grid((a.nb + TILE - 1) / TILE, periods);
    k_scan_tiles<<<grid, TILE, 0, stream>>>(a);
    return cudaGetLastError();
}

__global__ void k_merge(MergeArgs a) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < a.periods) merge_period(a, f);
}

// Many merges in one launch: thread i merges period i - p0[j] of job j.
__global__ void k_merge_jobs(const MergeArgs* __restrict__ jobs, const int* __restrict__ p0, int njobs,
                             int total) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (p0[mid] <= i)
            lo = mid;
        else
            hi = mid - 1;
    }
    merge_period(jobs[lo], i - p0[lo]);
}

cudaError_t launch_scan_jobs(const ScanArgs* jobs, const int* cta0, int njobs, int ctas, cudaStream_t stream) {
    if (njobs < 1 || ctas < 1) return cudaErrorInvalidValue;
    k_scan_jobs<<<ctas, TILE, 0, stream>>>(jobs, cta0, njobs);
    return cudaGetLastError();
}

cudaError_t launch_merge_jobs(const MergeArgs* jobs, const int* p0, int njobs, int total, cudaStream_t stream) {
    if (njobs < 1 || total < 1) return cudaErrorInvalidValue;
    k_merge_jobs<<<(total + 127) / 128, 128, 0, stream>>>(jobs, p0, njobs, total);
    return cudaGetLastError();
}

cudaError_t launch_merge(const MergeArgs& a, cudaStream_t stream) {
    k_merge<<<(a.periods + 127) / 128, 128, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace fbls
