// Peak-selection rescoring on sm_100a: the box sums of candidate rows over a
// family's observations outside the excluded set (rescore_rows,
// src/search/kernels.rs:936-990) and their in-transit counts over the merged
// time vector (count_rows, kernels.rs:993-1042).
//
// One CTA of 256 lanes per row, as the reference: lane l sums the
// observations i = l (mod 256) in increasing i, then the 256 partial sums meet
// in the reference's shared-memory tree (stride 128, 64, ..., 1), so the
// results are the reference's bit for bit. The reference visits every
// observation of every row; here a row's lanes first find, by binary search
// in the ascending times, the index range of every transit window
// [c + kP - D/2 - margin, c + kP + D/2 + margin] (margin 1e-6 d, far above
// the rounding of the reference's phase), and then visit only those indices,
// each tested with the reference's own phase expression. Out-of-transit
// observations add nothing in the reference either, so each lane's partial
// sum is formed from the same terms in the same order. A row whose windows
// do not fit the table (or whose period, epoch or duration is not a finite
// positive number) is scanned in full, as the reference does.
#include "common.cuh"
#include "kernels.h"

namespace fbls {

namespace {

constexpr int RB = RESCORE_BLOCK;          // lanes per row
constexpr int MAX_WINDOWS = 2048;          // transit windows a row may have for the windowed walk
constexpr double WINDOW_MARGIN = 1e-6;     // days

// First index with time[i] >= x (time ascending).
__device__ __forceinline__ int lower_bound(const double* time, int n, double x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (time[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// First index with time[i] > x.
__device__ __forceinline__ int upper_bound(const double* time, int n, double x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (time[mid] <= x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// The index ranges of a row's transit windows, centred on c + kP, into
// s_lo / s_hi (k from k0, `count` windows); false when the windowed walk does
// not apply. Every lane of the CTA calls it.
__device__ bool row_windows(const double* time, int n, double c, double period, double duration, int* s_lo,
                            int* s_hi, int* s_count) {
    __shared__ int s_ok;
    __shared__ long long s_k0;
    const int lane = threadIdx.x;
    if (lane == 0) {
        int ok = 0;
        long long k0 = 0, count = 0;
        if (n > 0 && period > 0.0 && isfinite(period) && isfinite(c) && duration >= 0.0 && isfinite(duration)) {
            const double klo = floor((time[0] - c) / period) - 1.0;
            const double khi = ceil((time[n - 1] - c) / period) + 1.0;
            if (khi - klo + 1.0 <= (double)MAX_WINDOWS) {
                k0 = (long long)klo;
                count = (long long)(khi - klo) + 1;
                ok = 1;
            }
        }
        s_ok = ok;
        s_k0 = k0;
        *s_count = (int)count;
    }
    __syncthreads();
    if (!s_ok) return false;
    const int count = *s_count;
    const double half = duration / 2.0;
    for (int j = lane; j < count; j += RB) {
        const double centre = c + (double)(s_k0 + j) * period;
        s_lo[j] = lower_bound(time, n, centre - half - WINDOW_MARGIN);
        s_hi[j] = upper_bound(time, n, centre + half + WINDOW_MARGIN);
    }
    __syncthreads();
    return true;
}

// Calls visit(i) for every index of the windows' union that is = lane
// (mod RB), in increasing i.
template <typename Visit>
__device__ __forceinline__ void walk_windows(const int* s_lo, const int* s_hi, int count, Visit visit) {
    const int lane = threadIdx.x;
    int done = 0;  // indices below `done` were covered by earlier windows
    for (int j = 0; j < count; j++) {
        const int start = max(s_lo[j], done);
        const int end = s_hi[j];
        if (start < end) {
            for (int i = start + ((lane - start) % RB + RB) % RB; i < end; i += RB) visit(i);
            done = end;
        }
    }
}

// The reference's tree over RB partial sums (stride RB/2 ... 1).
template <typename T>
__device__ __forceinline__ T tree_sum(T* red, T x) {
    const int lane = threadIdx.x;
    red[lane] = x;
    __syncthreads();
    for (int stride = RB / 2; stride > 0; stride >>= 1) {
        if (lane < stride) red[lane] = red[lane] + red[lane + stride];
        __syncthreads();
    }
    const T total = red[0];
    __syncthreads();
    return total;
}

__global__ void __launch_bounds__(RB) k_rescore_rows(RescoreArgs a) {
    __shared__ int s_lo[MAX_WINDOWS], s_hi[MAX_WINDOWS], s_count;
    __shared__ double s_red[RB];
    const int r = blockIdx.x;
    const int lane = threadIdx.x;
    const double period = a.rows[3 * r], epoch = a.rows[3 * r + 1], duration = a.rows[3 * r + 2];
    const double inverse = __ddiv_rn(1.0, period);
    const double half = duration / 2.0;
    double sa = 0.0, shp = 0.0, snorm = 0.0;
    auto visit = [&](int i) {
        if (a.excluded[i] == 0) {
            const double x = __dadd_rn(__dmul_rn(__dsub_rn(__dadd_rn(a.time[i], a.origin), epoch), inverse), 0.5);
            const double phase = __dmul_rn(__dsub_rn(__dsub_rn(x, floor(x)), 0.5), period);
            if (fabs(phase) <= half) {
                sa = __dadd_rn(sa, a.v[i]);
                shp = __dadd_rn(shp, a.w[i]);
                snorm = __dadd_rn(snorm, a.w[i]);
            }
        }
    };
    if (row_windows(a.time, a.n, __dsub_rn(epoch, a.origin), period, duration, s_lo, s_hi, &s_count)) {
        walk_windows(s_lo, s_hi, s_count, visit);
    } else {
        for (int i = lane; i < a.n; i += RB) visit(i);
    }
    const double ta = tree_sum(s_red, sa);
    const double thp = tree_sum(s_red, shp);
    const double tn = tree_sum(s_red, snorm);
    if (lane == 0) {
        a.sums[3 * r] = ta;
        a.sums[3 * r + 1] = thp;
        a.sums[3 * r + 2] = tn;
    }
}

__global__ void __launch_bounds__(RB) k_count_rows(RescoreArgs a) {
    __shared__ int s_lo[MAX_WINDOWS], s_hi[MAX_WINDOWS], s_count;
    __shared__ uint32_t s_red[RB];
    const int r = blockIdx.x;
    const int lane = threadIdx.x;
    const double period = a.rows[3 * r], epoch = a.rows[3 * r + 1], duration = a.rows[3 * r + 2];
    const double inverse = __ddiv_rn(1.0, period);
    const double half = duration / 2.0;
    uint32_t total = 0, unshared = 0;
    auto visit = [&](int i) {
        const double x = __dadd_rn(__dmul_rn(__dsub_rn(a.time[i], epoch), inverse), 0.5);
        const double phase = __dmul_rn(__dsub_rn(__dsub_rn(x, floor(x)), 0.5), period);
        if (fabs(phase) <= half) {
            total += 1u;
            unshared += a.excluded[i] == 0 ? 1u : 0u;
        }
    };
    if (row_windows(a.time, a.n, epoch, period, duration, s_lo, s_hi, &s_count)) {
        walk_windows(s_lo, s_hi, s_count, visit);
    } else {
        for (int i = lane; i < a.n; i += RB) visit(i);
    }
    const uint32_t t = tree_sum(s_red, total);
    const uint32_t u = tree_sum(s_red, unshared);
    if (lane == 0) {
        a.counts[2 * r] = t;
        a.counts[2 * r + 1] = u;
    }
}

}  // namespace

cudaError_t launch_rescore_rows(const RescoreArgs& a, cudaStream_t stream) {
    if (a.R < 1 || a.n < 0 || !a.time || !a.v || !a.w || !a.excluded || !a.rows || !a.sums) return cudaErrorInvalidValue;
    k_rescore_rows<<<a.R, RB, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_count_rows(const RescoreArgs& a, cudaStream_t stream) {
    if (a.R < 1 || a.n < 0 || !a.time || !a.excluded || !a.rows || !a.counts) return cudaErrorInvalidValue;
    k_count_rows<<<a.R, RB, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace fbls
