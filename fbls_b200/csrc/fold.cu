// Deterministic phase fold and doubled prefix sums on sm_100a.
//
// One CTA folds G periods (a power of two, at most 32) of one family.
// Because times are sorted, the cell floor(t * scale) never decreases along
// the observations, so every cell is one contiguous run of observations.
// The CTA needs no atomic:
//
//   1. the observations are cut (on the host) into chunks spanning at most
//      min(nb - 2, SPAN) cells at every period of the launch, so the cells of
//      one chunk fall in distinct bins;
//   2. the chunk is split into NS equal segments. Lane (q, s) of the CTA owns
//      period q and segment s and folds every run that starts in its
//      segment, continuing past the segment's end while the run lasts: it
//      loads the bin's sums, adds the run's observations one by one, and
//      stores them back. With G = 32 a warp's lanes are the 32 periods of one
//      segment: they step through the same observations together, so every
//      shared-memory read is a broadcast and loop control is shared.
//   3. the bins live in shared memory: the whole histogram when it fits
//      ("full" mode), otherwise a window of the chunk's cells, loaded from
//      and stored back to a global histogram around each chunk ("window"
//      mode; the cells of a chunk are consecutive, so its bins are too).
//
// Each bin's sums are thus formed in observation order, exactly as a
// sequential fold does, so the result is reproducible run to run and equal
// bit for bit to the CPU oracle (the reference's f64 atomics,
// src/search/kernels.rs:491, :540, give some order of the same additions).
// The doubled prefix sums then follow the association of the reference's
// prefix_block (kernels.rs:237-309), one warp per (period, field) row, and
// are written as f64 and (hi, lo) f32 pairs.
#include "common.cuh"
#include "kernels.h"

namespace fbls {

// v mod nb from the f64 reciprocal, corrected by one step (the quotient
// estimate is within one of the true quotient for v < 2^32), as the
// reference's phase_cell does (kernels.rs:314-327).
__device__ __forceinline__ uint32_t mod_nb(uint32_t v, uint32_t nb, double inv_nb) {
    uint32_t q = (uint32_t)__dmul_rn((double)v, inv_nb);
    uint32_t r = v - q * nb;
    if ((int32_t)r < 0)
        r += nb;
    else if (r >= nb)
        r -= nb;
    return r;
}

__device__ __forceinline__ float2 split_pair(double value) {
    float hi = __double2float_rn(value);
    float lo = __double2float_rn(__dsub_rn(value, (double)hi));
    return make_float2(hi, lo);
}

// Doubled exclusive prefix of one row by one warp, in the order of the
// reference's prefix_block: per segment of 256 bins, 8 groups of 32 scanned
// by Hillis-Steele steps, offset = carry + earlier group totals in order,
// carry += (sum of the 8 group totals); second copy = first + final carry.
template <typename Load>
__device__ __forceinline__ void prefix_row(Load load, int nb, double* __restrict__ out64,
                                           float2* __restrict__ out32) {
    const int lane = threadIdx.x & 31;
    if (lane == 0) {
        out64[0] = 0.0;
        out32[0] = make_float2(0.f, 0.f);
    }
    double carry = 0.0;
    for (int seg = 0; seg < nb; seg += 256) {
        double offset = carry;
        double total = 0.0;
#pragma unroll 1
        for (int g = 0; g < 8; g++) {
            const int b = seg + g * 32 + lane;
            double x = b < nb ? load(b) : 0.0;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                double o = __shfl_up_sync(0xffffffffu, x, off);
                if (lane >= off) x = __dadd_rn(x, o);
            }
            const double wt = __shfl_sync(0xffffffffu, x, 31);
            if (b < nb) {
                const double val = __dadd_rn(x, offset);
                out64[b + 1] = val;
                out32[b + 1] = split_pair(val);
            }
            offset = __dadd_rn(offset, wt);
            total = __dadd_rn(total, wt);
        }
        carry = __dadd_rn(carry, total);
    }
    for (int b = lane; b < nb; b += 32) {
        const double val = __dadd_rn(out64[b + 1], carry);
        out64[nb + b + 1] = val;
        out32[nb + b + 1] = split_pair(val);
    }
}

__global__ void __launch_bounds__(512, 2) k_fold(FoldArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double s_scale[MAX_GROUP];
    __shared__ uint32_t s_v0[MAX_GROUP], s_r0[MAX_GROUP];

    const int tid = threadIdx.x;
    const int T = blockDim.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int nb = a.nb;
    const uint32_t unb = (uint32_t)nb;
    const double inv_nb = 1.0 / (double)nb;
    const int G = a.group;  // power of two <= 32
    const int gshift = __ffs(G) - 1;
    const int S = 32 / G;   // segments per warp
    const int NS = (T / 32) * S;
    const int g0 = blockIdx.x * G;
    const int g = min(G, a.periods - g0);
    const int q = lane & (G - 1);
    const int seg = warp * S + (lane >> gshift);
    const bool full = a.window == 0;
    const int rows = full ? nb : a.window;  // bins per period held in shared memory
    const int rs = a.row_stride;            // >= rows, odd

    // Shared memory: staging t, v, w [stage_field] | sums v, w [G][rs] | counts [G][rs].
    double* st = reinterpret_cast<double*>(smem);
    double* sv = st + a.stage_field;
    double* sw = sv + a.stage_field;
    double* rv = sw + a.stage_field;
    double* rw = rv + (size_t)G * rs;
    uint32_t* rc = reinterpret_cast<uint32_t*>(rw + (size_t)G * rs);
    // Global histogram of this CTA's periods (window mode): [3][G][nb].
    double* gv = a.hist_global ? a.hist_global + (size_t)blockIdx.x * G * nb * 3 : nullptr;
    double* gw = gv ? gv + (size_t)G * nb : nullptr;
    uint32_t* gc = gv ? reinterpret_cast<uint32_t*>(gw + (size_t)G * nb) : nullptr;

    if (tid < g) s_scale[tid] = a.scales[g0 + tid];
    if (full) {
        for (int e = tid; e < G * rs; e += T) {
            rv[e] = 0.0;
            rw[e] = 0.0;
            rc[e] = 0u;
        }
    } else {
        for (int e = tid; e < G * nb; e += T) {
            gv[e] = 0.0;
            gw[e] = 0.0;
            gc[e] = 0u;
        }
    }
    __syncthreads();
    const bool live = q < g;
    const double scale = live ? s_scale[q] : 0.0;
    double* lv = rv + (size_t)q * rs;
    double* lw = rw + (size_t)q * rs;
    uint32_t* lc = rc + (size_t)q * rs;

    for (int c = 0; c < a.nchunks; c++) {
        const int i0 = a.chunks[c];
        const int len = a.chunks[c + 1] - i0;
        const int R = (len + NS - 1) / NS;
        // Stage the chunk, observation k at (k % R) * NS + k / R.
        for (int k = tid; k < len; k += T) {
            const int sk = k / R;
            const int at = (k - sk * R) * NS + sk;
            st[at] = a.time[i0 + k];
            sv[at] = a.v[i0 + k];
            sw[at] = a.w[i0 + k];
        }
        __syncthreads();
        if (!full) {
            // Window of the chunk's cells: slot u holds the bin of cell v0 + u.
            if (tid < g) {
                const uint32_t v0 = (uint32_t)floor(__dmul_rn(st[0], s_scale[tid]));
                s_v0[tid] = v0;
                s_r0[tid] = mod_nb(v0, unb, inv_nb);
            }
            __syncthreads();
            for (int e = tid; e < g * rows; e += T) {
                const int qq = e / rows, u = e - qq * rows;
                uint32_t bin = s_r0[qq] + (uint32_t)u;
                if (bin >= unb) bin -= unb;
                const size_t src = (size_t)qq * nb + bin, dst = (size_t)qq * rs + u;
                rv[dst] = gv[src];
                rw[dst] = gw[src];
                rc[dst] = gc[src];
            }
            __syncthreads();
        }

        const int a0 = seg * R;
        const int e0 = min(a0 + R, len);
        bool done = !live || a0 >= len;
        bool skip = false;
        int k = a0, j = 0, sk = seg, k0 = a0;
        uint32_t slot = 0, c0 = 0, v0 = full ? 0u : (live ? s_v0[q] : 0u);
        double nextb = 0.0, av = 0.0, aw = 0.0;
        if (!done) {
            const uint32_t v = (uint32_t)floor(__dmul_rn(st[seg], scale));
            if (a0 > 0) skip = (uint32_t)floor(__dmul_rn(st[(R - 1) * NS + seg - 1], scale)) == v;
            nextb = (double)v + 1.0;
            slot = full ? mod_nb(v, unb, inv_nb) : v - v0;
            if (!skip) {
                av = lv[slot];
                aw = lw[slot];
                c0 = lc[slot];
            }
        }
        while (__any_sync(0xffffffffu, !done)) {
            if (done) continue;
            const int at = j * NS + sk;
            if (!skip) {
                av = __dadd_rn(av, sv[at]);
                aw = __dadd_rn(aw, sw[at]);
            }
            ++k;
            if (++j == R) {
                j = 0;
                ++sk;
            }
            bool bnd = true;
            double x = 0.0;
            if (k < len) {
                x = __dmul_rn(st[j * NS + sk], scale);
                bnd = x >= nextb;
            }
            if (bnd || (skip && k >= e0)) {
                if (bnd && !skip) {
                    lv[slot] = av;
                    lw[slot] = aw;
                    lc[slot] = c0 + (uint32_t)(k - k0);
                }
                if (k >= e0) {
                    done = true;  // the next run starts in the next segment
                } else {
                    const double after = __dadd_rn(nextb, 1.0);
                    if (x < after) {  // the next cell
                        nextb = after;
                        slot = (full && slot + 1 == unb) ? 0u : slot + 1;
                    } else {  // empty cells in between
                        const uint32_t vn = (uint32_t)floor(x);
                        nextb = (double)vn + 1.0;
                        slot = full ? mod_nb(vn, unb, inv_nb) : vn - v0;
                    }
                    skip = false;
                    av = lv[slot];
                    aw = lw[slot];
                    c0 = lc[slot];
                    k0 = k;
                }
            }
        }
        __syncthreads();
        if (!full) {
            for (int e = tid; e < g * rows; e += T) {
                const int qq = e / rows, u = e - qq * rows;
                uint32_t bin = s_r0[qq] + (uint32_t)u;
                if (bin >= unb) bin -= unb;
                const size_t dst = (size_t)qq * nb + bin, src = (size_t)qq * rs + u;
                gv[dst] = rv[src];
                gw[dst] = rw[src];
                gc[dst] = rc[src];
            }
        }
        __syncthreads();
    }

    // Histogram of period qq, bin b.
    auto hv = [&](int qq, int b) { return full ? rv[(size_t)qq * rs + b] : gv[(size_t)qq * nb + b]; };
    auto hw = [&](int qq, int b) { return full ? rw[(size_t)qq * rs + b] : gw[(size_t)qq * nb + b]; };
    auto hc = [&](int qq, int b) { return full ? rc[(size_t)qq * rs + b] : gc[(size_t)qq * nb + b]; };
    if (a.hist_out) {
        // Raw histograms, field-major [3][nb] (the evidence fold, one period).
        for (int p = tid; p < nb; p += T) {
            a.hist_out[p] = hv(0, p);
            a.hist_out[nb + p] = hw(0, p);
            a.hist_out[2 * (size_t)nb + p] = (double)hc(0, p);
        }
        return;
    }
    const size_t stride = 2 * (size_t)nb + 1;
    for (int row = warp; row < g * NF; row += T / 32) {
        const int qq = row / NF, f = row - (row / NF) * NF;
        double* out64 = a.cum + ((size_t)(g0 + qq) * NF + f) * stride;
        float2* out32 = a.cum32 + ((size_t)(g0 + qq) * NF + f) * stride;
        if (f == F_V)
            prefix_row([&](int bb) { return hv(qq, bb); }, nb, out64, out32);
        else if (f == F_W)
            prefix_row([&](int bb) { return hw(qq, bb); }, nb, out64, out32);
        else
            prefix_row([&](int bb) { return (double)hc(qq, bb); }, nb, out64, out32);
    }
}

namespace {
constexpr size_t FOLD_SMEM_TARGET = 110 * 1024;  // two CTAs per SM
constexpr int FOLD_CTA_THREADS = 512;
constexpr int FOLD_STAGE_CAP = 1024;              // observations per chunk at most
constexpr int FOLD_SPAN_MAX = 256;                // window cells at most
constexpr size_t BIN_BYTES = 2 * sizeof(double) + sizeof(uint32_t);
}  // namespace

// Launch shape: a power-of-two period group (32 when the launch fills every
// SM twice), "full" mode when the group's histograms fit next to the
// staging area in half of an SM's shared memory, else "window" mode with the
// largest window that fits.
FoldShape fold_group_shape(int nb, int periods, int sm_count) {
    FoldShape s{};
    int g = MAX_GROUP;
    while (g > 1 && (size_t)(g / 2) * 2 * sm_count >= (size_t)periods) g /= 2;
    s.group = g;
    s.threads = FOLD_CTA_THREADS;
    const int ns = (FOLD_CTA_THREADS / 32) * (32 / g);
    s.stage_field = FOLD_STAGE_CAP + ns;
    const size_t stage = 3 * sizeof(double) * (size_t)s.stage_field;
    const size_t room = FOLD_SMEM_TARGET - stage;
    const int full_rs = nb | 1;
    if ((size_t)g * full_rs * BIN_BYTES <= room) {
        s.window = 0;
        s.row_stride = full_rs;
        s.hist_in_smem = true;
        s.span_cap = nb;
    } else {
        int rows = (int)(room / ((size_t)g * BIN_BYTES)) - 1;
        if (rows > FOLD_SPAN_MAX + 1) rows = FOLD_SPAN_MAX + 1;
        s.window = rows;  // cells v0 .. v0 + rows - 1
        s.row_stride = rows | 1;
        s.hist_in_smem = false;
        s.span_cap = rows - 1;
    }
    s.chunk_cap = FOLD_STAGE_CAP;
    s.smem = stage + (size_t)g * s.row_stride * BIN_BYTES;
    return s;
}

int fold_chunks(const double* time, int n, double scale_max, int nb, int span_cap, int chunk_cap, int* out,
                int capacity) {
    // A chunk spans less than `span` days, hence at most min(nb, span_cap) - 2
    // + 1 distinct cells at any scale <= scale_max (floor(x) - floor(y) <
    // x - y + 1): its cells are distinct bins and fit the window.
    const int cells = (nb < span_cap ? nb : span_cap) - 4;
    const double span = (double)(cells > 1 ? cells : 1) / scale_max;
    int count = 0;
    int i0 = 0;
    while (i0 < n) {
        if (count + 2 > capacity) return -1;
        out[count++] = i0;
        const double tlim = time[i0] + span;
        int lo = i0 + 1, hi = i0 + chunk_cap < n ? i0 + chunk_cap : n;
        // first index in [i0 + 1, hi) with time >= tlim, else hi
        while (lo < hi) {
            const int mid = lo + (hi - lo) / 2;
            if (time[mid] < tlim)
                lo = mid + 1;
            else
                hi = mid;
        }
        i0 = lo;
    }
    out[count] = n;
    return count;
}

cudaError_t launch_fold(const FoldArgs& a, const FoldShape& shape, cudaStream_t stream) {
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(k_fold, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MAX_FOLD_SMEM);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    if (shape.smem > MAX_FOLD_SMEM || a.group != shape.group || a.group > MAX_GROUP || a.group < 1 ||
        (a.group & (a.group - 1)) != 0 || a.nchunks < 1 || shape.threads != FOLD_CTA_THREADS ||
        a.stage_field != shape.stage_field || a.window != shape.window || a.row_stride != shape.row_stride ||
        (a.window != 0 && a.hist_global == nullptr))
        return cudaErrorInvalidValue;
    const int blocks = (a.periods + a.group - 1) / a.group;
    k_fold<<<blocks, shape.threads, shape.smem, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace fbls
