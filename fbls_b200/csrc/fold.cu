// Deterministic phase fold and doubled prefix sums on sm_100a.
//
// One CTA folds G periods (a power of two) of one family, with 32 / G of its
// warps per period. Because times are sorted, the cell floor(t * scale)
// never decreases along the observations, so every cell is one contiguous
// run of observations. The CTA needs no atomic:
//
//   1. the observations are cut (on the host) into chunks spanning at most
//      nb - 2 cells at every period of the launch, so the cells of one chunk
//      fall in distinct bins; a chunk is staged in shared memory;
//   2. each period's lanes split the chunk into equal segments, and every
//      lane moves its segment's start forward to the first run boundary of
//      its own period at or after it; a lane folds the runs from its start
//      up to the next lane's start, so every run belongs to exactly one lane;
//   3. the lanes of a warp step through their runs together, one
//      observation per step: add (v, w) to the run's sums, and at a cell
//      boundary store the sums to the bin and load the next bin's.
//
// Each bin's sums are thus formed in observation order, exactly as a
// sequential fold does, so the result is reproducible run to run and equal
// bit for bit to the CPU oracle (the reference's f64 atomics,
// src/search/kernels.rs:491, :540, give some order of the same additions).
// k_fold_walk (below) is the same scheme with the chunks staged by TMA; it
// folds every nb whose histograms fit shared memory, and k_fold the rest.
// The doubled prefix sums then follow the association of the reference's
// prefix_block (kernels.rs:237-309), one warp per (period, field) row, and
// are written as f64 and (hi, lo) f32 pairs.

#include <atomic>

#include "bulk.cuh"
#include "common.cuh"
#include "kernels.h"
#include "scan_tile.cuh"

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

__device__ __forceinline__ uint32_t cell_of(double t, double scale) {
    return (uint32_t)floor(__dmul_rn(t, scale));
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

// One (period, field) row of a walking-fold CTA's shared-memory histograms:
// the v or w sums (every other double of the period's double2 bins) or the
// counts. The prefix epilogues overwrite a bin with its prefix value once
// they have read it (a count prefix is an integer below 2^32).
struct HistRow {
    double* d;    // v or w sums, stride 2 doubles; null for the counts
    uint32_t* c;  // counts
    __device__ __forceinline__ double load(int b) const { return d ? d[2 * b] : (double)c[b]; }
    __device__ __forceinline__ void store(int b, double v) const {
        if (d)
            d[2 * b] = v;
        else
            c[b] = (uint32_t)v;
    }
};

// Inclusive Hillis-Steele scan of a warp's 32 values (the association of
// prefix_row and of the reference's prefix_block groups).
__device__ __forceinline__ double warp_scan(double x, int lane) {
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double o = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x = __dadd_rn(x, o);
    }
    return x;
}

// prefix_row of a shared-memory row by one warp, with the first copy kept in
// place, so the second copy (first + final carry) is read from shared memory
// rather than back from the global rows. With global = false only the
// in-place copy is made. Returns the final carry.
__device__ __forceinline__ double prefix_row_smem(const HistRow& r, int nb, bool global, double* __restrict__ out64,
                                                  float2* __restrict__ out32) {
    const int lane = threadIdx.x & 31;
    if (global && lane == 0) {
        if (out64) out64[0] = 0.0;
        out32[0] = make_float2(0.f, 0.f);
    }
    double carry = 0.0;
    for (int seg = 0; seg < nb; seg += 256) {
        double offset = carry;
        double total = 0.0;
#pragma unroll 1
        for (int g = 0; g < 8; g++) {
            const int b = seg + g * 32 + lane;
            const double x = warp_scan(b < nb ? r.load(b) : 0.0, lane);
            const double wt = __shfl_sync(0xffffffffu, x, 31);
            if (b < nb) {
                const double val = __dadd_rn(x, offset);
                if (global) {
                    if (out64) out64[b + 1] = val;
                    out32[b + 1] = split_pair(val);
                }
                r.store(b, val);
            }
            offset = __dadd_rn(offset, wt);
            total = __dadd_rn(total, wt);
        }
        carry = __dadd_rn(carry, total);
    }
    if (global)
        for (int b = lane; b < nb; b += 32) {  // bins this lane stored above
            const double val = __dadd_rn(r.load(b), carry);
            if (out64) out64[nb + b + 1] = val;
            out32[nb + b + 1] = split_pair(val);
        }
    return carry;
}

// The 256-bin segment `seg` of a row, by one warp, as prefix_row does it.
// SEG_TOTAL: returns the segment's total (the sum, in order, of its eight
// group totals) and writes nothing. SEG_GLOBAL: with `carry` (entering the
// segment) and `final` (the row's last carry) known, writes both copies to
// the global rows. SEG_IN_PLACE: stores the first copy in place.
constexpr int SEG_TOTAL = 0, SEG_GLOBAL = 1, SEG_IN_PLACE = 2;
__device__ __forceinline__ double prefix_segment(const HistRow& r, int nb, int seg, double carry, double final,
                                                 int mode, double* __restrict__ out64,
                                                 float2* __restrict__ out32) {
    const int lane = threadIdx.x & 31;
    double offset = carry;
    double total = 0.0;
#pragma unroll 1
    for (int g = 0; g < 8; g++) {
        const int b = seg + g * 32 + lane;
        const double x = warp_scan(b < nb ? r.load(b) : 0.0, lane);
        const double wt = __shfl_sync(0xffffffffu, x, 31);
        if (mode == SEG_GLOBAL && b < nb) {
            const double val = __dadd_rn(x, offset);
            const double val2 = __dadd_rn(val, final);
            if (out64) {
                out64[b + 1] = val;
                out64[nb + b + 1] = val2;
            }
            out32[b + 1] = split_pair(val);
            out32[nb + b + 1] = split_pair(val2);
        } else if (mode == SEG_IN_PLACE && b < nb) {
            r.store(b, __dadd_rn(x, offset));
        }
        offset = __dadd_rn(offset, wt);
        total = __dadd_rn(total, wt);
    }
    return total;
}

// The staged-by-threads fold of CTA `cta` (periods cta * G ..) of one fold.
__device__ __forceinline__ void fold_smem_cta(const FoldArgs& a, int cta) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ double s_scale[MAX_GROUP];

    const int tid = threadIdx.x;
    const int T = blockDim.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int nb = a.nb;
    const uint32_t unb = (uint32_t)nb;
    const double inv_nb = 1.0 / (double)nb;
    const int G = a.group;          // periods per CTA, a power of two
    const int wpp = (T / 32) / G;   // warps per period (>= 1)
    const int NS = wpp * 32;        // segments per period
    const int g0 = cta * G;
    const int g = min(G, a.periods - g0);
    const int q = warp / wpp;
    const int seg = (warp - q * wpp) * 32 + lane;
    const int rs = a.row_stride;    // >= nb

    // Shared memory: staging (t, v, w) triples [stage_field] | run starts [G][NS + 1]
    // (padded to 16 bytes) | sums v, w [G][rs] | counts [G][rs]; the sums
    // and counts live in global scratch instead when hist_global is set.
    double* st = reinterpret_cast<double*>(smem);
    int* starts = reinterpret_cast<int*>(st + 3 * (size_t)a.stage_field);
    const size_t starts_bytes = ((size_t)G * (NS + 1) * sizeof(int) + 15) & ~(size_t)15;
    double* hv = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(starts) + starts_bytes);
    double* hw = hv + (size_t)G * rs;
    uint32_t* hc = reinterpret_cast<uint32_t*>(hw + (size_t)G * rs);
    if (a.hist_global) {
        hv = a.hist_global + (size_t)cta * G * rs * 3;
        hw = hv + (size_t)G * rs;
        hc = reinterpret_cast<uint32_t*>(hw + (size_t)G * rs);
    }

    if (tid < g) s_scale[tid] = a.scales[g0 + tid];
    for (int e = tid; e < G * rs; e += T) {
        hv[e] = 0.0;
        hw[e] = 0.0;
        hc[e] = 0u;
    }
    __syncthreads();
    const bool live = q < g;
    const double scale = live ? s_scale[q] : 0.0;
    double* lv = hv + (size_t)q * rs;
    double* lw = hw + (size_t)q * rs;
    uint32_t* lc = hc + (size_t)q * rs;
    int* lstart = starts + q * (NS + 1);

    for (int c = 0; c < a.nchunks; c++) {
        const int i0 = a.chunks[c];
        const int len = a.chunks[c + 1] - i0;
        // Segment length, odd so that the lanes' (t, v, w) triples fall in
        // different shared-memory banks.
        const int R = ((len + NS - 1) / NS) | 1;
        // Stage the chunk: observation k at st[3k .. 3k + 2] = (t, v, w).
        for (int k = tid; k < len; k += T) {
            st[3 * k] = a.time[i0 + k];
            st[3 * k + 1] = a.v[i0 + k];
            st[3 * k + 2] = a.w[i0 + k];
        }
        __syncthreads();

        // Aligned start: the first run start of this period at or after seg * R.
        int k = seg * R;
        if (live && k < len && k > 0) {
            uint32_t prev = cell_of(st[3 * (k - 1)], scale);
            while (k < len) {
                const uint32_t v = cell_of(st[3 * k], scale);
                if (v != prev) break;
                prev = v;
                ++k;
            }
        }
        if (k > len) k = len;
        if (live) lstart[seg] = k;
        if (live && seg == 0) lstart[NS] = len;
        __syncthreads();
        const int end = live ? lstart[seg + 1] : 0;

        if (live && k < end) {
            const double* p = st + 3 * k;
            uint32_t v = cell_of(p[0], scale);
            double nextb = (double)v + 1.0;
            uint32_t slot = mod_nb(v, unb, inv_nb);
            double av = lv[slot], aw = lw[slot];
            uint32_t c0 = lc[slot];
            int k0 = k;
            while (k < end) {
                av = __dadd_rn(av, p[1]);
                aw = __dadd_rn(aw, p[2]);
                p += 3;
                ++k;
                // p[0] is staged or spare slack when k == end; it is unused then.
                const double x = __dmul_rn(p[0], scale);
                if (k == end || x >= nextb) {
                    lv[slot] = av;
                    lw[slot] = aw;
                    lc[slot] = c0 + (uint32_t)(k - k0);
                    if (k < end) {
                        const double after = __dadd_rn(nextb, 1.0);
                        if (x < after) {  // the next cell
                            nextb = after;
                            slot = slot + 1 == unb ? 0u : slot + 1;
                        } else {  // empty cells in between
                            const uint32_t vn = (uint32_t)floor(x);
                            nextb = (double)vn + 1.0;
                            slot = mod_nb(vn, unb, inv_nb);
                        }
                        av = lv[slot];
                        aw = lw[slot];
                        c0 = lc[slot];
                        k0 = k;
                    }
                }
            }
        }
        __syncthreads();
    }

    if (a.hist_out) {
        // Raw histograms, field-major [3][nb] (the evidence fold, one period).
        for (int p = tid; p < nb; p += T) {
            a.hist_out[p] = hv[p];
            a.hist_out[nb + p] = hw[p];
            a.hist_out[2 * (size_t)nb + p] = (double)hc[p];
        }
        return;
    }
    const size_t stride = 2 * (size_t)nb + 1;
    for (int row = warp; row < g * NF; row += T / 32) {
        const int qq = row / NF, f = row - (row / NF) * NF;
        double* out64 = a.cum + ((size_t)(g0 + qq) * NF + f) * stride;
        float2* out32 = a.cum32 + ((size_t)(g0 + qq) * NF + f) * stride;
        const size_t off = (size_t)qq * rs;
        if (f == F_V)
            prefix_row([&](int bb) { return hv[off + bb]; }, nb, out64, out32);
        else if (f == F_W)
            prefix_row([&](int bb) { return hw[off + bb]; }, nb, out64, out32);
        else
            prefix_row([&](int bb) { return (double)hc[off + bb]; }, nb, out64, out32);
    }
}

__global__ void __launch_bounds__(1024, 1) k_fold(FoldArgs a) { fold_smem_cta(a, blockIdx.x); }

// Many staged-by-threads folds in one launch: CTA c runs CTA c - cta0[j] of
// job j, where cta0[j] <= c < cta0[j + 1] (every job with the same CTA size).
__global__ void __launch_bounds__(1024, 1) k_fold_jobs(const FoldArgs* __restrict__ jobs, const int* __restrict__ cta0,
                                                       int njobs) {
    int lo = 0, hi = njobs - 1;
    const int c = blockIdx.x;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (cta0[mid] <= c)
            lo = mid;
        else
            hi = mid - 1;
    }
    fold_smem_cta(jobs[lo], c - cta0[lo]);
}

// ---------------------------------------------------------------------------
// TMA staging: mbarrier helpers and the bulk copies of one chunk.

namespace {

// Issues the three bulk copies of chunk [i0, i1), rounded out to whole
// 16-byte pieces, into one staging buffer (fields at `field` doubles apart).
__device__ __forceinline__ void stage_chunk(const FoldArgs& a, int i0, int i1, double* buf, int field, uint32_t bar) {
    const int a0 = i0 & ~1, a1 = (i1 + 1) & ~1;
    const uint32_t bytes = (uint32_t)(a1 - a0) * (uint32_t)sizeof(double);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(bar, 3u * bytes);
    bulk_load(smem_addr(buf), a.time + a0, bytes, bar);
    bulk_load(smem_addr(buf + field), a.v + a0, bytes, bar);
    bulk_load(smem_addr(buf + 2 * field), a.w + a0, bytes, bar);
}

}  // namespace


// ---------------------------------------------------------------------------
// Walking fold with TMA-staged chunks (the fold of every nb whose
// histograms fit shared memory beside the staging).
//
// As in k_fold, each period's lanes split a staged chunk into segments whose
// starts are moved to run boundaries, and each lane walks its runs in order,
// keeping the current run's sums in registers. The bin of a cell is
// cell - base (one wrap at most), base fixed per segment, so a cell change
// costs a compare, a subtraction and the store/load of the bin's sums.
// Chunks are staged by TMA bulk copies into two buffers (fields t, v, w),
// one chunk ahead of the one being folded, so the copy overlaps the walk.

// Segments at least this long are walked in lockstep (measured: shorter ones
// lose more to idle steps than the conflict-free reads gain).
constexpr int LOCKSTEP_MIN_SEGMENT = 11;

// The first observation of a lane's window in a chunk: its segment's start
// seg * R moved forward to the period's next cell boundary (so every run
// belongs to exactly one lane), at most len.
__device__ __forceinline__ int window_start(const double* tt, int len, int R, int seg, double scale) {
    int k = seg * R;
    if (k < len && k > 0) {
        const uint32_t prev = cell_of(tt[k - 1], scale);
        while (k < len) {
            if (cell_of(tt[k], scale) != prev) break;
            ++k;
        }
    }
    return k > len ? len : k;
}

// Short segments: one lane walks its window [k, end) of one period, loading
// a bin's sums when its run starts and storing them when it ends; a run's
// count goes to its bin by one shared-memory atomic add (no load).
__device__ __forceinline__ void walk_window(const double* tt, int F, int k, int end, double scale, uint32_t unb,
                                            double inv_nb, double2* lvw, uint32_t* lc) {
    uint32_t cur = cell_of(tt[k], scale);
    const uint32_t s0 = mod_nb(cur, unb, inv_nb);
    const uint32_t base = cur - s0;
    uint32_t slot = s0;
    double2 acc = lvw[slot];
    uint32_t cnt = 0;
    for (int j = k; j < end; j++) {
        const uint32_t cj = cell_of(tt[j], scale);
        if (cj != cur) {
            lvw[slot] = acc;
            atomicAdd(&lc[slot], cnt);
            cnt = 0;
            const uint32_t b = cj - base;
            slot = b >= unb ? b - unb : b;
            cur = cj;
            acc = lvw[slot];
        }
        acc.x = __dadd_rn(acc.x, tt[j + F]);
        acc.y = __dadd_rn(acc.y, tt[j + 2 * F]);
        cnt += 1u;
    }
    lvw[slot] = acc;
    atomicAdd(&lc[slot], cnt);
}

// A lane's run state for one period in the lockstep walk: the current
// cell's sums, and the next cell's bin prefetched at each cell change.
struct RunWalker {
    double2* lvw;
    uint32_t* lc;
    uint32_t cur, base, slot, nslot, cnt;
    double2 acc, pre;
    __device__ __forceinline__ void open(double t, double scale, uint32_t unb, double inv_nb) {
        cur = cell_of(t, scale);
        const uint32_t s0 = mod_nb(cur, unb, inv_nb);
        base = cur - s0;  // bin = cell - base (- nb past the wrap)
        slot = s0;
        nslot = s0 + 1u == unb ? 0u : s0 + 1u;
        acc = lvw[slot];
        pre = lvw[nslot];
        cnt = 0;
    }
    __device__ __forceinline__ void add(double t, double v, double w, double scale, uint32_t unb) {
        const uint32_t cj = cell_of(t, scale);
        if (cj != cur) {
            lvw[slot] = acc;
            atomicAdd(&lc[slot], cnt);
            cnt = 0;
            if (cj == cur + 1u) {
                acc = pre;
                slot = nslot;
            } else {  // empty cells skipped
                const uint32_t b = cj - base;
                slot = b >= unb ? b - unb : b;
                acc = lvw[slot];
            }
            cur = cj;
            nslot = slot + 1u == unb ? 0u : slot + 1u;
            pre = lvw[nslot];
        }
        acc.x = __dadd_rn(acc.x, v);
        acc.y = __dadd_rn(acc.y, w);
        cnt += 1u;
    }
    __device__ __forceinline__ void close() {
        lvw[slot] = acc;
        atomicAdd(&lc[slot], cnt);
    }
};

// The coarse-map epilogue of the walking fold (after the in-place prefix rows
// and a barrier), out of line: it runs once per CTA.
__device__ __noinline__ void fold_map_epilogue(float* map_out, const double* map_durations, const double* map_rho,
                                               int nd, double baseline, int n, const double2* hvw,
                                               const uint32_t* hc, const double* s_scale, const double* row_final,
                                               double* part, int nb, int rs, int g, int g0, int W) {
    // Coarse-map epilogue: for every (period, map duration) pair the best box
    // score over all phases from the in-place prefix rows, exactly as
    // k_box_map computes it from the global rows (the doubled row's entry i
    // is 0 at i = 0, the kept value of bin i - 1 up to nb, and that of bin
    // i - nb - 1 plus the row's final carry beyond). Pairs get W / pairs warps
    // each (or one warp takes several pairs); partial maxima meet in shared
    // memory.
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t unb = (uint32_t)nb;
    const int pairs = g * nd;
    const int per = pairs >= W ? 1 : W / pairs;
    const uint32_t half = unb / 2u;
    auto pre = [&](const HistRow& r, double carry, uint32_t i) -> double {
        return i == 0 ? 0.0 : (i <= unb ? r.load((int)i - 1) : __dadd_rn(r.load((int)(i - unb) - 1), carry));
    };
    for (int p = warp / per; p < pairs && warp < per * pairs; p += (pairs >= W ? W : pairs)) {
        const int qq = p / nd, d = p - qq * nd;
        const int slice = warp - (warp / per) * per;
        const double sc = s_scale[qq];
        const uint32_t raw = template_width(map_durations[d], sc);
        double best = 0.0;
        if (raw < half) {
            const uint32_t k = raw;
            const size_t o = (size_t)qq * rs;
            HistRow rv, rw, rn;
            double2* hv = const_cast<double2*>(hvw);
            uint32_t* hcc = const_cast<uint32_t*>(hc);
            rv.d = &hv[o].x;
            rv.c = hcc + o;
            rw.d = &hv[o].y;
            rw.c = hcc + o;
            rn.d = nullptr;
            rn.c = hcc + o;
            const double cv = row_final[qq * NF + F_V], cw = row_final[qq * NF + F_W],
                         cn = row_final[qq * NF + F_N];
            for (uint32_t j = (uint32_t)(slice * 32 + lane); j < unb; j += (uint32_t)(per * 32)) {
                const double count = __dsub_rn(pre(rn, cn, j + k), pre(rn, cn, j));
                if (!(count >= 3.0 && count <= (double)n - 3.0)) continue;
                const double av = __dsub_rn(pre(rv, cv, j + k), pre(rv, cv, j));
                if (!(av > 0.0)) continue;
                const double w = __dsub_rn(pre(rw, cw, j + k), pre(rw, cw, j));
                const double q = __dsub_rn(w, __ddiv_rn(__dmul_rn(w, w), baseline));
                if (!(q > 0.0)) continue;
                const double s = __ddiv_rn(__ddiv_rn(av, map_rho[d]), __dsqrt_rn(rmax(q, 1e-300)));
                if (s > best) best = s;
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, off));
        if (per == 1) {
            if (lane == 0) map_out[(size_t)(g0 + qq) * nd + d] = (float)best;
        } else if (lane == 0) {
            part[warp] = best;
        }
    }
    if (per > 1) {
        __syncthreads();
        if (tid < pairs) {
            double best = part[tid * per];
            for (int k = 1; k < per; k++) best = fmax(best, part[tid * per + k]);
            const int qq = tid / nd, d = tid - qq * nd;
            map_out[(size_t)(g0 + qq) * nd + d] = (float)best;
        }
    }
}


// Shared memory of the fused scan's tile winners: PART_STRIDE doubles, the
// key and the flags (in a double's slot) per (period, tile) of the CTA.
constexpr int FUSED_PART_DOUBLES = PART_STRIDE + 2;

// The fused tile scan and merge of a walking-fold CTA (after the in-place
// prefix rows and a barrier), out of line like the map epilogue, so the
// fold's loop keeps its registers: groups of TILE threads take the (period,
// tile) units of the CTA's periods in turn and scan them from the in-place
// rows, each group with its own scratch, into `parts`; then one thread per
// period merges its tiles into the records.
__device__ __noinline__ void fold_scan_epilogue(const ScanArgs& scan, const MergeArgs& merge, const double2* hvw,
                                                const uint32_t* hc, const double* row_final, const double* s_scale,
                                                TileScratch* scratch, double* parts, int nb, int rs, int g, int g0) {
    const int tiles = (nb + TILE - 1) / TILE;
    const int ngroups = (int)blockDim.x / TILE;
    const int gi = (int)threadIdx.x / TILE;
    const NamedGroup grp{1u + (uint32_t)gi, gi * TILE};
    for (int u = gi; u < g * tiles; u += ngroups) {
        const int qq = u / tiles, t = u - qq * tiles;
        SmemRows rows;
        rows.vw = hvw + (size_t)qq * rs;
        rows.c = hc + (size_t)qq * rs;
        rows.fin = row_final + qq * NF;
        rows.nb = (uint32_t)nb;
        double* slot = parts + (size_t)u * FUSED_PART_DOUBLES;
        grp.sync();  // the group's scratch is free: its previous unit is done with it
        scan_tile(scan, rows, grp, scratch[gi], t, s_scale[qq], slot, reinterpret_cast<uint64_t*>(slot + PART_STRIDE),
                  reinterpret_cast<uint32_t*>(slot + PART_STRIDE + 1));
    }
    __syncthreads();
    for (int qq = (int)threadIdx.x; qq < g; qq += (int)blockDim.x) {
        // The unit of tile t of period qq is qq * tiles + t: its tiles' slots
        // follow one another at FUSED_PART_DOUBLES doubles.
        const double* p0 = parts + (size_t)qq * tiles * FUSED_PART_DOUBLES;
        double best = neg_inf();
        uint64_t key = KEY_MAX;
        int chosen = 0;
        uint32_t fl = 0;
        for (int t = 0; t < tiles; t++) {
            const double* sl = p0 + (size_t)t * FUSED_PART_DOUBLES;
            const double v = sl[7];
            const uint64_t k = *reinterpret_cast<const uint64_t*>(sl + PART_STRIDE);
            fl |= *reinterpret_cast<const uint32_t*>(sl + PART_STRIDE + 1);
            if (v > best || (v == best && k < key)) {
                best = v;
                key = k;
                chosen = t;
            }
        }
        merge_record(merge, g0 + qq, p0 + (size_t)chosen * FUSED_PART_DOUBLES, best, fl);
    }
}

// One CTA of the walking fold: CTA `cta` of the launch described by `a`
// folds periods [cta * G, cta * G + G). `reuse`: this CTA ran an earlier
// fold (a persistent CTA), whose barriers are invalidated before the new
// ones. Returns false (uniformly over the CTA) when a staging wait gave up.
template <int CAP, bool PAIR>
__device__ __forceinline__ bool fold_walk_cta(const FoldArgs& a, const int cta, const bool reuse,
                                              const ScanArgs* scan, const MergeArgs* merge) {
    constexpr int F = CAP + 2;  // doubles per staged field
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ double s_scale[WALK_MAX_GROUP];
    __shared__ __align__(8) uint64_t s_bar[2];

    const int tid = threadIdx.x;
    const int T = blockDim.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int nb = a.nb;
    const uint32_t unb = (uint32_t)nb;
    const double inv_nb = 1.0 / (double)nb;
    const int G = a.group;
    // Paired walk: each lane walks two periods, q and q + G / 2, over the
    // same staged observations (one read of t, v, w serves both).
    // A lane set is WALK_MIN_LANES or more consecutive lanes: part of a warp
    // (several periods per warp, for short chunks), a warp, or several warps.
    const int GV = PAIR ? G / 2 : G;  // lane sets
    const int NS = T / GV;            // lanes per lane set = segments per period
    const int wpp = NS / 32;          // whole warps per lane set (0: a warp holds several sets)
    const int g0 = cta * G;
    const int g = min(G, a.periods - g0);
    const int q = tid / NS;
    const int seg = tid - q * NS;
    const bool live = q < g;
    const bool live_b = PAIR && q + GV < g;
    const int rs = a.row_stride;

    // Shared memory: staging [2][t | v | w][F] | run starts [G][NS + 1]
    // (padded to 16 bytes) | sums (v, w) [G][rs] | counts [G][rs].
    double* stage = reinterpret_cast<double*>(smem);
    int* starts = reinterpret_cast<int*>(stage + 6 * F);
    const size_t starts_bytes = ((size_t)G * (NS + 1) * sizeof(int) + 15) & ~(size_t)15;
    double2* hvw = reinterpret_cast<double2*>(reinterpret_cast<unsigned char*>(starts) + starts_bytes);
    uint32_t* hc = reinterpret_cast<uint32_t*>(hvw + (size_t)G * rs);

    if (tid < g) s_scale[tid] = a.scales[g0 + tid];
    for (int e = tid; e < G * rs; e += T) {
        hvw[e] = make_double2(0.0, 0.0);
        hc[e] = 0u;
    }
    const uint32_t bar0 = smem_addr(&s_bar[0]);
    if (tid == 0) {
        if (reuse) {  // a persistent CTA's earlier fold left its barriers valid (every phase completed)
            mbar_inval(bar0);
            mbar_inval(bar0 + 8);
        }
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const double scale = live ? s_scale[q] : 0.0;
    double2* lvw = hvw + (size_t)(live ? q : 0) * rs;
    uint32_t* lc = hc + (size_t)(live ? q : 0) * rs;
    int* lstart = starts + (live ? q : 0) * (NS + 1);
    const int qb = live_b ? q + GV : 0;
    const double scale_b = live_b ? s_scale[qb] : 0.0;
    double2* lvw_b = hvw + (size_t)qb * rs;
    uint32_t* lc_b = hc + (size_t)qb * rs;
    int* lstart_b = starts + qb * (NS + 1);
    const float inv_ns = 1.0f / (float)NS;
    const int lmin = a.lockstep_min > 0 ? a.lockstep_min : LOCKSTEP_MIN_SEGMENT;
    const int nch = a.nchunks;
    // Staging blocks: runs of consecutive chunks of at most CAP observations
    // in all, one bulk copy per field. Between the chunks of a block only the
    // warps of a period group synchronise (named barrier 1 + warp / U over U
    // warps, U >= a lane set's wpp warps and a whole number of lane sets, at
    // most 8 groups): periods share no bins, so a CTA-wide barrier is needed
    // only when a staging buffer turns over.
    const int* ch = a.chunks;
    auto block_end = [&](int c0) {
        int c1 = c0 + 1;
        while (c1 < nch && ch[c1 + 1] - ch[c0] <= CAP) c1++;
        return c1;
    };
    const int U = wpp > 4 ? wpp : 4;
    const uint32_t gbar = 1u + (uint32_t)(warp / U), gthreads = 32u * (uint32_t)U;
    int blk_lo = 0, blk_hi = block_end(0);  // chunks of the block being folded
    if (tid == 0) stage_chunk(a, ch[0], ch[blk_hi], stage, F, bar0);

    for (int blk = 0; blk_lo < nch; blk++) {
        const int buf = blk & 1;
        const bool landed = mbar_wait_bounded(bar0 + 8 * buf, (uint32_t)(blk >> 1) & 1u);
        if (!__syncthreads_and(landed)) {
            // Give up on this fold, but not while the block's bulk copies may
            // still write into this CTA's shared memory: thread 0 (which
            // issued them; the next block's copies are not issued yet) waits
            // again with a longer bound. If that also runs out the copies may
            // still be pending when the CTA ends; the fault word is set either
            // way and the host discards the pass.
            if (tid == 0) {
                for (int again = 0; again < 16; again++)
                    if (mbar_wait_bounded(bar0 + 8 * buf, (uint32_t)(blk >> 1) & 1u)) break;
                atomicOr(a.fault, 1u);
            }
            return false;
        }
        const int next_lo = blk_hi, next_hi = next_lo < nch ? block_end(next_lo) : next_lo;
        if (tid == 0 && next_lo < nch)
            stage_chunk(a, ch[next_lo], ch[next_hi], stage + 3 * F * (buf ^ 1), F, bar0 + 8 * (buf ^ 1));
        const int base_i = ch[blk_lo];
        const double* sb = stage + 3 * F * buf + (base_i & 1);  // staged slot of observation i: sb[i - base_i]
        for (int c = blk_lo; c < blk_hi; c++) {
        const int i0 = ch[c];
        const int len = ch[c + 1] - i0;
        const double* tt = sb + (i0 - base_i);
        // Segment length: at least ceil(len / NS), odd.
        const int R = ((int)((float)len * inv_ns) + 1) | 1;
        const int k = live ? window_start(tt, len, R, seg, scale) : 0;
        int kb = 0;
        if constexpr (PAIR) kb = live_b ? window_start(tt, len, R, seg, scale_b) : 0;
        if (live) {
            lstart[seg] = k;
            if (seg == 0) lstart[NS] = len;
        }
        if constexpr (PAIR) {
            if (live_b) {
                lstart_b[seg] = kb;
                if (seg == 0) lstart_b[NS] = len;
            }
        }
        group_sync(gbar, gthreads);
        const int end = live ? lstart[seg + 1] : 0;
        int end_b = 0;
        if constexpr (PAIR) end_b = live_b ? lstart_b[seg + 1] : 0;
        if (R < lmin) {
            // Short segments: each lane walks its own window(s).
            if (live && k < end) walk_window(tt, F, k, end, scale, unb, inv_nb, lvw, lc);
            if constexpr (PAIR)
                if (live_b && kb < end_b) walk_window(tt, F, kb, end_b, scale_b, unb, inv_nb, lvw_b, lc_b);
        } else {
        // Lockstep walk: at step i every lane whose window [k, end) holds
        // observation seg * R + i reads and folds it (R odd, so the lanes'
        // reads fall in distinct banks). Entering a cell takes the bin's sums
        // prefetched at the previous cell change (the next cell's bin), and
        // prefetches the bin after it. Counts are integers, so a run's count
        // is added to its bin with one shared-memory atomic add when the run
        // ends (no load of the bin's count). A paired lane folds each read
        // observation into both its periods' windows that hold it.
        const int b0 = seg * R;
        const bool has = live && k < end;
        if constexpr (!PAIR) {
            const int steps = __reduce_max_sync(0xffffffffu, has ? end - b0 : 0);
            if (steps > 0) {
                RunWalker wa;
                wa.lvw = lvw;
                wa.lc = lc;
                if (has) wa.open(tt[k], scale, unb, inv_nb);
                for (int i = 0; i < steps; i++) {
                    const int o = b0 + i;
                    // Only the lanes whose windows hold o read it, so a step's
                    // reads take fewer wavefronts as lanes run out of window.
                    if (o >= k && o < end) wa.add(tt[o], tt[o + F], tt[o + 2 * F], scale, unb);
                }
                if (has) wa.close();
            }
        } else {
            const bool has_b = live_b && kb < end_b;
            const int steps =
                __reduce_max_sync(0xffffffffu, max(has ? end - b0 : 0, has_b ? end_b - b0 : 0));
            if (steps > 0) {
                RunWalker wa, wb;
                wa.lvw = lvw;
                wa.lc = lc;
                wb.lvw = lvw_b;
                wb.lc = lc_b;
                if (has) wa.open(tt[k], scale, unb, inv_nb);
                if (has_b) wb.open(tt[kb], scale_b, unb, inv_nb);
                for (int i = 0; i < steps; i++) {
                    const int o = b0 + i;
                    const bool in = o >= k && o < end;
                    const bool in_b = o >= kb && o < end_b;
                    if (in || in_b) {
                        const double tj = tt[o], vj = tt[o + F], wj = tt[o + 2 * F];
                        if (in) wa.add(tj, vj, wj, scale, unb);
                        if (in_b) wb.add(tj, vj, wj, scale_b, unb);
                    }
                }
                if (has) wa.close();
                if (has_b) wb.close();
            }
        }
        }
        group_sync(gbar, gthreads);  // the chunk's bins are written before the next chunk's walk
        }
        blk_lo = next_lo;
        blk_hi = next_hi;
    }
    __syncthreads();

    if (a.hist_out) {
        for (int p = tid; p < nb; p += T) {
            a.hist_out[p] = hvw[p].x;
            a.hist_out[nb + p] = hvw[p].y;
            a.hist_out[2 * (size_t)nb + p] = (double)hc[p];
        }
        return true;
    }
    // Doubled prefix rows. A row has S segments of 256 bins whose carries
    // chain; with few rows (large nb, small G) the rows' segments are spread
    // over every warp in three passes (segment totals, the carry chains, then
    // the values with their carries known), else one warp takes a whole row.
    // Both give prefix_row's values bit for bit.
    const size_t stride = 2 * (size_t)nb + 1;
    const int W = T / 32;
    const int rows = g * NF;
    const int S = (nb + 255) >> 8;
    const bool map = a.map_out != nullptr;
    const bool in_place = map || scan != nullptr;  // the rows stay in shared memory
    auto row_of = [&](int row, double*& out64, float2*& out32) {
        const int qq = row / NF, f = row - qq * NF;
        out64 = (a.rows32_only || in_place) ? nullptr : a.cum + ((size_t)(g0 + qq) * NF + f) * stride;
        out32 = in_place ? nullptr : a.cum32 + ((size_t)(g0 + qq) * NF + f) * stride;
        const size_t o = (size_t)qq * rs;
        HistRow r;
        r.d = f == F_V ? &hvw[o].x : f == F_W ? &hvw[o].y : nullptr;
        r.c = hc + o;
        return r;
    };
    const int items = rows * S;
    double* row_final = stage;  // rows: each row's final carry (map epilogue, fused scan)
    // The tail of the staging buffers is kept for the epilogue: the map's
    // per-warp partial maxima, or the fused scan's per-group scratch.
    // Fused scan: the groups' scratch, below it the tile winners.
    const int ngroups = T / TILE;
    const int scratch_doubles = scan ? ngroups * (int)((sizeof(TileScratch) + 7) / 8) : W;
    const int reserve = scratch_doubles + (scan ? G * ((nb + TILE - 1) / TILE) * FUSED_PART_DOUBLES : 0);
    if (2 * ((items + W - 1) / W) < ((rows + W - 1) / W) * S && 2 * items + rows + reserve <= 6 * F) {
        double* seg_total = stage;             // rows x S (the staging buffers are idle now)
        double* seg_carry = stage + items;     // rows x S
        row_final = stage + 2 * items;         // rows
        for (int it = warp; it < items; it += W) {
            const int row = it / S, sg = it - row * S;
            double* o64;
            float2* o32;
            const HistRow r = row_of(row, o64, o32);
            const double tot = prefix_segment(r, nb, sg * 256, 0.0, 0.0, SEG_TOTAL, o64, o32);
            if (lane == 0) seg_total[it] = tot;
        }
        __syncthreads();
        for (int row = tid; row < rows; row += T) {
            double carry = 0.0;
            for (int sg = 0; sg < S; sg++) {
                seg_carry[row * S + sg] = carry;
                carry = __dadd_rn(carry, seg_total[row * S + sg]);
            }
            row_final[row] = carry;
        }
        __syncthreads();
        for (int it = warp; it < items; it += W) {
            const int row = it / S, sg = it - row * S;
            double* o64;
            float2* o32;
            const HistRow r = row_of(row, o64, o32);
            if (!in_place && sg == 0 && lane == 0) {
                if (o64) o64[0] = 0.0;
                o32[0] = make_float2(0.f, 0.f);
            }
            prefix_segment(r, nb, sg * 256, seg_carry[it], row_final[row], in_place ? SEG_IN_PLACE : SEG_GLOBAL, o64,
                           o32);
        }
    } else {
        for (int row = warp; row < rows; row += W) {
            double* o64;
            float2* o32;
            const HistRow r = row_of(row, o64, o32);
            const double carry = prefix_row_smem(r, nb, !in_place, o64, o32);
            if (in_place && lane == 0) row_final[row] = carry;
        }
    }
    if (!in_place) return true;

    __syncthreads();
    if (scan) {
        fold_scan_epilogue(*scan, *merge, hvw, hc, row_final, s_scale,
                           reinterpret_cast<TileScratch*>(stage + 6 * F - scratch_doubles),
                           stage + 6 * F - reserve, nb, rs, g, g0);
        return true;
    }
    fold_map_epilogue(a.map_out, a.map_durations, a.map_rho, a.map_nd, a.map_baseline, a.n, hvw, hc, s_scale,
                      row_final, stage + 6 * F - W, nb, rs, g, g0, W);
    return true;
}

// The kernels come in two forms: one period per lane (CTAs of up to 1024
// threads, 64 registers) and the paired walk (two periods per lane, CTAs of
// up to 512 threads, 128 registers).
template <int CAP, bool PAIR>
__global__ void __launch_bounds__(PAIR ? 512 : 1024, 1) k_fold_walk(FoldArgs a) {
    fold_walk_cta<CAP, PAIR>(a, blockIdx.x, false, nullptr, nullptr);
}

// The walking fold with the tile scan and merge fused (launch_fold_scan).
template <int CAP, bool PAIR>
__global__ void __launch_bounds__(PAIR ? 512 : 1024, 1) k_fold_scan(FoldArgs a, const __grid_constant__ ScanArgs s,
                                                                    const __grid_constant__ MergeArgs m) {
    fold_walk_cta<CAP, PAIR>(a, blockIdx.x, false, &s, &m);
}

// Many folds in one launch (the batched search): CTA c runs CTA
// c - cta0[j] of job j, where cta0[j] <= c < cta0[j + 1]. Every job uses the
// walking fold with TMA staging; the launch's shared memory is the largest
// job's.
template <int CAP, bool PAIR>
__global__ void __launch_bounds__(PAIR ? 512 : 1024, 1) k_fold_walk_jobs(const FoldArgs* __restrict__ jobs,
                                                                         const int* __restrict__ cta0, int njobs) {
    int lo = 0, hi = njobs - 1;
    const int c = blockIdx.x;
    while (lo < hi) {  // last job with cta0[j] <= c
        const int mid = (lo + hi + 1) / 2;
        if (cta0[mid] <= c)
            lo = mid;
        else
            hi = mid - 1;
    }
    fold_walk_cta<CAP, PAIR>(jobs[lo], c - cta0[lo], false, jobs[lo].scan, jobs[lo].merge);
}

// One unit of the persistent grid, out of line so the fold's registers are
// allocated as in a CTA per unit rather than around the grid's unit loop.
template <int CAP, bool PAIR>
__device__ __noinline__ bool fold_walk_unit(const FoldArgs& a, int cta, bool reuse) {
    return fold_walk_cta<CAP, PAIR>(a, cta, reuse, a.scan, a.merge);
}

// The same jobs as k_fold_walk_jobs, by a persistent grid (one CTA per SM)
// that steals work: each CTA takes the next unit (one walking-fold CTA's
// periods of one job) from a global counter until none is left. A CTA whose
// staging wait gave up stops taking units (its copies may still be pending).
template <int CAP, bool PAIR>
__global__ void __launch_bounds__(PAIR ? 512 : 1024, 1) k_fold_walk_steal(const FoldArgs* __restrict__ jobs,
                                                                          const int* __restrict__ cta0, int njobs,
                                                                          int units, unsigned int* __restrict__ next) {
    __shared__ int s_unit;
    for (bool reuse = false;; reuse = true) {
        if (threadIdx.x == 0) s_unit = (int)atomicAdd(next, 1u);
        __syncthreads();
        const int u = s_unit;
        __syncthreads();  // every thread has read s_unit before it is taken again
        if (u >= units) return;
        int lo = 0, hi = njobs - 1;
        while (lo < hi) {  // last job with cta0[j] <= u
            const int mid = (lo + hi + 1) / 2;
            if (cta0[mid] <= u)
                lo = mid;
            else
                hi = mid - 1;
        }
        if (!fold_walk_unit<CAP, PAIR>(jobs[lo], u - cta0[lo], reuse)) return;
        __syncthreads();  // the unit's shared memory is free before the next one
    }
}

namespace {
constexpr size_t BIN_BYTES = 2 * sizeof(double) + sizeof(uint32_t);
constexpr size_t SLOT_BYTES = 3 * sizeof(double);
constexpr int STAGE_MAX = 4096;
constexpr int WALK_CAP = 2048;

// Walking-fold shape: chunks of up to WALK_CAP observations, the largest
// power-of-two group whose histograms fit beside the staging, 1024 threads.
// Tuning (process-wide, set by fbls_set_tuning from a measured table), per nb
// class floor(log2(nb)): the largest period group (0 = the built-in rule),
// and for the callers that ask for it the paired walk (two periods per lane,
// CTAs of at most 512 threads, groups of at least 2), the CTA size (a power of
// two from 128 to 1024, 0 = 1024, or 512 paired; a CTA has at least one warp
// per lane set) and the lockstep threshold (0 = built-in).
std::atomic<uint32_t> g_group_cap[32];
std::atomic<uint32_t> g_threads[32];
std::atomic<uint32_t> g_lockstep[32];
std::atomic<uint32_t> g_pair[32];
std::atomic<uint32_t> g_launch_periods{16384};
std::atomic<uint32_t> g_fold_steal{0};
std::atomic<uint32_t> g_fused_scan{0};
std::atomic<uint32_t> g_map_lockstep{0};
std::atomic<uint32_t> g_map_threads{0};
std::atomic<uint32_t> g_map_group{0};
std::atomic<uint32_t> g_batch_no_fill{0};

int nb_class(int nb) { return nb > 0 ? 31 - __builtin_clz((unsigned)nb) : 0; }

uint32_t group_cap(int nb) { return g_group_cap[nb_class(nb)].load(std::memory_order_relaxed); }

bool walk_threads_ok(int t) { return t == 128 || t == 256 || t == 512 || t == 1024; }

// The walking-fold shape for CTAs of T threads, `pair` (two periods per
// lane), a group cap (0: the rule's MAX_GROUP; a tuned cap may reach
// WALK_MAX_GROUP, with lane sets down to WALK_MIN_LANES lanes) and a lockstep
// threshold. Groups are cut until the fold has at least `fill_ctas` CTAs
// (0: only to the periods there are, for callers whose launch holds many
// such jobs). False when one lane set's histograms do not fit.
bool walk_shape_for(int nb, int periods, int T, bool pair, uint32_t gcap, int lockstep, int fill_ctas,
                    FoldShape* out) {
    FoldShape s{};
    s.kind = FOLD_WALK;
    s.threads = T;
    s.pair = pair;
    s.lockstep_min = lockstep;
    const int PV = pair ? 2 : 1;  // periods per lane
    s.row_stride = nb | 1;
    const size_t stage = 6 * sizeof(double) * (size_t)(WALK_CAP + 2);
    const size_t hist_per = (size_t)s.row_stride * BIN_BYTES;
    // run starts [g][NS + 1], NS = the lanes of a lane set (g / PV sets)
    auto lanes = [&](int g) { return T / (g / PV > 0 ? g / PV : 1); };
    auto starts = [&](int g) { return ((size_t)g * (lanes(g) + 1) * sizeof(int) + 15) & ~(size_t)15; };
    if (stage + starts(PV) + (size_t)PV * hist_per > MAX_FOLD_SMEM) return false;
    const int gmax = gcap > (uint32_t)MAX_GROUP ? (int)std::min<uint32_t>(gcap, WALK_MAX_GROUP) : MAX_GROUP;
    int g = PV;
    while (2 * g <= gmax && lanes(2 * g) >= WALK_MIN_LANES &&
           stage + starts(2 * g) + (size_t)(2 * g) * hist_per <= MAX_FOLD_SMEM)
        g *= 2;
    while (g > PV && (g / 2 >= periods || (periods + g - 1) / g < fill_ctas)) g /= 2;
    while (gcap && g > PV && (uint32_t)g > gcap) g /= 2;
    s.group = g;
    s.hist_in_smem = true;
    s.window = 0;
    s.span_cap = nb;
    s.chunk_cap = WALK_CAP;
    s.stage_field = WALK_CAP + 2;
    s.smem = stage + starts(g) + (size_t)g * hist_per;
    *out = s;
    return true;
}

bool walk_shape(int nb, int periods, bool tuned, int fill_ctas, FoldShape* out) {
    const int cls = nb_class(nb);
    int T = 1024, lockstep = 0;
    bool pair = false;
    if (tuned) {
        pair = periods >= 2 && g_pair[cls].load(std::memory_order_relaxed) != 0;
        const uint32_t t = g_threads[cls].load(std::memory_order_relaxed);
        if (t) T = (int)t;
        lockstep = (int)g_lockstep[cls].load(std::memory_order_relaxed);
    }
    const uint32_t gcap = group_cap(nb);
    if (pair && walk_shape_for(nb, periods, T > 512 ? 512 : T, true, gcap, lockstep, fill_ctas, out)) return true;
    return walk_shape_for(nb, periods, T, false, gcap, lockstep, fill_ctas, out);
}

}  // namespace

FoldShape fold_map_shape(int nb, int periods, int sm_count) {
    const uint32_t t = g_map_threads.load(std::memory_order_relaxed);
    const uint32_t gcap = g_map_group.load(std::memory_order_relaxed);
    FoldShape w;
    // A tuned cap drops the fill rule: a map batch's launch holds every
    // star's groups.
    if (walk_shape_for(nb, periods, t ? (int)t : 1024, false, gcap, (int)g_map_lockstep.load(std::memory_order_relaxed),
                       gcap == 0 ? sm_count : 0, &w))
        return w;
    return fold_group_shape(nb, periods, sm_count);
}

// Launch shape: the walking fold's (walk_shape) where one lane set's
// histograms fit beside its staging buffers; else k_fold's: the largest
// power-of-two period group (<= 32 and at most enough to give the fold
// fill_ctas CTAs) whose histograms leave room to stage at least 2048
// observations; the staging capacity is what is left (up to STAGE_MAX); the
// CTA has 1024 threads, or 512 when segments would otherwise be shorter than
// 16 observations. A single period whose histogram does not fit folds into
// global scratch.
FoldShape fold_group_shape(int nb, int periods, int sm_count, bool tuned, int fill_ctas) {
    if (fill_ctas < 0) fill_ctas = sm_count;
    FoldShape w;
    if (walk_shape(nb, periods, tuned, fill_ctas, &w)) return w;
    FoldShape s{};
    s.kind = FOLD_SMEM;
    s.row_stride = nb | 1;
    const size_t hist_per = (size_t)s.row_stride * BIN_BYTES;
    const size_t stage_min = SLOT_BYTES * (2048 + 1024) + 4 * (1024 + 32);
    int g = 1;
    while (g < MAX_GROUP && (size_t)(2 * g) * hist_per + stage_min <= MAX_FOLD_SMEM) g *= 2;
    const int fill = fill_ctas > 0 ? (periods + fill_ctas - 1) / fill_ctas : periods;
    while (g > 1 && g / 2 >= fill) g /= 2;
    const uint32_t gcap = group_cap(nb);
    while (gcap && g > 1 && (uint32_t)g > gcap) g /= 2;
    s.group = g;
    s.hist_in_smem = (size_t)g * hist_per + stage_min <= MAX_FOLD_SMEM;
    const size_t room = MAX_FOLD_SMEM - (s.hist_in_smem ? (size_t)g * hist_per : 0) - 4 * (1024 + 32);
    int cap = (int)(room / SLOT_BYTES) - 1024;
    if (cap > STAGE_MAX) cap = STAGE_MAX;
    s.chunk_cap = cap;
    s.threads = 1024;
    if ((double)cap * g / 1024.0 < 16.0) s.threads = 512;
    const int ns = (s.threads / 32 / g) * 32;
    s.stage_field = cap + ns;
    s.span_cap = nb;
    s.window = 0;
    const size_t starts_bytes = (sizeof(int) * (size_t)g * (ns + 1) + 15) & ~(size_t)15;
    s.smem = SLOT_BYTES * (size_t)s.stage_field + starts_bytes + (s.hist_in_smem ? (size_t)g * hist_per : 0);
    return s;
}

void set_fold_tuning(const FoldTuning& t) {
    for (int c = 0; c < 32; c++) {
        g_group_cap[c].store(t.group_cap[c], std::memory_order_relaxed);
        g_threads[c].store(t.threads[c], std::memory_order_relaxed);
        g_lockstep[c].store(t.lockstep_min[c], std::memory_order_relaxed);
        g_pair[c].store(t.pair[c] ? 1u : 0u, std::memory_order_relaxed);
    }
    g_launch_periods.store(t.launch_periods ? t.launch_periods : 16384u, std::memory_order_relaxed);
    g_fold_steal.store(t.steal ? 1u : 0u, std::memory_order_relaxed);
    g_fused_scan.store(t.fused_scan ? 1u : 0u, std::memory_order_relaxed);
    g_map_lockstep.store(t.map_lockstep_min, std::memory_order_relaxed);
    g_map_threads.store(t.map_threads, std::memory_order_relaxed);
    g_map_group.store(t.map_group_max, std::memory_order_relaxed);
    g_batch_no_fill.store(t.batch_no_fill ? 1u : 0u, std::memory_order_relaxed);
}

void get_fold_tuning(FoldTuning* t) {
    for (int c = 0; c < 32; c++) {
        t->group_cap[c] = g_group_cap[c].load(std::memory_order_relaxed);
        t->threads[c] = g_threads[c].load(std::memory_order_relaxed);
        t->lockstep_min[c] = g_lockstep[c].load(std::memory_order_relaxed);
        t->pair[c] = g_pair[c].load(std::memory_order_relaxed);
    }
    t->launch_periods = g_launch_periods.load(std::memory_order_relaxed);
    t->steal = g_fold_steal.load(std::memory_order_relaxed);
    t->fused_scan = g_fused_scan.load(std::memory_order_relaxed);
    t->map_lockstep_min = g_map_lockstep.load(std::memory_order_relaxed);
    t->map_threads = g_map_threads.load(std::memory_order_relaxed);
    t->map_group_max = g_map_group.load(std::memory_order_relaxed);
    t->batch_no_fill = g_batch_no_fill.load(std::memory_order_relaxed);
}

bool tuned_batch_no_fill() { return g_batch_no_fill.load(std::memory_order_relaxed) != 0; }



bool tuned_fused_scan() { return g_fused_scan.load(std::memory_order_relaxed) != 0; }

bool tuned_fold_steal() { return g_fold_steal.load(std::memory_order_relaxed) != 0; }

uint32_t tuned_launch_periods() { return g_launch_periods.load(std::memory_order_relaxed); }

int fold_chunks(const double* time, int n, double scale_max, int nb, int span_cap, int chunk_cap, int* out,
                int capacity) {
    // A chunk spans less than `span` days, hence at most min(nb, span_cap) - 2
    // distinct cells at any scale <= scale_max (floor(x) - floor(y) <
    // x - y + 1): its cells are distinct bins.
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

int fold_chunk_list(const double* time, int n, double scale_max, int nb, int span_cap, int chunk_cap,
                    std::vector<int>& out) {
    const size_t full = (size_t)(n > 0 ? n : 0) + 2;
    size_t cap = full;
    if (n > 0 && chunk_cap > 0 && scale_max > 0.0) {
        const int cells = (nb < span_cap ? nb : span_cap) - 4;
        const double span = (double)(cells > 1 ? cells : 1) / scale_max;
        const double by_time = (time[n - 1] - time[0]) / span * (1.0 + 1e-9);
        if (by_time >= 0.0 && by_time < (double)n) cap = (size_t)by_time + (size_t)(n / chunk_cap) + 4;
        if (cap > full) cap = full;
    }
    out.resize(cap);
    int count = fold_chunks(time, n, scale_max, nb, span_cap, chunk_cap, out.data(), (int)out.size());
    if (count < 0 && cap < full) {  // the bound was short (it is not expected to be): the full size
        out.resize(full);
        count = fold_chunks(time, n, scale_max, nb, span_cap, chunk_cap, out.data(), (int)out.size());
    }
    if (count >= 0) out.resize((size_t)count + 1);
    return count;
}

// A CTA size and form of the walking fold: a power of two from 128 to 1024
// threads, at most 512 paired.
static bool walk_form_ok(int threads, bool pair) { return walk_threads_ok(threads) && (!pair || threads <= 512); }

// A group within a walking-fold shape's CTA: a power of two up to
// WALK_MAX_GROUP, at least WALK_MIN_LANES lanes per lane set (a period, or a
// pair of periods).
static bool walk_group_ok(int group, const FoldShape& shape) {
    return shape.kind == FOLD_WALK && walk_form_ok(shape.threads, shape.pair) && group == shape.group &&
           group >= (shape.pair ? 2 : 1) && group <= WALK_MAX_GROUP && (group & (group - 1)) == 0 &&
           (shape.pair ? group / 2 : group) <= shape.threads / WALK_MIN_LANES && shape.smem <= MAX_FOLD_SMEM;
}

template <bool PAIR>
static cudaError_t launch_fold_jobs_t(const FoldArgs* jobs, const int* cta0, int njobs, int ctas, int threads,
                                      size_t smem, cudaStream_t stream) {
    // Set at every launch: the attribute belongs to the module loaded in the
    // current context, which a cudaDeviceReset replaces.
    const cudaError_t e = cudaFuncSetAttribute(k_fold_walk_jobs<WALK_CAP, PAIR>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MAX_FOLD_SMEM);
    if (e != cudaSuccess) return e;
    k_fold_walk_jobs<WALK_CAP, PAIR><<<ctas, threads, smem, stream>>>(jobs, cta0, njobs);
    return cudaGetLastError();
}

cudaError_t launch_fold_jobs(const FoldArgs* jobs, const int* cta0, int njobs, int ctas, int threads, bool pair,
                             size_t smem, cudaStream_t stream) {
    if (njobs < 1 || ctas < 1 || smem > MAX_FOLD_SMEM || !walk_form_ok(threads, pair)) return cudaErrorInvalidValue;
    return pair ? launch_fold_jobs_t<true>(jobs, cta0, njobs, ctas, threads, smem, stream)
                : launch_fold_jobs_t<false>(jobs, cta0, njobs, ctas, threads, smem, stream);
}

template <bool PAIR>
static cudaError_t launch_fold_steal_t(const FoldArgs* jobs, const int* cta0, int njobs, int units, int threads,
                                       size_t smem, unsigned int* counter, int sm_count, cudaStream_t stream) {
    cudaError_t e = cudaFuncSetAttribute(k_fold_walk_steal<WALK_CAP, PAIR>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MAX_FOLD_SMEM);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), stream);
    if (e != cudaSuccess) return e;
    const int grid = units < sm_count ? units : sm_count;
    k_fold_walk_steal<WALK_CAP, PAIR><<<grid, threads, smem, stream>>>(jobs, cta0, njobs, units, counter);
    return cudaGetLastError();
}

cudaError_t launch_fold_steal(const FoldArgs* jobs, const int* cta0, int njobs, int units, int threads, bool pair,
                              size_t smem, unsigned int* counter, int sm_count, cudaStream_t stream) {
    if (njobs < 1 || units < 1 || smem > MAX_FOLD_SMEM || !counter || sm_count < 1 || !walk_form_ok(threads, pair))
        return cudaErrorInvalidValue;
    return pair ? launch_fold_steal_t<true>(jobs, cta0, njobs, units, threads, smem, counter, sm_count, stream)
                : launch_fold_steal_t<false>(jobs, cta0, njobs, units, threads, smem, counter, sm_count, stream);
}

// The fused scan's epilogue keeps, in the idle staging buffers (6 F
// doubles), each row's final carry, the groups' scratch and the CTA's tile
// winners.
static bool fused_epilogue_fits(const FoldArgs& a, const FoldShape& shape) {
    const size_t scratch = (size_t)(shape.threads / TILE) * ((sizeof(TileScratch) + 7) / 8);
    const size_t winners = (size_t)a.group * ((a.nb + TILE - 1) / TILE) * FUSED_PART_DOUBLES;
    return (size_t)a.group * NF + scratch + winners <= 6 * (size_t)(WALK_CAP + 2);
}

// The walking-fold limits on everything but the outputs.
static bool fold_job_ok_rows(const FoldArgs& a, const FoldShape& shape) {
    return walk_group_ok(a.group, shape) && a.lockstep_min >= 0 && a.nchunks >= 1 && a.nb >= 2 &&
           a.stage_field == WALK_CAP + 2 && shape.chunk_cap == WALK_CAP && a.row_stride == shape.row_stride &&
           a.row_stride >= a.nb && a.fault != nullptr && a.time && a.v && a.w && a.scales && a.chunks &&
           !(reinterpret_cast<uintptr_t>(a.time) & 15) && !(reinterpret_cast<uintptr_t>(a.v) & 15) &&
           !(reinterpret_cast<uintptr_t>(a.w) & 15);
}

bool fold_job_ok(const FoldArgs& a, const FoldShape& shape) {
    return walk_group_ok(a.group, shape) && a.lockstep_min >= 0 && a.nchunks >= 1 &&
           a.nb >= 2 && a.stage_field == WALK_CAP + 2 && shape.chunk_cap == WALK_CAP &&
           a.row_stride == shape.row_stride && a.row_stride >= a.nb && a.fault != nullptr &&
           (a.hist_out == nullptr || (a.group == 1 && a.periods == 1 && a.map_out == nullptr)) &&
           a.time && a.v && a.w && a.scales && a.chunks &&
           (a.map_out || a.hist_out || a.scan || (a.cum && a.cum32)) && (!a.scan == !a.merge) &&
           (!a.scan || (!a.map_out && !a.hist_out && fused_epilogue_fits(a, shape))) &&
           (!a.map_out || (a.map_nd >= 1 && a.map_nd <= MAP_MAX_DURATIONS && a.map_durations && a.map_rho)) &&
           !(reinterpret_cast<uintptr_t>(a.time) & 15) && !(reinterpret_cast<uintptr_t>(a.v) & 15) &&
           !(reinterpret_cast<uintptr_t>(a.w) & 15);
}

bool fold_smem_job_ok(const FoldArgs& a, const FoldShape& shape) {
    return shape.kind == FOLD_SMEM && shape.smem <= MAX_FOLD_SMEM && a.group == shape.group && a.group >= 1 &&
           a.group <= MAX_GROUP && (a.group & (a.group - 1)) == 0 && a.nchunks >= 1 &&
           (shape.threads == 1024 || shape.threads == 512) && a.group <= shape.threads / 32 &&
           a.stage_field == shape.stage_field && a.row_stride == shape.row_stride &&
           (shape.hist_in_smem || a.hist_global != nullptr) && a.map_out == nullptr && a.time && a.v && a.w &&
           a.scales && a.chunks && (a.hist_out ? (a.group == 1 && a.periods == 1) : (a.cum && a.cum32));
}

cudaError_t launch_fold_smem_jobs(const FoldArgs* jobs, const int* cta0, int njobs, int ctas, int threads, size_t smem,
                                  cudaStream_t stream) {
    if (njobs < 1 || ctas < 1 || smem > MAX_FOLD_SMEM || (threads != 1024 && threads != 512))
        return cudaErrorInvalidValue;
    // Set at every launch, as for the other fold kernels.
    const cudaError_t e =
        cudaFuncSetAttribute(k_fold_jobs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MAX_FOLD_SMEM);
    if (e != cudaSuccess) return e;
    k_fold_jobs<<<ctas, threads, smem, stream>>>(jobs, cta0, njobs);
    return cudaGetLastError();
}

bool fused_scan_ok(const FoldArgs& a, const ScanArgs& s, const MergeArgs& m) {
    return !a.map_out && !a.hist_out && s.scales && s.durations && s.rho && s.ingress && s.factors &&
           s.nb == a.nb && s.nd >= 1 && s.nd <= MAX_DURATIONS && s.ns >= 1 && s.ns <= MAX_SHAPES && s.layers >= 1 &&
           s.layers <= MAX_LAYERS && m.periods_in && m.scales && m.records && m.score && m.depth && m.flags_out &&
           m.periods == a.periods && m.offset >= 0;
}

cudaError_t launch_fold_scan(const FoldArgs& a, const FoldShape& shape, const ScanArgs& s, const MergeArgs& m,
                             cudaStream_t stream) {
    if (shape.kind != FOLD_WALK || a.scan || a.merge || !fused_scan_ok(a, s, m)) return cudaErrorInvalidValue;
    FoldArgs f = a;
    f.cum = nullptr;
    f.cum32 = nullptr;
    if (!fold_job_ok_rows(f, shape) || !fused_epilogue_fits(f, shape)) return cudaErrorInvalidValue;
    const int blocks = (a.periods + a.group - 1) / a.group;
    if (shape.pair) {
        const cudaError_t e = cudaFuncSetAttribute(k_fold_scan<WALK_CAP, true>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MAX_FOLD_SMEM);
        if (e != cudaSuccess) return e;
        k_fold_scan<WALK_CAP, true><<<blocks, shape.threads, shape.smem, stream>>>(f, s, m);
    } else {
        const cudaError_t e = cudaFuncSetAttribute(k_fold_scan<WALK_CAP, false>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MAX_FOLD_SMEM);
        if (e != cudaSuccess) return e;
        k_fold_scan<WALK_CAP, false><<<blocks, shape.threads, shape.smem, stream>>>(f, s, m);
    }
    return cudaGetLastError();
}

cudaError_t launch_fold(const FoldArgs& a, const FoldShape& shape, cudaStream_t stream) {
    // The shared-memory limit is an attribute of each kernel in the module
    // loaded in the current context; it is set at every launch, so a context
    // made again after cudaDeviceReset (which reloads the module) gets it too.
    {
        cudaError_t e = cudaFuncSetAttribute(k_fold, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MAX_FOLD_SMEM);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_fold_walk<WALK_CAP, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)MAX_FOLD_SMEM);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_fold_walk<WALK_CAP, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)MAX_FOLD_SMEM);
        if (e != cudaSuccess) return e;
    }
    if (!a.time || !a.v || !a.w || !a.scales || !a.chunks || (!a.hist_out && !a.map_out && (!a.cum || !a.cum32)))
        return cudaErrorInvalidValue;
    if (a.map_out && (shape.kind != FOLD_WALK || a.hist_out || a.map_nd < 1 || a.map_nd > MAP_MAX_DURATIONS ||
                      !a.map_durations || !a.map_rho))
        return cudaErrorInvalidValue;
    if (shape.kind == FOLD_WALK) {
        if (!walk_group_ok(a.group, shape) || a.lockstep_min < 0 || a.nchunks < 1 || a.nb < 2 ||
            a.stage_field != WALK_CAP + 2 || shape.chunk_cap != WALK_CAP || a.row_stride != shape.row_stride ||
            a.row_stride < a.nb || a.fault == nullptr || (a.hist_out != nullptr && a.group != 1) ||
            (reinterpret_cast<uintptr_t>(a.time) & 15) || (reinterpret_cast<uintptr_t>(a.v) & 15) ||
            (reinterpret_cast<uintptr_t>(a.w) & 15))
            return cudaErrorInvalidValue;
        const int blocks = (a.periods + a.group - 1) / a.group;
        if (shape.pair)
            k_fold_walk<WALK_CAP, true><<<blocks, shape.threads, shape.smem, stream>>>(a);
        else
            k_fold_walk<WALK_CAP, false><<<blocks, shape.threads, shape.smem, stream>>>(a);
        return cudaGetLastError();
    }
    if (shape.smem > MAX_FOLD_SMEM || a.group != shape.group || a.group > MAX_GROUP || a.group < 1 ||
        (a.group & (a.group - 1)) != 0 || a.nchunks < 1 || (shape.threads != 1024 && shape.threads != 512) ||
        a.group > shape.threads / 32 || a.stage_field != shape.stage_field || a.row_stride != shape.row_stride ||
        (!shape.hist_in_smem && a.hist_global == nullptr))
        return cudaErrorInvalidValue;
    const int blocks = (a.periods + a.group - 1) / a.group;
    k_fold<<<blocks, shape.threads, shape.smem, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace fbls
