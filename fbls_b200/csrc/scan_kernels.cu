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

namespace fbls {

// ---------------------------------------------------------------------------
// Tile scan (kernels.rs:610-845).
// ---------------------------------------------------------------------------

struct LaneState {
    double best;  // f64 pass
    float bestf;  // f32 pass: the reference keeps its f32 merits in the same f64 slot, exactly
    uint64_t key;
    uint32_t di;
    bool bad, sensitive, unsafe_merit;
    __device__ void reset() {
        best = neg_inf();
        bestf = -__builtin_huge_valf();
        key = KEY_MAX;
        di = 0;
        bad = sensitive = unsafe_merit = false;
    }
};

__device__ __forceinline__ float interval32(const float2* __restrict__ row, uint32_t start, uint32_t width) {
    float2 s = row[start];
    float2 e = row[start + width];
    return __fadd_rn(__fsub_rn(e.x, s.x), __fsub_rn(e.y, s.y));
}

__device__ __forceinline__ double interval64(const double* __restrict__ row, uint32_t start, uint32_t width) {
    return __dsub_rn(row[start + width], row[start]);
}

// f32 merit a^2 / (rho^2 (c norm - hp^2)) and the lane bookkeeping of
// rank_fast (kernels.rs:389-425).
__device__ __forceinline__ float rank_fast(LaneState& s, float a32, float hp32, float norm32, float rho2f,
                                           float basef, bool valid, uint64_t key, uint32_t di) {
    float cn = __fmul_rn(basef, norm32);
    float qq = __fmul_rn(rho2f, __fsub_rn(cn, __fmul_rn(hp32, hp32)));
    float merit = __fdiv_rn(__fmul_rn(a32, a32), qq);
    bool safe = cn > 0.0f && qq >= __fmul_rn(0.001f, cn) && merit >= 1e-30f && merit <= 1e30f;
    s.unsafe_merit |= valid && !safe;
    const float best = s.bestf;
    const float guard = 1e-5f;
    bool near = best > 0.0f && fabsf(__fsub_rn(merit, best)) <= __fmul_rn(guard, rmaxf(merit, best));
    bool far_better = merit > __fmul_rn(best, 1.00004f);
    if (valid && safe && far_better)
        s.sensitive = false;
    else
        s.sensitive = s.sensitive || (valid && safe && near);
    bool better = valid && safe && (merit > best || (merit == best && key < s.key));
    if (better) {
        s.bestf = merit;
        s.key = key;
        s.di = di;
    }
    return (valid && safe) ? merit : -__builtin_huge_valf();
}

// f64 score (a / rho) / sqrt(norm - hp^2 / c) and the bookkeeping of
// rank_exact (kernels.rs:428-455).
__device__ __forceinline__ double rank_exact(LaneState& s, double a, double hp, double norm, double rho,
                                             double baseline, bool valid, uint64_t key, uint32_t di) {
    double d = __ddiv_rn(__dmul_rn(hp, hp), baseline);
    double q = __dsub_rn(norm, d);
    s.bad |= valid && q <= 0.0;
    double candidate = __ddiv_rn(__ddiv_rn(a, rho), __dsqrt_rn(rmax(q, 1e-300)));
    double merit = (valid && q > 0.0 && candidate < __builtin_huge_val()) ? candidate : neg_inf();
    bool better = merit > s.best || (merit == s.best && key < s.key);
    if (better) {
        s.best = merit;
        s.key = key;
        s.di = di;
    }
    return merit;
}

// Staircase sums of shape si at (j, k) in f64 (kernels.rs:84-113).
__device__ __forceinline__ void shape_sums64(const double* __restrict__ rv, const double* __restrict__ rw, uint32_t j,
                                             uint32_t k, double oa, double ohp, double onorm, double ing,
                                             const double* __restrict__ factors, int si, int layers, double& a,
                                             double& hp, double& norm) {
    if (ing == 0.0) {
        a = oa;
        hp = ohp;
        norm = onorm;
        return;
    }
    const double l = (double)layers;
    const double l2 = __dmul_rn(l, l);
    a = __ddiv_rn(oa, l);
    hp = __ddiv_rn(ohp, l);
    norm = __ddiv_rn(onorm, l2);
    for (int layer = 1; layer < layers; layer++) {
        uint32_t width = layer_width(k, factors[si * layers + layer]);
        uint32_t start = j + (k - width) / 2;
        double dw = interval64(rw, start, width);
        a = __dadd_rn(a, __ddiv_rn(interval64(rv, start, width), l));
        hp = __dadd_rn(hp, __ddiv_rn(dw, l));
        norm = __dadd_rn(norm, __dmul_rn(dw, __ddiv_rn(__dadd_rn(__dmul_rn(2.0, (double)layer), 1.0), l2)));
    }
}

// The same sums in f32 from the (hi, lo) pairs (kernels.rs:117-146).
__device__ __forceinline__ void shape_sums32(const float2* __restrict__ rv, const float2* __restrict__ rw, uint32_t j,
                                             uint32_t k, float oa, float ohp, float onorm, double ing,
                                             const double* __restrict__ factors, int si, int layers, float& a,
                                             float& hp, float& norm) {
    if (ing == 0.0) {
        a = oa;
        hp = ohp;
        norm = onorm;
        return;
    }
    const float l = (float)layers;
    const float l2 = __fmul_rn(l, l);
    a = __fdiv_rn(oa, l);
    hp = __fdiv_rn(ohp, l);
    norm = __fdiv_rn(onorm, l2);
    for (int layer = 1; layer < layers; layer++) {
        uint32_t width = layer_width(k, factors[si * layers + layer]);
        uint32_t start = j + (k - width) / 2;
        float dw = interval32(rw, start, width);
        a = __fadd_rn(a, __fdiv_rn(interval32(rv, start, width), l));
        hp = __fadd_rn(hp, __fdiv_rn(dw, l));
        norm = __fadd_rn(norm, __fmul_rn(dw, __fdiv_rn(__fadd_rn(__fmul_rn(2.0f, (float)layer), 1.0f), l2)));
    }
}

// One CTA of the tile scan: tile `tile` (of `tiles`) of period `f`.
__device__ __forceinline__ void scan_tile_cta(const ScanArgs& a, const int tile, const int f, const int tiles) {
    __shared__ double s_rho[MAX_DURATIONS], s_ing[MAX_SHAPES];
    __shared__ double s_fac[MAX_SHAPES * MAX_LAYERS];
    __shared__ double s_wv[TILE / 32];
    __shared__ unsigned long long s_wk[TILE / 32];
    __shared__ int s_wl[TILE / 32];
    __shared__ uint32_t s_di;
    // Per duration, the same for every lane: width k = min(raw, nb / 2),
    // whether raw < nb / 2, and rho^2 in f32.
    __shared__ uint32_t s_k[MAX_DURATIONS];
    __shared__ unsigned char s_kok[MAX_DURATIONS];
    __shared__ float s_r2f[MAX_DURATIONS];

    const int lane = threadIdx.x;
    const int nb = a.nb;
    const int nd = a.nd, ns = a.ns, layers = a.layers;
    const uint32_t half = (uint32_t)(nb / 2);
    const double scale = a.scales[f];
    for (int i = lane; i < nd; i += TILE) {
        const double d = a.durations[i], r = a.rho[i];
        s_rho[i] = r;
        const uint32_t raw_k = template_width(d, scale);
        s_k[i] = min(raw_k, half);
        s_kok[i] = raw_k < half;
        s_r2f[i] = (float)(r * r);
    }
    for (int i = lane; i < ns; i += TILE) s_ing[i] = a.ingress[i];
    for (int i = lane; i < ns * layers; i += TILE) s_fac[i] = a.factors[i];
    __syncthreads();

    const uint32_t j = (uint32_t)(tile * TILE + lane);
    const uint32_t jj = min(j, (uint32_t)(nb - 1));
    const size_t stride = 2 * (size_t)nb + 1;
    const double* c64 = a.cum + (size_t)f * NF * stride;
    const float2* c32 = a.cum32 + (size_t)f * NF * stride;
    const double* rv64 = c64 + F_V * stride;
    const double* rw64 = c64 + F_W * stride;
    const double* rn64 = c64 + F_N * stride;
    const float2* rv32 = c32 + F_V * stride;
    const float2* rw32 = c32 + F_W * stride;
    const float2* rn32 = c32 + F_N * stride;
    const double baseline = a.baseline;
    const float basef = (float)baseline;
    const double nobs = a.n;
    const uint64_t nb1 = (uint64_t)nb + 1;
    // For an f32 count c: (double)c <= nobs - 3 exactly when c <= count_max.
    float count_max = (float)(nobs - 3.0);
    if ((double)count_max > nobs - 3.0) count_max = nextafterf(count_max, -__builtin_huge_valf());

    LaneState st;
    st.reset();
    // mixed: 1 = the reference's f32 pre-rank with f64 rescans and winner,
    // 0 = f64 ranking, 2 = the f32 form (f32 ranking and winner, no rescan).
    const bool f32_only = a.mixed == 2;
    bool fast = a.mixed != 0;
    bool retry = false;
    uint64_t winner_key = KEY_MAX;
    uint32_t winner_di = 0;
    double winner_value = neg_inf();
    bool bad_any = false;
    bool rescanned = false;

    for (int pass = 0; pass < 2; pass++) {
        if (pass == 1) {
            if (!retry) break;
            fast = false;
            rescanned = true;
            st.reset();
        }
        const double gate_value = fast ? __ddiv_rn(__dmul_rn(a.gate, a.gate), baseline) : a.gate;
        // For an f32 merit m: (double)m >= gate_value exactly when m >= gate_f.
        float gate_f = (float)gate_value;
        if ((double)gate_f < gate_value) gate_f = nextafterf(gate_f, __builtin_huge_valf());
        for (int di = 0; di < nd; di++) {
            const uint32_t k = s_k[di];
            const bool k_ok = s_kok[di] != 0;
            const double r = s_rho[di];
            const uint64_t key = (uint64_t)k * nb1 + jj;
            bool usable, open;
            float oa32 = 0.f, ow32 = 0.f;
            if (fast) {
                float count = interval32(rn32, jj, k);
                ow32 = interval32(rw32, jj, k);
                oa32 = interval32(rv32, jj, k);
                usable = j < (uint32_t)nb && k_ok && count >= 3.0f && count <= count_max;
                const bool valid = usable && oa32 > 0.0f;
                const float merit = rank_fast(st, oa32, ow32, ow32, s_r2f[di], basef, valid, key, (uint32_t)di);
                open = valid && merit >= gate_f;
            } else {
                double count = interval64(rn64, jj, k);
                double w = interval64(rw64, jj, k);
                double av = interval64(rv64, jj, k);
                usable = j < (uint32_t)nb && k_ok && count >= 3.0 && count <= nobs - 3.0;
                const bool valid = usable && av > 0.0;
                const double merit = rank_exact(st, av, w, w, r, baseline, valid, key, (uint32_t)di);
                open = valid && merit >= gate_value;
            }
            // Tile-level shape gate (kernels.rs:715-726).
            if (!__syncthreads_or(open)) continue;
            for (int si = 1; si < ns; si++) {
                const double ing = s_ing[si];
                const uint64_t skey = ((uint64_t)si * nb1 + k) * nb1 + jj;
                if (fast) {
                    float sa, shp, snorm;
                    shape_sums32(rv32, rw32, jj, k, oa32, ow32, ow32, ing, s_fac, si, layers, sa, shp, snorm);
                    rank_fast(st, sa, shp, snorm, s_r2f[di], basef, usable && sa > 0.0f, skey, (uint32_t)di);
                } else {
                    double w = interval64(rw64, jj, k);
                    double av = interval64(rv64, jj, k);
                    double sa, shp, snorm;
                    shape_sums64(rv64, rw64, jj, k, av, w, w, ing, s_fac, si, layers, sa, shp, snorm);
                    rank_exact(st, sa, shp, snorm, r, baseline, usable && sa > 0.0, skey, (uint32_t)di);
                }
            }
        }
        if (fast) st.best = (double)st.bestf;
        if (fast && st.best <= 0.0) st.key = nb1 + jj;
        // Block winner: largest value, then smallest key, then lowest lane.
        double v = st.best;
        unsigned long long k = st.key;
        int l = lane;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            double ov = __shfl_xor_sync(0xffffffffu, v, off);
            unsigned long long ok = __shfl_xor_sync(0xffffffffu, k, off);
            int ol = __shfl_xor_sync(0xffffffffu, l, off);
            if (ov > v || (ov == v && (ok < k || (ok == k && ol < l)))) {
                v = ov;
                k = ok;
                l = ol;
            }
        }
        if ((lane & 31) == 0) {
            s_wv[lane >> 5] = v;
            s_wk[lane >> 5] = k;
            s_wl[lane >> 5] = l;
        }
        __syncthreads();
        double bv = s_wv[0];
        unsigned long long bk = s_wk[0];
        int bl = s_wl[0];
#pragma unroll
        for (int w = 1; w < TILE / 32; w++) {
            double cv = s_wv[w];
            unsigned long long ck = s_wk[w];
            int cl = s_wl[w];
            if (cv > bv || (cv == bv && (ck < bk || (ck == bk && cl < bl)))) {
                bv = cv;
                bk = ck;
                bl = cl;
            }
        }
        const double guard = fast ? 1e-5 : 1e-10;
        const bool near_top = st.best > 0.0 && st.best >= __dmul_rn(bv, __dsub_rn(1.0, guard));
        if (lane == bl) s_di = st.di;
        const int near_count = __syncthreads_count(near_top);
        const bool near_sensitive = __syncthreads_or(near_top && st.sensitive);
        const bool unsafe_any = __syncthreads_or(st.unsafe_merit);
        const bool bad = __syncthreads_or(st.bad);
        winner_key = bk;
        winner_value = bv;
        winner_di = s_di;
        retry = fast && !f32_only && (unsafe_any || near_count > 1 || near_sensitive);
        bad_any = bad_any || bad;
        __syncthreads();
    }

    if (lane == 0 && f32_only) {
        // The f32 form: the winner's statistics from the (hi, lo) pairs in
        // f32, as the pre-rank reads them; no f64 rows are read.
        const uint32_t phase = (uint32_t)(winner_key % nb1);
        const uint32_t width = (uint32_t)((winner_key / nb1) % nb1);
        const uint32_t si = (uint32_t)(winner_key / (nb1 * nb1));
        const int sic = min((int)si, ns - 1);
        const double ing = s_ing[sic];
        const float rf = (float)s_rho[winner_di];
        const float w = interval32(rw32, phase, width);
        const float av = interval32(rv32, phase, width);
        float a0, hp, norm;
        shape_sums32(rv32, rw32, phase, width, av, w, w, ing, s_fac, sic, layers, a0, hp, norm);
        const float aa = __fdiv_rn(a0, rf);
        const float d = __fdiv_rn(__fmul_rn(hp, hp), basef);
        const float q = rmaxf(__fsub_rn(norm, d), 1e-30f);
        const double value = winner_value > neg_inf() ? (double)__fdiv_rn(aa, __fsqrt_rn(q)) : neg_inf();
        const double depth = (double)__fmul_rn(__fdiv_rn(aa, q), rf);
        const size_t idx = (size_t)f * tiles + tile;
        double* out = a.parts + idx * PART_STRIDE;
        out[0] = (double)phase;
        out[1] = (double)width;
        out[2] = (double)aa;
        out[3] = (double)norm;
        out[4] = (double)d;
        out[5] = ing;
        out[6] = s_rho[winner_di];
        out[7] = value;
        out[8] = depth;
        a.keys[idx] = winner_key;
        a.flags[idx] = 0u;
    } else if (lane == 0) {
        // The winner recomputed in f64 (kernels.rs:800-843).
        const uint32_t phase = (uint32_t)(winner_key % nb1);
        const uint32_t width = (uint32_t)((winner_key / nb1) % nb1);
        const uint32_t si = (uint32_t)(winner_key / (nb1 * nb1));
        const int sic = min((int)si, ns - 1);
        const double ing = s_ing[sic];
        const double r = s_rho[winner_di];
        const double w = interval64(rw64, phase, width);
        const double av = interval64(rv64, phase, width);
        double a0, hp, norm;
        shape_sums64(rv64, rw64, phase, width, av, w, w, ing, s_fac, sic, layers, a0, hp, norm);
        const double aa = __ddiv_rn(a0, r);
        const double d = __ddiv_rn(__dmul_rn(hp, hp), baseline);
        const double q = rmax(__dsub_rn(norm, d), 1e-300);
        const double value = winner_value > neg_inf() ? __ddiv_rn(aa, __dsqrt_rn(q)) : neg_inf();
        const double depth = __dmul_rn(__ddiv_rn(aa, q), r);
        const size_t idx = (size_t)f * tiles + tile;
        double* out = a.parts + idx * PART_STRIDE;
        out[0] = (double)phase;
        out[1] = (double)width;
        out[2] = aa;
        out[3] = norm;
        out[4] = d;
        out[5] = ing;
        out[6] = r;
        out[7] = value;
        out[8] = depth;
        a.keys[idx] = winner_key;
        a.flags[idx] = (uint32_t)retry | ((uint32_t)bad_any << 1) | ((uint32_t)rescanned << 2);
    }
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
    double best = neg_inf();
    uint64_t key = KEY_MAX;
    int chosen = 0;
    uint32_t fl = 0;
    for (int t = 0; t < a.tiles; t++) {
        const size_t idx = (size_t)f * a.tiles + t;
        double v = a.parts[idx * PART_STRIDE + 7];
        uint64_t k = a.keys[idx];
        fl |= a.flags[idx];
        if (v > best || (v == best && k < key)) {
            best = v;
            key = k;
            chosen = t;
        }
    }
    const double* part = a.parts + ((size_t)f * a.tiles + chosen) * PART_STRIDE;
    const size_t g = (size_t)a.offset + f;
    double* rec = a.records + g * RECORD_STRIDE;
    rec[0] = a.periods_in[f];
    rec[1] = a.scales[f];
    for (int i = 0; i < 7; i++) rec[2 + i] = part[i];
    a.score[g] = best;
    a.depth[g] = part[8];
    a.flags_out[g] = fl;
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
    const size_t stride = 2 * (size_t)nb + 1;
    const double* rv = a.cum + F_V * stride;
    const double* rw = a.cum + F_W * stride;
    const double* rn = a.cum + F_N * stride;
    const uint32_t half = nb / 2;
    for (int di = 0; di < a.nd; di++) {
        const uint32_t raw = template_width(a.durations[di], a.scale);
        const uint32_t k = raw < half ? raw : half;
        const double r = a.rho[di];
        const double count = interval64(rn, j, k);
        const double w = interval64(rw, j, k);
        const double av = interval64(rv, j, k);
        if (!(raw < half && count >= 3.0 && count <= a.n - 3.0)) continue;
        for (int si = 0; si < a.ns; si++) {
            double aa, hp, norm;
            shape_sums64(rv, rw, j, k, av, w, w, a.ingress[si], a.factors, si, a.layers, aa, hp, norm);
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
