// The tile scan of one (tile, period) by a group of TILE threads
// (src/search/kernels.rs:610-845: the two-pass f32 pre-rank / f64 rescan,
// the keys and tie-breaks, the shape gate and the f64 winner), written once
// over two choices:
//
//  * where the doubled prefix rows come from: the fold's rows in global
//    memory (GlobalRows: f64 rows and their (hi, lo) f32 pairs), or the
//    fold CTA's in-place prefix sums in shared memory (SmemRows: the f64
//    values, with the pair of a value split from it as the fold would have
//    written it, and the doubled half as first half + the row's final carry);
//  * which threads make up the group: a whole CTA of TILE threads (CtaGroup,
//    k_scan_tiles), or TILE threads of a larger fold CTA that scans its own
//    periods after the fold (NamedGroup: named-barrier reductions).
//
// Both row sources give the same values bit for bit, so every form of the
// scan returns the same records.
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace fbls {

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

__device__ __forceinline__ float2 split_pair(double value) {
    float hi = __double2float_rn(value);
    float lo = __double2float_rn(__dsub_rn(value, (double)hi));
    return make_float2(hi, lo);
}

__device__ __forceinline__ float pair_interval(float2 s, float2 e) {
    return __fadd_rn(__fsub_rn(e.x, s.x), __fsub_rn(e.y, s.y));
}

// Doubled prefix rows (2 nb + 1 entries per field) in global memory.
struct GlobalRows {
    const double* r64;   // NF rows of f64 values, stride 2 nb + 1
    const float2* r32;   // NF rows of (hi, lo) pairs
    size_t stride;
    __device__ __forceinline__ float i32(int f, uint32_t start, uint32_t width) const {
        const float2* row = r32 + f * stride;
        return pair_interval(row[start], row[start + width]);
    }
    __device__ __forceinline__ double i64(int f, uint32_t start, uint32_t width) const {
        const double* row = r64 + f * stride;
        return __dsub_rn(row[start + width], row[start]);
    }
};

// The same rows from a fold CTA's in-place prefix sums: bin b holds the
// inclusive prefix through b (v and w sums interleaved, counts as integers);
// entry i of the doubled row is 0 at i = 0, bin i - 1 up to nb, and bin
// i - nb - 1 plus the row's final carry beyond, as the fold's global rows
// are written.
struct SmemRows {
    const double2* vw;
    const uint32_t* c;
    const double* fin;  // NF final carries
    uint32_t nb;
    __device__ __forceinline__ double val(int f, uint32_t i) const {
        if (i == 0) return 0.0;
        const bool first = i <= nb;
        const uint32_t b = first ? i - 1 : i - nb - 1;
        const double x = f == F_V ? vw[b].x : (f == F_W ? vw[b].y : (double)c[b]);
        return first ? x : __dadd_rn(x, fin[f]);
    }
    __device__ __forceinline__ float i32(int f, uint32_t start, uint32_t width) const {
        return pair_interval(split_pair(val(f, start)), split_pair(val(f, start + width)));
    }
    __device__ __forceinline__ double i64(int f, uint32_t start, uint32_t width) const {
        return __dsub_rn(val(f, start + width), val(f, start));
    }
};

// A whole CTA of TILE threads.
struct CtaGroup {
    __device__ __forceinline__ int lane() const { return threadIdx.x; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
    __device__ __forceinline__ bool any(bool p) const { return __syncthreads_or(p) != 0; }
    __device__ __forceinline__ int count(bool p) const { return __syncthreads_count(p); }
};

// TILE consecutive threads (whole warps) of a larger CTA, on named barrier id.
struct NamedGroup {
    uint32_t id;
    int base;  // first thread
    __device__ __forceinline__ int lane() const { return (int)threadIdx.x - base; }
    __device__ __forceinline__ void sync() const {
        asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(TILE) : "memory");
    }
    __device__ __forceinline__ bool any(bool p) const {
        uint32_t r;
        asm volatile(
            "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, %2, %3, p;\n\t"
            "selp.u32 %0, 1, 0, q;\n\t}"
            : "=r"(r)
            : "r"((uint32_t)p), "r"(id), "n"(TILE)
            : "memory");
        return r != 0;
    }
    __device__ __forceinline__ int count(bool p) const {
        uint32_t r;
        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.popc.u32 %0, %2, %3, p;\n\t}"
                     : "=r"(r)
                     : "r"((uint32_t)p), "r"(id), "n"(TILE)
                     : "memory");
        return (int)r;
    }
};

// Shared memory of one scanning group.
struct TileScratch {
    double rho[MAX_DURATIONS];
    double ing[MAX_SHAPES];
    double fac[MAX_SHAPES * MAX_LAYERS];
    double wv[TILE / 32];
    unsigned long long wk[TILE / 32];
    float r2f[MAX_DURATIONS];   // rho^2 in f32
    uint32_t k[MAX_DURATIONS];  // width min(raw, nb / 2)
    int wl[TILE / 32];
    uint32_t di;
    unsigned char kok[MAX_DURATIONS];  // raw < nb / 2
};

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
template <typename Rows>
__device__ __forceinline__ void shape_sums64(const Rows& rows, uint32_t j, uint32_t k, double oa, double ohp,
                                             double onorm, double ing, const double* __restrict__ factors, int si,
                                             int layers, double& a, double& hp, double& norm) {
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
        double dw = rows.i64(F_W, start, width);
        a = __dadd_rn(a, __ddiv_rn(rows.i64(F_V, start, width), l));
        hp = __dadd_rn(hp, __ddiv_rn(dw, l));
        norm = __dadd_rn(norm, __dmul_rn(dw, __ddiv_rn(__dadd_rn(__dmul_rn(2.0, (double)layer), 1.0), l2)));
    }
}

// The same sums in f32 from the (hi, lo) pairs (kernels.rs:117-146).
template <typename Rows>
__device__ __forceinline__ void shape_sums32(const Rows& rows, uint32_t j, uint32_t k, float oa, float ohp,
                                             float onorm, double ing, const double* __restrict__ factors, int si,
                                             int layers, float& a, float& hp, float& norm) {
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
        float dw = rows.i32(F_W, start, width);
        a = __fadd_rn(a, __fdiv_rn(rows.i32(F_V, start, width), l));
        hp = __fadd_rn(hp, __fdiv_rn(dw, l));
        norm = __fadd_rn(norm, __fmul_rn(dw, __fdiv_rn(__fadd_rn(__fmul_rn(2.0f, (float)layer), 1.0f), l2)));
    }
}

// The per-period tables of a tile scan, by `count` threads from `first`:
// per duration the width k = min(raw, nb / 2), whether raw < nb / 2, rho and
// rho^2 in f32; the ingress fractions and layer factors.
__device__ __forceinline__ void fill_tile_tables(const ScanArgs& a, TileScratch& sc, double scale, int first,
                                                 int count) {
    const uint32_t half = (uint32_t)(a.nb / 2);
    for (int i = first; i < a.nd; i += count) {
        const double d = a.durations[i], r = a.rho[i];
        sc.rho[i] = r;
        const uint32_t raw_k = template_width(d, scale);
        sc.k[i] = min(raw_k, half);
        sc.kok[i] = raw_k < half;
        sc.r2f[i] = (float)(r * r);
    }
    for (int i = first; i < a.ns; i += count) sc.ing[i] = a.ingress[i];
    for (int i = first; i < a.ns * a.layers; i += count) sc.fac[i] = a.factors[i];
}

// Lane 0's last step of a tile: the winner's statistics (recomputed in f64
// (kernels.rs:800-843), or in f32 from the pairs in the f32 form) into
// out[PART_STRIDE], the key and the flags.
template <typename Rows>
__device__ __forceinline__ void write_tile_winner(const ScanArgs& a, const Rows& rows, const TileScratch& sc,
                                                  bool f32_only, uint64_t winner_key, uint32_t winner_di,
                                                  double winner_value, bool retry, bool bad_any, bool rescanned,
                                                  double* out, uint64_t* key_out, uint32_t* flag_out) {
    const int nb = a.nb, ns = a.ns, layers = a.layers;
    const uint64_t nb1 = (uint64_t)nb + 1;
    const double baseline = a.baseline;
    const float basef = (float)baseline;
    if (f32_only) {
        // The f32 form: the winner's statistics from the (hi, lo) pairs in
        // f32, as the pre-rank reads them; no f64 rows are read.
        const uint32_t phase = (uint32_t)(winner_key % nb1);
        const uint32_t width = (uint32_t)((winner_key / nb1) % nb1);
        const uint32_t si = (uint32_t)(winner_key / (nb1 * nb1));
        const int sic = min((int)si, ns - 1);
        const double ing = sc.ing[sic];
        const float rf = (float)sc.rho[winner_di];
        const float w = rows.i32(F_W, phase, width);
        const float av = rows.i32(F_V, phase, width);
        float a0, hp, norm;
        shape_sums32(rows, phase, width, av, w, w, ing, sc.fac, sic, layers, a0, hp, norm);
        const float aa = __fdiv_rn(a0, rf);
        const float d = __fdiv_rn(__fmul_rn(hp, hp), basef);
        const float q = rmaxf(__fsub_rn(norm, d), 1e-30f);
        const double value = winner_value > neg_inf() ? (double)__fdiv_rn(aa, __fsqrt_rn(q)) : neg_inf();
        const double depth = (double)__fmul_rn(__fdiv_rn(aa, q), rf);
        out[0] = (double)phase;
        out[1] = (double)width;
        out[2] = (double)aa;
        out[3] = (double)norm;
        out[4] = (double)d;
        out[5] = ing;
        out[6] = sc.rho[winner_di];
        out[7] = value;
        out[8] = depth;
        *key_out = winner_key;
        *flag_out = 0u;
    } else {
        // The winner recomputed in f64 (kernels.rs:800-843).
        const uint32_t phase = (uint32_t)(winner_key % nb1);
        const uint32_t width = (uint32_t)((winner_key / nb1) % nb1);
        const uint32_t si = (uint32_t)(winner_key / (nb1 * nb1));
        const int sic = min((int)si, ns - 1);
        const double ing = sc.ing[sic];
        const double r = sc.rho[winner_di];
        const double w = rows.i64(F_W, phase, width);
        const double av = rows.i64(F_V, phase, width);
        double a0, hp, norm;
        shape_sums64(rows, phase, width, av, w, w, ing, sc.fac, sic, layers, a0, hp, norm);
        const double aa = __ddiv_rn(a0, r);
        const double d = __ddiv_rn(__dmul_rn(hp, hp), baseline);
        const double q = rmax(__dsub_rn(norm, d), 1e-300);
        const double value = winner_value > neg_inf() ? __ddiv_rn(aa, __dsqrt_rn(q)) : neg_inf();
        const double depth = __dmul_rn(__ddiv_rn(aa, q), r);
        out[0] = (double)phase;
        out[1] = (double)width;
        out[2] = aa;
        out[3] = norm;
        out[4] = d;
        out[5] = ing;
        out[6] = r;
        out[7] = value;
        out[8] = depth;
        *key_out = winner_key;
        *flag_out = (uint32_t)retry | ((uint32_t)bad_any << 1) | ((uint32_t)rescanned << 2);
    }
}

// Tile `tile` of one period of scan `a` (scale nb / period) by group `grp`,
// with its shared memory `sc`; the tile's winner goes to out[PART_STRIDE],
// *key_out and *flag_out. Every thread of the group calls it; the group's
// threads must not touch `sc` from an earlier call when it starts (it begins
// by filling it).
template <typename Rows, typename Group>
__device__ __forceinline__ void scan_tile(const ScanArgs& a, const Rows& rows, const Group& grp, TileScratch& sc,
                                          const int tile, const double scale, double* out, uint64_t* key_out,
                                          uint32_t* flag_out) {
    const int lane = grp.lane();
    const int nb = a.nb;
    const int nd = a.nd, ns = a.ns, layers = a.layers;
    fill_tile_tables(a, sc, scale, lane, TILE);
    grp.sync();

    const uint32_t j = (uint32_t)(tile * TILE + lane);
    const uint32_t jj = min(j, (uint32_t)(nb - 1));
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
            const uint32_t k = sc.k[di];
            const bool k_ok = sc.kok[di] != 0;
            const double r = sc.rho[di];
            const uint64_t key = (uint64_t)k * nb1 + jj;
            bool usable, open;
            float oa32 = 0.f, ow32 = 0.f;
            if (fast) {
                float count = rows.i32(F_N, jj, k);
                ow32 = rows.i32(F_W, jj, k);
                oa32 = rows.i32(F_V, jj, k);
                usable = j < (uint32_t)nb && k_ok && count >= 3.0f && count <= count_max;
                const bool valid = usable && oa32 > 0.0f;
                const float merit = rank_fast(st, oa32, ow32, ow32, sc.r2f[di], basef, valid, key, (uint32_t)di);
                open = valid && merit >= gate_f;
            } else {
                double count = rows.i64(F_N, jj, k);
                double w = rows.i64(F_W, jj, k);
                double av = rows.i64(F_V, jj, k);
                usable = j < (uint32_t)nb && k_ok && count >= 3.0 && count <= nobs - 3.0;
                const bool valid = usable && av > 0.0;
                const double merit = rank_exact(st, av, w, w, r, baseline, valid, key, (uint32_t)di);
                open = valid && merit >= gate_value;
            }
            // Tile-level shape gate (kernels.rs:715-726).
            if (!grp.any(open)) continue;
            for (int si = 1; si < ns; si++) {
                const double ing = sc.ing[si];
                const uint64_t skey = ((uint64_t)si * nb1 + k) * nb1 + jj;
                if (fast) {
                    float sa, shp, snorm;
                    shape_sums32(rows, jj, k, oa32, ow32, ow32, ing, sc.fac, si, layers, sa, shp, snorm);
                    rank_fast(st, sa, shp, snorm, sc.r2f[di], basef, usable && sa > 0.0f, skey, (uint32_t)di);
                } else {
                    double w = rows.i64(F_W, jj, k);
                    double av = rows.i64(F_V, jj, k);
                    double sa, shp, snorm;
                    shape_sums64(rows, jj, k, av, w, w, ing, sc.fac, si, layers, sa, shp, snorm);
                    rank_exact(st, sa, shp, snorm, r, baseline, usable && sa > 0.0, skey, (uint32_t)di);
                }
            }
        }
        if (fast) st.best = (double)st.bestf;
        if (fast && st.best <= 0.0) st.key = nb1 + jj;
        // Group winner: largest value, then smallest key, then lowest lane.
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
            sc.wv[lane >> 5] = v;
            sc.wk[lane >> 5] = k;
            sc.wl[lane >> 5] = l;
        }
        grp.sync();
        double bv = sc.wv[0];
        unsigned long long bk = sc.wk[0];
        int bl = sc.wl[0];
#pragma unroll
        for (int w = 1; w < TILE / 32; w++) {
            double cv = sc.wv[w];
            unsigned long long ck = sc.wk[w];
            int cl = sc.wl[w];
            if (cv > bv || (cv == bv && (ck < bk || (ck == bk && cl < bl)))) {
                bv = cv;
                bk = ck;
                bl = cl;
            }
        }
        const double guard = fast ? 1e-5 : 1e-10;
        const bool near_top = st.best > 0.0 && st.best >= __dmul_rn(bv, __dsub_rn(1.0, guard));
        if (lane == bl) sc.di = st.di;
        const int near_count = grp.count(near_top);
        const bool near_sensitive = grp.any(near_top && st.sensitive);
        const bool unsafe_any = grp.any(st.unsafe_merit);
        const bool bad = grp.any(st.bad);
        winner_key = bk;
        winner_value = bv;
        winner_di = sc.di;
        retry = fast && !f32_only && (unsafe_any || near_count > 1 || near_sensitive);
        bad_any = bad_any || bad;
        grp.sync();
    }

    if (lane == 0)
        write_tile_winner(a, rows, sc, f32_only, winner_key, winner_di, winner_value, retry, bad_any, rescanned, out,
                          key_out, flag_out);
}

// Period f's record from its best tile's part (PART_STRIDE doubles), its
// score and its ORed tile flags (kernels.rs:1115-1155).
__device__ __forceinline__ void merge_record(const MergeArgs& a, const int f, const double* part, double best,
                                             uint32_t fl) {
    const size_t g = (size_t)a.offset + f;
    double* rec = a.records + g * RECORD_STRIDE;
    rec[0] = a.periods_in[f];
    rec[1] = a.scales[f];
    for (int i = 0; i < 7; i++) rec[2 + i] = part[i];
    a.score[g] = best;
    a.depth[g] = part[8];
    a.flags_out[g] = fl;
}

// Best tile of period f by (score, lowest key), flags ORed, into the merge's
// record; parts, keys and flags are the period's `tiles` tile winners.
__device__ __forceinline__ void merge_tiles(const double* parts, const uint64_t* keys, const uint32_t* flags,
                                            int tiles, const MergeArgs& a, const int f) {
    double best = neg_inf();
    uint64_t key = KEY_MAX;
    int chosen = 0;
    uint32_t fl = 0;
    for (int t = 0; t < tiles; t++) {
        double v = parts[(size_t)t * PART_STRIDE + 7];
        uint64_t k = keys[t];
        fl |= flags[t];
        if (v > best || (v == best && k < key)) {
            best = v;
            key = k;
            chosen = t;
        }
    }
    merge_record(a, f, parts + (size_t)chosen * PART_STRIDE, best, fl);
}

}  // namespace fbls
