// Joint planet / binary / noise evidence for a batch of candidates on sm_100a.
//
// What is computed is compare_search (src/search/evidence.rs): the family is
// folded over two periods (2 nb bins, so a template at phase j pairs with its
// odd-cycle counterpart at j + nb); for every phase, duration and staircase
// shape a screen statistic, then a joint pass in which each template's planet
// and binary evidences integrate a positive depth under half-normal priors
// over discrete secondary-eclipse scenarios (quarter phases) and odd/even
// depth ratios at twice the period, pruned per tile of 64 phases against
// floors set by one pilot template; finally log-sum-exp over every template
// and the two winners (by joint evidence and by amplitude).
//
// How it runs here (this file's own decomposition):
//   * Candidates are batched: many (family, period) pairs go through one set
//     of launches on one stream with one host synchronisation. The folds are
//     job launches of the deterministic fold kernels (fold.cu), then
//     k_ev_prefix (all candidates' rows), k_ev_screen, k_ev_pilot, k_ev_joint.
//   * The host turns each candidate's durations, staircase shapes and orbit
//     bank into segment tables (interval offsets and widths per layer,
//     coefficients, secondary shifts), so the device only reads tables and
//     prefix rows; nothing is recomputed per phase lane.
//   * A CTA holds 8 tiles of the same candidate (512 threads) and first
//     bulk-copies the candidate's three prefix rows into shared memory (one
//     cp.async.bulk on an mbarrier, bounded wait) when they fit.
//   * A tile is two warps. All tile-level decisions (the pruning maxima, the
//     winners, the log-sum-exp) are warp butterflies plus one exchange
//     through shared memory under a 64-thread named barrier; the four
//     pruning maxima of a (duration, shape) step are reduced together, one
//     barrier per step.
//   * The pilot (winner tile of the screen, its template evaluated without
//     pruning, the floors) runs on the device, one warp per candidate, so the
//     joint pass follows without a host round trip; a candidate below the
//     threshold is marked inactive there and its joint CTAs return at once.
//
// The per-template arithmetic (interval sums, the two-template subspace
// bound, the evidence integrals and their log-sum order) and the per-tile
// pruning decisions are the reference's: both are visible in the output.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "bulk.cuh"
#include "common.cuh"
#include "evidence.h"
#include "kernels.h"

namespace fbls {

namespace {

constexpr int EV_CTA_TILES = 8;                     // tiles per CTA
constexpr int EV_THREADS = EV_CTA_TILES * EV_TILE;  // 512
constexpr int EV_REC = 22;     // per tile: 2 selections x 10 values, then the tile's planet and binary log sums
constexpr int EV_SCREEN = 4;   // per tile: max score, planet bound, binary bound, key
constexpr int EV_PILOT = 6;    // floor_p, floor_b, pilot key, active, screen maximum, pilot tile
constexpr int EV_NRATIO = 5;   // secondary-depth ratios of the quarter-phase scenarios
constexpr int EV_NODD = 7;     // odd/even depth ratios at twice the period

// Duration step: width k in bins (capped at nb2 / 8 - 1), whether the raw
// width is below nb2 / 8, rho^2 and the duration's log mass.
struct EvDur {
    double rho2;
    double dlm;
    int k;
    int raw_ok;
};

// One staircase layer of an interval template: the layer covers
// [start + off, start + off + inner) with weights lin (sums) and sq (norms).
struct EvLayer {
    int off;
    int inner;
    double lin;
    double sq;
};

// One secondary phase of the orbit bank at a duration: the secondary's start
// relative to the primary's, its phase and log masses (planet, binary).
struct EvOrbit {
    int shift;
    int pad;
    double phase;
    double logwp;
    double logwb;
};

struct EvCand {
    const double* hist;  // 3 x nb2, the two-period fold
    double* cum;         // 3 rows of rs = nb2 + 2 doubles: exclusive prefix (v, w, count) over 2 nb bins
    double* screen;      // tiles x EV_SCREEN
    double* rec;         // tiles x parts x EV_REC
    double* pilot;       // EV_PILOT
    const EvDur* dur;    // nd
    const EvLayer* lay;  // nd x ns x L: the template at width k
    const EvOrbit* orb;  // nd x NORB
    double* mom;         // (nd x ns) x 3 x nb2: the moment table (see k_ev_screen)
    const double* priors;  // ns x 2: shape log priors (planet, binary)
    double c;            // baseline_norm
    double n;            // observations
    double threshold;
    double margin;       // log(rtol) - log((NORB + 1) nb nd ns)
    int nb, nd, ns, L, tiles, stage;
    int cta0;            // first CTA of the candidate in its screen launch
    int cta0j;           // first CTA of the candidate in its joint launch
    int parts;           // the joint pass splits the durations into this many parts, one CTA each
};

// Batch-wide constants of the evidence model (evidence.rs:665-689 and the
// logs of its scenario weights).
struct EvConst {
    double tau_p, tau_b, tau_d;
    double ratio_p[EV_NRATIO], lnw_p[EV_NRATIO], lnw_b[EV_NRATIO];
    double ratio_o[EV_NODD];
    double ln_odd;        // log(0.25 / 7)
    double ln_screen_p;   // log 0.75
    double ln_screen_b;   // log 0.025
    double ln_tile;       // log 64: a pilot tile's log sum of 64 equal terms
};

__device__ __forceinline__ double qnan() { return __longlong_as_double(0x7ff8000000000000ll); }

// Circular interval sum of one prefix row over 2 nb bins: [start, start +
// width) with start < 2 nb2 (the host checks the tables against this bound).
__device__ __forceinline__ double circ(const double* row, int start, int width, int nb2) {
    const int j = start >= nb2 ? start - nb2 : start;
    const int end = j + width;
    const double left = row[j];
    const double right = row[end < nb2 ? end : nb2];
    const double wrap = row[end > nb2 ? end - nb2 : 0];
    return right - left + wrap;
}

// Staircase sums of one template at the even start p0 and the odd start p1:
// v-field sums (a0, a1), w-field sums (p0, p1) and norms (n0, n1).
struct Sums {
    double a0, a1, w0, w1, q0, q1;
};

__device__ __forceinline__ Sums staircase(const double* cum, int rs, int nb2, int p0, int p1, const EvLayer* T,
                                          int L) {
    Sums s{0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const double* rv = cum;
    const double* rw = cum + rs;
    for (int l = 0; l < L; l++) {
        const EvLayer t = T[l];
        const double v0 = circ(rv, p0 + t.off, t.inner, nb2), v1 = circ(rv, p1 + t.off, t.inner, nb2);
        const double w0 = circ(rw, p0 + t.off, t.inner, nb2), w1 = circ(rw, p1 + t.off, t.inner, nb2);
        s.a0 += t.lin * v0;
        s.a1 += t.lin * v1;
        s.w0 += t.lin * w0;
        s.w1 += t.lin * w1;
        s.q0 += t.sq * w0;
        s.q1 += t.sq * w1;
    }
    return s;
}

// Exchange of per-warp partial results between the two warps of a tile: one
// 64-thread named barrier per exchange, slots double-buffered so that a slot
// is rewritten only after both warps passed the barrier of the exchange in
// between.
struct TileRed {
    double (*slot)[EV_CTA_TILES][2][4];
    int tl, half, bar, parity;

    __device__ __forceinline__ void exchange(const double* mine, int count, double* other) {
        if ((threadIdx.x & 31) == 0)
            for (int i = 0; i < count; i++) slot[parity][tl][half][i] = mine[i];
        group_sync((uint32_t)bar, 2 * 32);
        for (int i = 0; i < count; i++) other[i] = slot[parity][tl][half ^ 1][i];
        parity ^= 1;
    }

    // Maximum over the tile's 64 lanes of four values (NaN loses).
    __device__ __forceinline__ void max4(double* v) {
        for (int off = 16; off > 0; off >>= 1)
            for (int i = 0; i < 4; i++) v[i] = rmax(v[i], __shfl_xor_sync(0xffffffffu, v[i], off));
        double o[4];
        exchange(v, 4, o);
        for (int i = 0; i < 4; i++) v[i] = rmax(v[i], o[i]);
    }

    __device__ __forceinline__ double max1(double v) {
        for (int off = 16; off > 0; off >>= 1) v = rmax(v, __shfl_xor_sync(0xffffffffu, v, off));
        double o;
        exchange(&v, 1, &o);
        return rmax(v, o);
    }

    __device__ __forceinline__ double sum1(double v) {
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        double o;
        exchange(&v, 1, &o);
        return half == 0 ? v + o : o + v;  // the same sum on both warps
    }
};

// Pruning decisions of one (duration, shape) step, as a 4-bit mask: bit o
// (o < 3) keeps the quarter-phase secondary o, bit 3 keeps the odd/even
// alternative. A step keeps a scenario when the tile's largest upper bound
// reaches its floor (0 for the secondaries, floor_b for odd/even).
__device__ __forceinline__ uint32_t keep_mask(const double* up, double floor_b) {
    return (up[0] >= 0.0 ? 1u : 0u) | (up[1] >= 0.0 ? 2u : 0u) | (up[2] >= 0.0 ? 4u : 0u) |
           (up[3] >= floor_b ? 8u : 0u);
}

// Decisions of a tile: the maxima over its 64 lanes; lane 0 records the
// step's mask for the replay of the tile's winners.
struct TileDecide {
    TileRed* red;
    uint8_t* record;  // [nd x ns] of this tile
    int lane;
    __device__ __forceinline__ uint32_t operator()(double* up, double floor_b, int step) const {
        red->max4(up);
        const uint32_t m = keep_mask(up, floor_b);
        if (lane == 0) record[step] = (uint8_t)m;
        return m;
    }
};

// Decisions of a single template (the pilot): its own bounds.
struct OwnDecide {
    __device__ __forceinline__ uint32_t operator()(double* up, double floor_b, int) const {
        return keep_mask(up, floor_b);
    }
};

// Decisions recorded by the tile pass, for replaying one template.
struct ReplayDecide {
    uint32_t mask;
    __device__ __forceinline__ uint32_t operator()(double*, double, int) const { return mask; }
};

// One evaluated template.
struct Eval {
    double snr, depth, lp, lb, sec_ratio, sec_phase, odd_ratio, binary_multiple;
    bool valid;
};

// Running state of one phase lane over its templates: the winners' merits
// and keys (their values are recomputed at the end by replaying the winning
// template) and the log sums.
struct Lane {
    double best_joint, best_signal;
    unsigned long long joint_key, signal_key;
    double sum_p, sum_b;
};

__device__ __forceinline__ void lane_init(Lane& S) {
    S.best_joint = S.best_signal = neg_inf();
    S.joint_key = S.signal_key = KEY_MAX;
    S.sum_p = S.sum_b = neg_inf();
}

// Row p (taken mod 2 nb) of step `step`'s moment table: the staircase's
// v sum, w sum and norm of the template starting at bin p.
__device__ __forceinline__ void moment(const EvCand& C, int step, int p, double& a, double& w, double& q) {
    const int nb2 = 2 * C.nb;
    if (p >= nb2) p -= nb2;
    const double* t = C.mom + (size_t)step * 3 * nb2;
    a = t[p];
    w = t[nb2 + p];
    q = t[2 * (size_t)nb2 + p];
}

// The secondary of orbit entry `o` (a template of the same width, the
// reference's bank having duration ratio 1, at the primary's start plus the
// entry's shift) over both cycles: its v sum, w sum and norm.
__device__ __forceinline__ void secondary(const EvCand& C, int step, int jj, int di, int o, double& ass, double& ps,
                                          double& nsum) {
    const int s0 = jj + C.orb[di * NORB + o].shift;
    double a0, w0, q0, a1, w1, q1;
    moment(C, step, s0, a0, w0, q0);
    moment(C, step, (s0 >= 2 * C.nb ? s0 - 2 * C.nb : s0) + C.nb, a1, w1, q1);
    ass = a0 + a1;
    ps = w0 + w1;
    nsum = q0 + q1;
}

// One template (phase jj, duration di, shape si) of the joint pass: its
// amplitude statistics, the upper bounds of its quarter-phase secondaries and
// odd/even alternative, the tile-level pruning (red.max4: the tile's maxima,
// or the template's own values in the pilot), the evidence sums of the
// scenarios kept, and the lane's winners and log sums.
template <class Decide>
__device__ __forceinline__ Eval joint_template(const EvCand& C, const EvConst& K, const double* cum, int rs, int jj,
                                               bool jv, int di, int si, double floor_p, double floor_b, bool usable,
                                               const Decide& decide) {
    const int nb = C.nb, nb2 = 2 * nb;
    const double c = C.c;
    const EvDur D = C.dur[di];
    const double rho2 = D.rho2, dlm = D.dlm;
    const int step = di * C.ns + si;
    double ae, ao, pe, po, ne, no;
    moment(C, step, jj, ae, pe, ne);
    moment(C, step, jj + nb, ao, po, no);
    const double qe = ne - pe * pe / c, qo = no - po * po / c, qeo = -pe * po / c;
    const double ap = ae + ao, qp = qe + qo + 2.0 * qeo;
    const double snr = ap / sqrt(rmax(qp * rho2, 1e-300));
    const double depth = ap / rmax(qp, 1e-300);
    const bool valid = usable && ap > 0.0 && qp > 0.0 && snr >= C.threshold;

    // Upper bounds: [0..2] the quarter-phase secondaries, [3] odd/even.
    double up[4], raw[4];
    for (int o = 0; o < NORB; o++) {
        const EvOrbit& O = C.orb[di * NORB + o];
        double ass, ps, nsum;
        secondary(C, step, jj, di, o, ass, ps, nsum);
        const double qs = nsum - ps * ps / c;
        const double qps = -(pe + po) * ps / c;
        const double su = subspace_upper(ap / rho2, ass / rho2, qp / rho2, qs / rho2, qps / rho2, 1.0);
        const double pu = su + O.logwp + 1e-6;
        const double bu = su + O.logwb + 1e-6;
        double u = rmax(pu - floor_p, bu - floor_b) + dlm;
        if (!(O.logwp > neg_inf() || O.logwb > neg_inf())) u = neg_inf();
        raw[o] = O.logwb > neg_inf() ? bu : neg_inf();
        up[o] = jv ? u : neg_inf();
    }
    const double ba = ae / rho2, bb = ao / rho2, bq = qe / rho2, br = qo / rho2, bx = qeo / rho2;
    const double alias_mass = D.k < nb2 / 8 ? 0.0 : neg_inf();
    raw[3] = subspace_upper(ba, bb, bq, br, bx, 1.0) + 1e-6 + alias_mass;
    up[3] = jv ? raw[3] + dlm : neg_inf();
    const uint32_t keep = decide(up, floor_b, step);

    double lp = neg_inf(), lb = neg_inf(), component_best = neg_inf(), omitted_upper = neg_inf();
    double sec_ratio = 0.0, sec_phase = 0.5, odd_ratio = 1.0, binary_multiple = 1.0;
    for (int o = 0; o < NORB; o++) {
        if (keep & (1u << o)) {
            const EvOrbit& O = C.orb[di * NORB + o];
            double ass, ps, nsum;
            secondary(C, step, jj, di, o, ass, ps, nsum);
            const double qs = nsum - ps * ps / c;
            const double qps = -(pe + po) * ps / c;
            const double pa = ap / rho2, pb = ass / rho2, pq = qp / rho2, pr = qs / rho2, px = qps / rho2;
            for (int ri = 0; ri < EV_NRATIO; ri++) {
                const double ratio = K.ratio_p[ri];
                const double aa = pa + ratio * pb;
                const double qq = pq + 2.0 * ratio * px + ratio * ratio * pr;
                const double ep = positive_amplitude_evidence(aa, qq, K.tau_p) + K.lnw_p[ri] + O.logwp;
                const double diluted = positive_amplitude_evidence(aa, qq, K.tau_d);
                const double eb = log_add(positive_amplitude_evidence(aa, qq, K.tau_b), diluted) + K.lnw_b[ri] + O.logwb;
                lp = log_add(lp, ep);
                lb = log_add(lb, eb);
                if (eb > component_best) {
                    sec_ratio = ratio;
                    sec_phase = O.phase;
                    component_best = eb;
                }
            }
        } else if (raw[o] > omitted_upper) {
            omitted_upper = raw[o];
        }
    }
    if (keep & 8u) {
        for (int ri = 0; ri < EV_NODD; ri++) {
            const double ratio = K.ratio_o[ri];
            const double aa = ba + ratio * bb;
            const double qq = bq + 2.0 * ratio * bx + ratio * ratio * br;
            const double diluted = positive_amplitude_evidence(aa, qq, K.tau_d);
            const double eb = log_add(positive_amplitude_evidence(aa, qq, K.tau_b), diluted) + alias_mass + K.ln_odd;
            lb = log_add(lb, eb);
            if (eb > component_best) {
                sec_ratio = 0.0;
                sec_phase = 0.5;
                odd_ratio = ratio;
                binary_multiple = 2.0;
                component_best = eb;
            }
        }
    } else if (raw[3] > omitted_upper) {
        omitted_upper = raw[3];
    }
    if (!(component_best > omitted_upper)) sec_ratio = sec_phase = odd_ratio = binary_multiple = qnan();
    lp += C.priors[2 * si] + dlm;
    lb += C.priors[2 * si + 1] + dlm;
    return Eval{snr, depth, lp, lb, sec_ratio, sec_phase, odd_ratio, binary_multiple, valid};
}

// Folds one evaluated template (phase jj, duration di, shape si) into the
// lane's log sums (phases inside the cycle only) and winners.
__device__ __forceinline__ void lane_add(const EvCand& C, Lane& S, const Eval& e, bool jv, int jj, int di, int si) {
    if (jv) {
        S.sum_p = log_add(S.sum_p, e.lp);
        S.sum_b = log_add(S.sum_b, e.lb);
    }
    const unsigned long long key =
        (unsigned long long)(si * C.nd + di) * (unsigned long long)C.nb + (unsigned long long)jj;
    if (e.valid && (e.lp > S.best_joint || (e.lp == S.best_joint && key < S.joint_key))) {
        S.best_joint = e.lp;
        S.joint_key = key;
    }
    if (e.valid && (e.snr > S.best_signal || (e.snr == S.best_signal && key < S.signal_key))) {
        S.best_signal = e.snr;
        S.signal_key = key;
    }
}

// Count window check of a template at duration di: 3 .. n - 3 observations
// over both cycles and the raw width below nb2 / 8.
__device__ __forceinline__ bool usable_at(const EvCand& C, const double* cum, int rs, int jj, bool jv, int di) {
    const int nb2 = 2 * C.nb;
    const EvDur D = C.dur[di];
    const double* rn = cum + 2 * (size_t)rs;
    const double count = circ(rn, jj, D.k, nb2) + circ(rn, jj + C.nb, D.k, nb2);
    return jv && D.raw_ok && count >= 3.0 && count <= C.n - 3.0;
}

// The candidate of a CTA: the last candidate whose first CTA (cta0 in the
// screen launch, cta0j in the joint launch) is at or before it.
__device__ __forceinline__ int candidate_of(const EvCand* __restrict__ cands, int ncand, int cta, bool joint) {
    int lo = 0, hi = ncand - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if ((joint ? cands[mid].cta0j : cands[mid].cta0) <= cta)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// The candidate's prefix rows for this CTA: bulk-copied into shared memory
// when the candidate is staged, else the global rows. ok = false when the
// copy did not land within the bound (the fault word is set).
__device__ __forceinline__ const double* stage_rows(const EvCand& C, double* smem, uint64_t* bar, uint32_t* fault,
                                                    bool& ok) {
    ok = true;
    if (!C.stage) return C.cum;
    const uint32_t b = smem_addr(bar);
    if (threadIdx.x == 0) {
        mbar_init(b, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const uint32_t bytes = 3u * (uint32_t)(2 * C.nb + 2) * (uint32_t)sizeof(double);
    if (threadIdx.x == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(b, bytes);
        bulk_load(smem_addr(smem), C.cum, bytes, b);
    }
    const bool landed = mbar_wait_bounded(b, 0);
    if (!__syncthreads_and(landed)) {
        // Thread 0 issued the copy: it waits again (bounded) so that the CTA
        // does not end with the copy still writing its shared memory.
        if (threadIdx.x == 0) {
            for (int again = 0; again < 16; again++)
                if (mbar_wait_bounded(b, 0)) break;
            atomicOr(fault, 1u);
        }
        ok = false;
    }
    return smem;
}

// ---------------------------------------------------------------------------
// Kernels.

// Exclusive prefix of every candidate's three fields over 2 nb bins
// (evidence.rs:96-144: per segment of 256 bins a Hillis-Steele scan with
// strides 1 .. 128, plus the running carry; that association fixes the
// values' last bits, which the interval sums inherit). CTA (candidate, field).
__global__ void __launch_bounds__(256) k_ev_prefix(const EvCand* __restrict__ cands) {
    __shared__ double x[2][256];
    const EvCand& C = cands[blockIdx.x / 3];
    const int f = blockIdx.x % 3, t = threadIdx.x;
    const int nb2 = 2 * C.nb, rs = nb2 + 2;
    const double* h = C.hist + (size_t)f * nb2;
    double* out = C.cum + (size_t)f * rs;
    if (t == 0) {
        out[0] = 0.0;
        out[nb2 + 1] = 0.0;  // the row's padding slot, copied with the rows
    }
    double carry = 0.0;
    for (int seg = 0; seg < nb2; seg += 256) {
        const int b = seg + t;
        int cur = 0;
        x[0][t] = b < nb2 ? h[b] : 0.0;
        __syncthreads();
        for (int s = 1; s < 256; s <<= 1) {
            x[cur ^ 1][t] = t >= s ? __dadd_rn(x[cur][t], x[cur][t - s]) : x[cur][t];
            __syncthreads();
            cur ^= 1;
        }
        if (b < nb2) out[b + 1] = __dadd_rn(x[cur][t], carry);
        carry = __dadd_rn(carry, x[cur][255]);
        __syncthreads();
    }
}

// Screen (evidence.rs:151-273), which also writes the moment table: for
// every step (duration, shape) whose raw width is in range, the staircase's
// v sum, w sum and norm of the template starting at each of the 2 nb bins
// (lane j writes bins j and j + nb). The joint pass reads its templates and
// their quarter-phase secondaries (the same width, shifted) from it. Then
// per tile the maximum score over its usable templates, and for the tile's
// best template by merit (0.5 score^2 + log masses; the first lane and first
// template on ties) the planet and binary evidence lower bounds and its key.
// A tile without a usable template records zeros.
__global__ void __launch_bounds__(EV_THREADS, 1) k_ev_screen(const EvCand* __restrict__ cands, int ncand, EvConst K,
                                                             uint32_t* fault) {
    extern __shared__ __align__(128) double ev_rows[];
    __shared__ double slot[2][EV_CTA_TILES][2][4];
    __shared__ __align__(8) uint64_t bar;
    const EvCand& C = cands[candidate_of(cands, ncand, blockIdx.x, false)];
    bool ok;
    const double* cum = stage_rows(C, ev_rows, &bar, fault, ok);
    if (!ok) return;
    const int tl = threadIdx.x >> 6, lane = threadIdx.x & 63;
    const int tile = ((int)blockIdx.x - C.cta0) * EV_CTA_TILES + tl;
    if (tile >= C.tiles) return;
    TileRed red{slot, tl, (int)((threadIdx.x >> 5) & 1), 1 + tl, 0};
    const int nb = C.nb, nb2 = 2 * nb, rs = nb2 + 2;
    const int j = tile * EV_TILE + lane;
    const bool jv = j < nb;
    const int jj = jv ? j : nb - 1;
    const double c = C.c;

    double best = neg_inf(), bound = neg_inf();
    double best_a = 0.0, best_q = 1.0, best_null = 0.0, best_ps = 0.0, best_bs = 0.0;
    unsigned long long best_key = 0;
    for (int di = 0; di < C.nd; di++) {
        const EvDur D = C.dur[di];
        if (!D.raw_ok) continue;  // no template of this duration is usable
        const bool usable = usable_at(C, cum, rs, jj, jv, di);
        for (int si = 0; si < C.ns; si++) {
            const Sums m = staircase(cum, rs, nb2, jj, jj + nb, C.lay + ((size_t)di * C.ns + si) * C.L, C.L);
            if (jv) {  // the moment table: this template's sums at bins j and j + nb
                double* t = C.mom + (size_t)(di * C.ns + si) * 3 * nb2;
                t[j] = m.a0;
                t[j + nb] = m.a1;
                t[nb2 + j] = m.w0;
                t[nb2 + j + nb] = m.w1;
                t[2 * (size_t)nb2 + j] = m.q0;
                t[2 * (size_t)nb2 + j + nb] = m.q1;
            }
            const double a = m.a0 + m.a1;
            const double qe = m.q0 - m.w0 * m.w0 / c, qo = m.q1 - m.w1 * m.w1 / c, qeo = -m.w0 * m.w1 / c;
            const double q = qe + qo + 2.0 * qeo;
            const double score = a / sqrt(rmax(q * D.rho2, 1e-300));
            const bool score_valid = usable && a > 0.0 && q > 0.0;
            const double merit = 0.5 * score * score + D.dlm + C.priors[2 * si];
            if (score_valid && merit > bound) {
                best_a = a / D.rho2;
                best_q = q / D.rho2;
                best_null = D.dlm;
                best_ps = C.priors[2 * si];
                best_bs = C.priors[2 * si + 1];
                best_key = (unsigned long long)(si * C.nd + di) * (unsigned long long)nb + (unsigned long long)jj;
                bound = merit;
            }
            if (score_valid && score > best) best = score;
        }
    }
    const double tile_best = red.max1(best);
    // The tile's best merit, lowest lane first.
    double bm = bound;
    int bl = lane;
    for (int off = 16; off > 0; off >>= 1) {
        const double om = __shfl_xor_sync(0xffffffffu, bm, off);
        const int ol = __shfl_xor_sync(0xffffffffu, bl, off);
        if (om > bm || (om == bm && ol < bl)) {
            bm = om;
            bl = ol;
        }
    }
    double mine[2] = {bm, (double)bl}, other[2];
    red.exchange(mine, 2, other);
    if (other[0] > bm || (other[0] == bm && (int)other[1] < bl)) {
        bm = other[0];
        bl = (int)other[1];
    }
    double* out = C.screen + (size_t)tile * EV_SCREEN;
    if (!(bm > neg_inf())) {
        if (lane == 0) out[0] = out[1] = out[2] = out[3] = 0.0;
        return;
    }
    if (lane == bl) {
        const double lower_p =
            positive_amplitude_evidence(best_a, best_q, K.tau_p) + K.ln_screen_p + best_null + best_ps;
        const double lower_b = log_add(positive_amplitude_evidence(best_a, best_q, K.tau_b),
                                       positive_amplitude_evidence(best_a, best_q, K.tau_d)) +
                               K.ln_screen_b + best_null + best_bs;
        out[0] = tile_best;
        out[1] = lower_p;
        out[2] = lower_b;
        out[3] = (double)best_key;
    }
}

// Pilot, one warp per candidate (evidence.rs:834-875): the screen maximum
// against the threshold (below it the candidate is inactive: no rows), the
// winner tile (largest planet bound, the last on ties), its template
// evaluated without pruning, and the floors of the joint pass.
__global__ void __launch_bounds__(128) k_ev_pilot(const EvCand* __restrict__ cands, int ncand, EvConst K) {
    const int ci = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (ci >= ncand) return;
    const EvCand& C = cands[ci];
    const int lane = threadIdx.x & 31;
    double mx = neg_inf(), bv = neg_inf();
    int bt = -1;
    for (int t = lane; t < C.tiles; t += 32) {
        const double* s = C.screen + (size_t)t * EV_SCREEN;
        mx = rmax(mx, s[0]);
        if (s[1] > bv || (s[1] == bv && t > bt)) {
            bv = s[1];
            bt = t;
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        mx = rmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
        const int ot = __shfl_xor_sync(0xffffffffu, bt, off);
        if (ov > bv || (ov == bv && ot > bt)) {
            bv = ov;
            bt = ot;
        }
    }
    if (lane != 0) return;
    if (bt < 0) bt = 0;
    double* P = C.pilot;
    const bool active = mx >= C.threshold * (1.0 - 1e-12);
    const double key = C.screen[(size_t)bt * EV_SCREEN + 3];
    P[2] = key;
    P[3] = active ? 1.0 : 0.0;
    P[4] = mx;
    P[5] = (double)bt;
    P[0] = P[1] = neg_inf();
    if (!active) return;
    const unsigned long long pk = key > 0.0 ? (unsigned long long)key : 0ull;
    const unsigned long long nbu = (unsigned long long)C.nb, ndu = (unsigned long long)C.nd;
    const int jj = (int)(pk % nbu), di = (int)((pk / nbu) % ndu), si = (int)(pk / (nbu * ndu));
    Lane S;
    lane_init(S);
    if (si < C.ns && C.dur[di].raw_ok) {
        const int rs = 2 * C.nb + 2;
        const bool usable = usable_at(C, C.cum, rs, jj, true, di);
        const Eval e = joint_template(C, K, C.cum, rs, jj, true, di, si, neg_inf(), neg_inf(), usable, OwnDecide{});
        lane_add(C, S, e, true, jj, di, si);
    }
    // The pilot tile's log sums: 64 equal terms.
    const double sp = S.sum_p > neg_inf() ? S.sum_p + K.ln_tile : neg_inf();
    const double sb = S.sum_b > neg_inf() ? S.sum_b + K.ln_tile : neg_inf();
    P[0] = sp + C.margin;
    P[1] = sb + C.margin;
}

// Joint tiles (evidence.rs:280-632): every template of the tile's phases,
// pruned against the pilot's floors; per tile the winners by joint evidence
// and by amplitude (largest value, lowest key) with their values, and the
// tile's log sums of planet and binary evidence.
__global__ void __launch_bounds__(EV_THREADS, 1) k_ev_joint(const EvCand* __restrict__ cands, int ncand, EvConst K) {
    __shared__ double slot[2][EV_CTA_TILES][2][4];
    __shared__ uint8_t decisions[EV_CTA_TILES][MAX_DURATIONS * MAX_SHAPES];
    const EvCand& C = cands[candidate_of(cands, ncand, blockIdx.x, true)];
    if (C.pilot[3] == 0.0) return;  // inactive candidate (uniform over the CTA)
    const double floor_p = C.pilot[0], floor_b = C.pilot[1];
    const double* cum = C.cum;  // the count row only (the sums come from the moment table)
    const int tl = threadIdx.x >> 6, lane = threadIdx.x & 63;
    // CTA (tile group, part): the part's durations of the group's tiles.
    const int local = (int)blockIdx.x - C.cta0j;
    const int part = local % C.parts;
    const int tile = (local / C.parts) * EV_CTA_TILES + tl;
    if (tile >= C.tiles) return;
    const int di0 = part * C.nd / C.parts, di1 = (part + 1) * C.nd / C.parts;
    TileRed red{slot, tl, (int)((threadIdx.x >> 5) & 1), 1 + tl, 0};
    const int nb = C.nb, rs = 2 * nb + 2;
    const int j = tile * EV_TILE + lane;
    const bool jv = j < nb;
    const int jj = jv ? j : nb - 1;

    Lane S;
    lane_init(S);
    const TileDecide decide{&red, decisions[tl], lane};
    for (int di = di0; di < di1; di++) {
        if (!C.dur[di].raw_ok) continue;  // uniform: no template of this duration enters the sums
        const bool usable = usable_at(C, cum, rs, jj, jv, di);
        for (int si = 0; si < C.ns; si++) {
            const Eval e = joint_template(C, K, cum, rs, jj, jv, di, si, floor_p, floor_b, usable, decide);
            lane_add(C, S, e, jv, jj, di, si);
        }
    }

    // One record per (tile, part): the winners and log sums of the part's
    // templates. The host takes the best record by (value, lowest key) and
    // log-sum-exps all records, which is the whole tile's result.
    double* rec = C.rec + ((size_t)tile * C.parts + part) * EV_REC;
    for (int sel = 0; sel < 2; sel++) {
        const double m = sel ? S.best_signal : S.best_joint;
        const unsigned long long key = sel ? S.signal_key : S.joint_key;
        double bm = m;
        unsigned long long bk = key;
        for (int off = 16; off > 0; off >>= 1) {
            const double om = __shfl_xor_sync(0xffffffffu, bm, off);
            const unsigned long long ok2 = __shfl_xor_sync(0xffffffffu, bk, off);
            if (om > bm || (om == bm && ok2 < bk)) {
                bm = om;
                bk = ok2;
            }
        }
        double mine[2] = {bm, __longlong_as_double((long long)bk)}, other[2];
        red.exchange(mine, 2, other);
        const unsigned long long obk = (unsigned long long)__double_as_longlong(other[1]);
        if (other[0] > bm || (other[0] == bm && obk < bk)) {
            bm = other[0];
            bk = obk;
        }
        // The lane holding the winner writes; without any key (no valid
        // template in the tile) the last lane does, as the reference's
        // fallback index does.
        const bool writer = bk == KEY_MAX ? lane == EV_TILE - 1 : (key == bk && m == bm);
        if (writer) {
            double* o = rec + sel * 10;
            o[0] = (double)bk;
            o[1] = bm;
            if (bk == KEY_MAX) {  // no valid template: zero values (the row is never reported)
                o[2] = sel ? S.best_signal : 0.0;
                for (int i = 3; i < 10; i++) o[i] = 0.0;
            } else {
                // Replay the winning template with the tile's recorded decisions.
                const int wj = (int)(bk % (unsigned long long)nb);
                const int wd = (int)((bk / (unsigned long long)nb) % (unsigned long long)C.nd);
                const int ws = (int)(bk / ((unsigned long long)nb * (unsigned long long)C.nd));
                const bool usable = usable_at(C, cum, rs, wj, true, wd);
                const Eval e = joint_template(C, K, cum, rs, wj, true, wd, ws, floor_p, floor_b, usable,
                                              ReplayDecide{decisions[tl][wd * C.ns + ws]});
                o[2] = sel ? S.best_signal : e.snr;
                o[3] = e.depth;
                o[4] = e.sec_ratio;
                o[5] = e.sec_phase;
                o[6] = e.odd_ratio;
                o[7] = e.binary_multiple;
                o[8] = e.lp;
                o[9] = e.lb;
            }
        }
    }
    for (int sel = 0; sel < 2; sel++) {
        const double s = sel ? S.sum_b : S.sum_p;
        const double high = red.max1(s);
        double log_sum = high;
        if (high > neg_inf()) log_sum = high + log(red.sum1(exp(s - high)));
        if (lane == 0) rec[20 + sel] = log_sum;
    }
}

// ---------------------------------------------------------------------------
// Host side of compare_search (evidence.rs:693-1003), batched.

double host_logsumexp(const std::vector<double>& v) {
    double high = neg_inf();
    for (double x : v) high = rmax(high, x);
    if (high == neg_inf()) return high;
    double s = 0.0;
    for (double x : v) s += std::exp(x - high);
    return high + std::log(s);
}

// Everything the device needs about one candidate, in host memory.
struct Plan {
    bool run = false;  // false: no rows (no duration below period / 4) or rejected (status set)
    int nb = 0, nd = 0, ns = 0, L = 0, tiles = 0, cls = 0, parts = 1;
    double scale = 0.0, margin = 0.0, log_mass = 0.0;
    std::vector<double> durations, priors;
    std::vector<EvDur> dur;
    std::vector<EvLayer> lay;
    std::vector<EvOrbit> orb;
    FoldShape shape{};
    std::vector<int> chunks;
    int nchunks = 0;
    // workspace offsets (bytes)
    size_t o_dur = 0, o_lay = 0, o_orb = 0, o_mom = 0, o_pri = 0, o_scale = 0, o_chunks = 0, o_hist = 0,
           o_fscratch = 0, o_cum = 0, o_screen = 0, o_rec = 0, o_pilot = 0;
};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

constexpr size_t EV_STAGE_MAX = 200 * 1024;  // prefix rows staged in shared memory up to this size
// Launch classes by staged bytes: each class launches with its own dynamic
// shared memory, so small candidates keep several CTAs per SM.
constexpr size_t EV_CLASS_BYTES[3] = {48 * 1024, 100 * 1024, EV_STAGE_MAX};

int plan_candidate(const EvidenceCandidate& E, const fbls_config& cfg, int sm_count, Plan& P, std::string& message) {
    std::vector<std::pair<double, double>> ds;
    for (uint32_t i = 0; i < E.nd; i++)
        if (E.durations[i] < E.period / 4.0) ds.push_back({E.durations[i], E.rho[i]});
    std::stable_sort(ds.begin(), ds.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    if (ds.empty()) return 0;  // no rows
    const int nd = (int)ds.size(), ns = (int)cfg.n_ingress, L = (int)cfg.shape_layers;
    if (ns < 1 || ns > MAX_SHAPES || L < 1 || L > MAX_LAYERS || nd > MAX_DURATIONS) {
        message = "invalid shape bank";
        return FBLS_ERR_ARGUMENT;
    }
    const double dmin = ds[0].first;
    uint64_t nb = 4 * as_u64(std::ceil((double)cfg.phase_oversample * E.period / dmin / 4.0));
    if (nb < 8) nb = 8;
    const uint64_t nb2 = 2 * nb;
    if (nb2 > (1ull << 26)) {
        message = "evidence phase grid too large";
        return FBLS_ERR_ARGUMENT;
    }
    const double scale = (double)nb / E.period;
    if (!(std::floor(E.r.t_last * scale) < 4294967295.0 - 2.0 * (double)nb2 - 2.0)) {
        message = "phase cell exceeds 32 bits";
        return FBLS_ERR_ARGUMENT;
    }
    P.nb = (int)nb;
    P.nd = nd;
    P.ns = ns;
    P.L = L;
    P.scale = scale;
    P.tiles = (int)((nb + EV_TILE - 1) / EV_TILE);
    const double n = (double)E.r.n;
    // Duration log masses (evidence.rs:720-726), shape priors (:728-738).
    std::vector<double> dlm(nd);
    for (int i = 0; i < nd; i++) {
        const double rr = ds[i].second;
        dlm[i] = -0.5 * ((n - 1.0) * std::log(rr * rr) + E.r.residual_energy / (rr * rr));
    }
    double dmax = neg_inf();
    for (double x : dlm) dmax = rmax(dmax, x);
    for (double& x : dlm) x -= dmax;
    std::vector<double> lpl(ns), lbl(ns);
    for (int s = 0; s < ns; s++) {
        lpl[s] = -4.0 * cfg.ingress_fractions[s];
        lbl[s] = 2.0 * cfg.ingress_fractions[s];
    }
    const double lp0 = host_logsumexp(lpl), lb0 = host_logsumexp(lbl);
    P.priors.resize(2 * ns);
    for (int s = 0; s < ns; s++) {
        P.priors[2 * s] = lpl[s] - lp0;
        P.priors[2 * s + 1] = lbl[s] - lb0;
    }
    // Staircase layers (evidence.rs:739-747): fraction of the width, the
    // layer's increment (weight of its sums) and squared-sum coefficient.
    std::vector<double> frac((size_t)ns * L), inc((size_t)ns * L), sq((size_t)ns * L);
    for (int s = 0; s < ns; s++) {
        double previous = 0.0;
        for (int l = 0; l < L; l++) {
            const double a = 1.0 / (double)L;
            frac[(size_t)s * L + l] = 1.0 - 2.0 * cfg.ingress_fractions[s] * (double)l / (double)(std::max(L, 2) - 1);
            inc[(size_t)s * L + l] = a;
            sq[(size_t)s * L + l] = a * (2.0 * previous + a);
            previous += a;
        }
    }
    auto layers_at = [&](uint64_t width, std::vector<EvLayer>& out) {
        for (int s = 0; s < ns; s++)
            for (int l = 0; l < L; l++) {
                uint64_t inner = as_u64(std::floor((double)width * frac[(size_t)s * L + l] + 0.5));
                if (inner < 1) inner = 1;
                if (inner > width) inner = width;  // fractions are at most 1
                out.push_back({(int)((width - inner) / 2), (int)inner, inc[(size_t)s * L + l], sq[(size_t)s * L + l]});
            }
    };
    // Orbit bank (evidence.rs:751-789): secondary phases 0.25, 0.5, 0.75 with
    // masses 0.1, 0.8, 0.1, kept where the secondary fits inside the cycle.
    const double phases[NORB] = {0.25, 0.5, 0.75};
    const double logw[NORB] = {std::log(0.1), std::log(0.8), std::log(0.1)};
    std::vector<double> lp_bank((size_t)nd * NORB, neg_inf()), lb_bank((size_t)nd * NORB, neg_inf());
    size_t valid_count = 0;
    for (int di = 0; di < nd; di++) {
        const double k = rmax(std::floor(ds[di].first * scale + 0.5), 1.0);
        if (k < (double)(nb / 4)) valid_count++;
        for (int o = 0; o < NORB; o++) {
            const double ks = rmax(std::floor(k + 0.5), 1.0);
            const double shift = std::floor(phases[o] * (double)nb + 0.5);
            const double start = shift + std::floor((k - ks) / 2.0);
            if (k < (double)(nb / 4) && ks < (double)(nb / 2) && start >= k && start + ks <= (double)nb)
                lp_bank[(size_t)di * NORB + o] = lb_bank[(size_t)di * NORB + o] = logw[o];
        }
    }
    const double lcount = std::log((double)valid_count);
    const double norm_p = lcount - host_logsumexp(lp_bank), norm_b = lcount - host_logsumexp(lb_bank);
    int64_t max_start = 0;
    for (int di = 0; di < nd; di++) {
        const uint64_t raw_k = template_width(ds[di].first, scale);
        const uint64_t k = std::min<uint64_t>(raw_k, nb2 / 8 - 1);
        const double rr = ds[di].second;
        P.dur.push_back({rr * rr, dlm[di], (int)k, raw_k < nb2 / 8 ? 1 : 0});
        layers_at(k, P.lay);
        for (int o = 0; o < NORB; o++) {
            const double duration_ratio = 1.0;  // the bank without extended physics
            const int64_t offset = (int64_t)std::floor(phases[o] * (double)nb + 0.5);
            int64_t sk = (int64_t)std::floor((double)k * duration_ratio + 0.5);
            sk = std::min<int64_t>(std::max<int64_t>(sk, 1), (int64_t)nb - 1);
            const int64_t shift = offset + (int64_t)std::floor(((double)k - (double)sk) / 2.0);
            // The secondary has the primary's width (ratio 1), so its sums are
            // rows of the primary's moment table, shift bins further on.
            if (shift < 0 || sk != (int64_t)k || shift >= (int64_t)nb2) {
                message = "evidence orbit bank outside the cycle";
                return FBLS_ERR_ARGUMENT;
            }
            P.orb.push_back({(int)shift, 0, phases[o], lp_bank[(size_t)di * NORB + o] + norm_p,
                             lb_bank[(size_t)di * NORB + o] + norm_b});
            max_start = std::max<int64_t>(max_start, shift + (int64_t)sk);
        }
        max_start = std::max<int64_t>(max_start, (int64_t)k);
    }
    // Interval starts stay below 2 nb2: phase < nb, plus nb for the odd
    // cycle, plus the largest shift and layer offset.
    if ((int64_t)nb - 1 + (int64_t)nb + max_start >= 2 * (int64_t)nb2) {
        message = "evidence interval beyond two cycles";
        return FBLS_ERR_ARGUMENT;
    }
    std::vector<double> in_bank;
    for (int i = 0; i < nd; i++)
        if (rmax(std::floor(ds[i].first * scale + 0.5), 1.0) < (double)(nb / 4)) in_bank.push_back(dlm[i]);
    P.log_mass = std::log((double)nb) + host_logsumexp(in_bank);
    P.margin = cfg.evidence_rtol > 0.0
                   ? std::log(cfg.evidence_rtol) - std::log((double)((NORB + 1) * nb * (uint64_t)nd * ns))
                   : neg_inf();
    P.durations.resize(nd);
    for (int i = 0; i < nd; i++) P.durations[i] = ds[i].first;
    // Fold of two periods: one period at scale nb / P into 2 nb bins.
    P.shape = fold_group_shape((int)nb2, 1, sm_count);
    P.chunks.resize((size_t)E.r.n + 2);
    P.nchunks = fold_chunks(E.r.time_host, (int)E.r.n, scale, (int)nb2, P.shape.span_cap, P.shape.chunk_cap,
                            P.chunks.data(), (int)P.chunks.size());
    if (P.nchunks < 1) {
        message = "fold chunking failed";
        return FBLS_ERR_ARGUMENT;
    }
    const size_t stage_bytes = 3 * (nb2 + 2) * sizeof(double);
    P.cls = 3;  // rows read from global memory
    for (int k = 0; k < 3; k++)
        if (stage_bytes <= EV_CLASS_BYTES[k]) {
            P.cls = k;
            break;
        }
    P.run = true;
    return 0;
}

}  // namespace

void evidence_parameters(const fbls_config& cfg, double* p) {
    const double dilution = cfg.target_flux_fraction;
    double planet_scale = cfg.planet_depth_scale;
    if (!std::isnan(cfg.stellar_radius_solar)) {
        double x = 0.10045 * cfg.planet_radius_scale_rj / cfg.stellar_radius_solar;
        planet_scale = x * x;
    }
    p[0] = planet_scale * dilution;
    p[1] = cfg.binary_depth_scale * dilution;
    p[2] = cfg.diluted_binary_depth_scale;
    p[3] = std::log(cfg.planet_prior);
    p[4] = std::log(cfg.binary_prior);
    p[5] = std::log(1.0 - cfg.planet_prior - cfg.binary_prior);
    const double ratios[5] = {0.0, 0.01, 0.1, 0.5, 1.0};
    const double wp[5] = {0.75, 0.15, 0.08, 0.015, 0.005};
    const double wb[5] = {0.10, 0.10, 0.20, 0.25, 0.35};
    for (int i = 0; i < 5; i++) {
        p[6 + 3 * i] = ratios[i];
        p[7 + 3 * i] = wp[i];
        p[8 + 3 * i] = wb[i];
    }
    const double odd[7] = {0.25, 0.5, 0.75, 1.0, 4.0 / 3.0, 2.0, 4.0};
    for (int i = 0; i < 7; i++) p[21 + i] = odd[i];
    p[28] = 0.001;
    p[29] = 0.05;
}

int compare_batch(cudaStream_t stream, EvidenceCandidate* cands, size_t count, const fbls_config& cfg,
                  std::string& message, const std::function<void*(size_t)>& workspace, int sm_count,
                  uint64_t* launches) {
    for (size_t i = 0; i < count; i++) {
        cands[i].n_rows = 0;
        cands[i].status = 0;
        cands[i].message.clear();
    }
    if (count == 0) return 0;
    if (cfg.n_ingress < 1 || !cfg.ingress_fractions) {
        message = "invalid shape bank";
        return FBLS_ERR_ARGUMENT;
    }
    double params[NPARAM];
    evidence_parameters(cfg, params);
    EvConst K{};
    K.tau_p = params[0];
    K.tau_b = params[1];
    K.tau_d = params[2];
    for (int i = 0; i < EV_NRATIO; i++) {
        K.ratio_p[i] = params[6 + 3 * i];
        K.lnw_p[i] = std::log(params[7 + 3 * i]);
        K.lnw_b[i] = std::log(0.25 * params[8 + 3 * i]);
    }
    for (int i = 0; i < EV_NODD; i++) K.ratio_o[i] = params[21 + i];
    K.ln_odd = std::log(0.25 / 7.0);
    K.ln_screen_p = std::log(0.75);
    K.ln_screen_b = std::log(0.025);
    K.ln_tile = std::log((double)EV_TILE);

    std::vector<Plan> plans(count);
    for (size_t i = 0; i < count; i++) {
        EvidenceCandidate& E = cands[i];
        if (!E.durations || !E.rho || !E.r.time || !E.r.time_host || E.r.n < 6 || !(E.period > 0.0) ||
            !std::isfinite(E.period)) {
            E.status = FBLS_ERR_ARGUMENT;
            E.message = "bad candidate (null arrays, fewer than six observations or a nonpositive period)";
            continue;
        }
        E.status = plan_candidate(E, cfg, sm_count, plans[i], E.message);
    }
    // Candidates that run, ordered by launch class.
    std::vector<size_t> order;
    for (int cls = 0; cls < 4; cls++)
        for (size_t i = 0; i < count; i++)
            if (plans[i].run && plans[i].cls == cls) order.push_back(i);
    if (order.empty()) return 0;
    const size_t R = order.size();
    // Parts of the joint pass: enough (tile group, part) CTAs for about two
    // per SM, at most 8 parts and one duration per part.
    {
        size_t groups = 0;
        for (size_t i : order) groups += (size_t)(plans[i].tiles + EV_CTA_TILES - 1) / EV_CTA_TILES;
        const int target = (int)std::min<size_t>(8, (2 * (size_t)std::max(sm_count, 1) + groups - 1) / groups);
        for (size_t i : order) plans[i].parts = std::max(1, std::min(target, plans[i].nd));
    }

    // Workspace layout: [EvCand x R | fold jobs | cta0 | per-candidate tables,
    // scale, chunks] uploaded; then hist, fold scratch, cum, screen, rec,
    // pilot and the fault word, written on the device.
    size_t at = 0;
    auto take = [&](size_t bytes) {
        const size_t o = at;
        at += align256(bytes);
        return o;
    };
    const size_t o_cands = take(R * sizeof(EvCand));
    const size_t o_jobs = take(R * sizeof(FoldArgs));
    const size_t o_cta0 = take((R + 1) * sizeof(int));
    for (size_t r = 0; r < R; r++) {
        Plan& P = plans[order[r]];
        P.o_dur = take(P.dur.size() * sizeof(EvDur));
        P.o_lay = take(P.lay.size() * sizeof(EvLayer));
        P.o_orb = take(P.orb.size() * sizeof(EvOrbit));
        P.o_pri = take(P.priors.size() * sizeof(double));
        P.o_scale = take(sizeof(double));
        P.o_chunks = take(((size_t)P.nchunks + 1) * sizeof(int));
    }
    const size_t upload_bytes = at;
    for (size_t r = 0; r < R; r++) {
        Plan& P = plans[order[r]];
        const size_t nb2 = 2 * (size_t)P.nb;
        P.o_hist = take(3 * nb2 * sizeof(double));
        P.o_fscratch = P.shape.hist_in_smem ? 0 : take(3 * (size_t)P.shape.row_stride * sizeof(double));
        P.o_cum = take(3 * (nb2 + 2) * sizeof(double));
        P.o_mom = take((size_t)P.nd * P.ns * 3 * nb2 * sizeof(double));
        P.o_screen = take((size_t)P.tiles * EV_SCREEN * sizeof(double));
    }
    // What comes back to the host, in one contiguous region.
    const size_t o_first = at;
    for (size_t r = 0; r < R; r++) {
        Plan& P = plans[order[r]];
        P.o_rec = take((size_t)P.tiles * P.parts * EV_REC * sizeof(double));
        P.o_pilot = take(EV_PILOT * sizeof(double));
    }
    const size_t o_fault = take(sizeof(uint32_t));
    const size_t total = at;
    unsigned char* ws = static_cast<unsigned char*>(workspace(total));
    if (!ws) {
        message = "evidence workspace allocation failed";
        return FBLS_ERR_CUDA;
    }

    std::vector<unsigned char> blob(upload_bytes, 0);
    auto put = [&](size_t off, const void* src, size_t bytes) {
        if (bytes) std::memcpy(blob.data() + off, src, bytes);
    };
    EvCand* hc = reinterpret_cast<EvCand*>(blob.data() + o_cands);
    FoldArgs* hj = reinterpret_cast<FoldArgs*>(blob.data() + o_jobs);
    int* h_cta0 = reinterpret_cast<int*>(blob.data() + o_cta0);
    for (size_t r = 0; r <= R; r++) h_cta0[r] = (int)r;
    // CTA numbering of the screen and joint launches restarts in each class.
    int cls_first[5] = {0, 0, 0, 0, 0};
    {
        int cls_prev = -1, cta = 0, ctaj = 0;
        for (size_t r = 0; r < R; r++) {
            const Plan& P = plans[order[r]];
            if (P.cls != cls_prev) {
                for (int k = cls_prev + 1; k <= P.cls; k++) cls_first[k] = (int)r;
                cls_prev = P.cls;
                cta = ctaj = 0;
            }
            hc[r].cta0 = cta;
            hc[r].cta0j = ctaj;
            hc[r].parts = P.parts;
            cta += (P.tiles + EV_CTA_TILES - 1) / EV_CTA_TILES;
            ctaj += (P.tiles + EV_CTA_TILES - 1) / EV_CTA_TILES * P.parts;
        }
        for (int k = cls_prev + 1; k <= 4; k++) cls_first[k] = (int)R;
    }
    for (size_t r = 0; r < R; r++) {
        const size_t i = order[r];
        const Plan& P = plans[i];
        const EvidenceCandidate& E = cands[i];
        put(P.o_dur, P.dur.data(), P.dur.size() * sizeof(EvDur));
        put(P.o_lay, P.lay.data(), P.lay.size() * sizeof(EvLayer));
        put(P.o_orb, P.orb.data(), P.orb.size() * sizeof(EvOrbit));
        put(P.o_pri, P.priors.data(), P.priors.size() * sizeof(double));
        put(P.o_scale, &P.scale, sizeof(double));
        put(P.o_chunks, P.chunks.data(), ((size_t)P.nchunks + 1) * sizeof(int));
        EvCand& c = hc[r];
        c.hist = reinterpret_cast<const double*>(ws + P.o_hist);
        c.cum = reinterpret_cast<double*>(ws + P.o_cum);
        c.screen = reinterpret_cast<double*>(ws + P.o_screen);
        c.rec = reinterpret_cast<double*>(ws + P.o_rec);
        c.pilot = reinterpret_cast<double*>(ws + P.o_pilot);
        c.dur = reinterpret_cast<const EvDur*>(ws + P.o_dur);
        c.lay = reinterpret_cast<const EvLayer*>(ws + P.o_lay);
        c.orb = reinterpret_cast<const EvOrbit*>(ws + P.o_orb);
        c.mom = reinterpret_cast<double*>(ws + P.o_mom);
        c.priors = reinterpret_cast<const double*>(ws + P.o_pri);
        c.c = E.r.baseline_norm;
        c.n = (double)E.r.n;
        c.threshold = cfg.threshold;
        c.margin = P.margin;
        c.nb = P.nb;
        c.nd = P.nd;
        c.ns = P.ns;
        c.L = P.L;
        c.tiles = P.tiles;
        c.stage = P.cls < 3 ? 1 : 0;
        // fold_two (evidence.rs:75-92) on the fold kernels: one period at
        // scale nb / P into 2 nb bins, the raw histogram out.
        FoldArgs& fa = hj[r];
        fa.time = E.r.time;
        fa.v = E.r.v;
        fa.w = E.r.w;
        fa.scales = reinterpret_cast<const double*>(ws + P.o_scale);
        fa.n = (int)E.r.n;
        fa.nb = 2 * P.nb;
        fa.periods = 1;
        fa.group = 1;
        fa.hist_global = P.shape.hist_in_smem ? nullptr : reinterpret_cast<double*>(ws + P.o_fscratch);
        fa.hist_out = reinterpret_cast<double*>(ws + P.o_hist);
        fa.chunks = reinterpret_cast<const int*>(ws + P.o_chunks);
        fa.nchunks = P.nchunks;
        fa.stage_field = P.shape.stage_field;
        fa.window = P.shape.window;
        fa.row_stride = P.shape.row_stride;
        fa.fault = reinterpret_cast<uint32_t*>(ws + o_fault);
    }
    auto check = [&](cudaError_t e, const char* where) {
        if (e != cudaSuccess) message = std::string(where) + ": " + cudaGetErrorString(e);
        return e == cudaSuccess;
    };
    auto counted = [&](cudaError_t e, const char* where) {
        if (launches && e == cudaSuccess) (*launches)++;
        return check(e, where);
    };
    if (!check(cudaMemcpyAsync(ws, blob.data(), upload_bytes, cudaMemcpyHostToDevice, stream), "evidence upload") ||
        !check(cudaMemsetAsync(ws + o_fault, 0, sizeof(uint32_t), stream), "evidence fault word"))
        return FBLS_ERR_CUDA;

    // Folds: one job launch per fold kind (and CTA size); a job is one CTA.
    {
        const FoldArgs* d_jobs = reinterpret_cast<const FoldArgs*>(ws + o_jobs);
        const int* d_cta0 = reinterpret_cast<const int*>(ws + o_cta0);
        // A launch covers a run of consecutive candidates (in `order`) with
        // the same fold kind and CTA size; a job is one CTA, so job j of any
        // launch starts at CTA j (the table h_cta0 holds 0, 1, 2, ...).
        size_t r = 0;
        while (r < R) {
            const FoldShape& s0 = plans[order[r]].shape;
            size_t e = r + 1;
            size_t smem = s0.smem;
            while (e < R && plans[order[e]].shape.kind == s0.kind && plans[order[e]].shape.threads == s0.threads) {
                smem = std::max(smem, plans[order[e]].shape.smem);
                e++;
            }
            for (size_t q = r; q < e; q++) {
                const FoldArgs& a = hj[q];
                const FoldShape& sh = plans[order[q]].shape;
                if (!(s0.kind == FOLD_WALK ? fold_job_ok(a, sh) : fold_smem_job_ok(a, sh))) {
                    message = "evidence fold outside the fold kernels' limits";
                    return FBLS_ERR_ARGUMENT;
                }
            }
            const int njobs = (int)(e - r);
            cudaError_t err;
            if (s0.kind == FOLD_WALK)
                err = launch_fold_jobs(d_jobs + r, d_cta0, njobs, njobs, s0.threads, false, smem, stream);
            else
                err = launch_fold_smem_jobs(d_jobs + r, d_cta0, njobs, njobs, s0.threads, smem, stream);
            if (!counted(err, "evidence fold")) return FBLS_ERR_CUDA;
            r = e;
        }
    }
    const EvCand* d_cands = reinterpret_cast<const EvCand*>(ws + o_cands);
    uint32_t* d_fault = reinterpret_cast<uint32_t*>(ws + o_fault);
    k_ev_prefix<<<(unsigned)(3 * R), 256, 0, stream>>>(d_cands);
    if (!counted(cudaGetLastError(), "evidence prefix")) return FBLS_ERR_CUDA;
    auto per_class = [&](bool joint) {
        for (int cls = 0; cls < 4; cls++) {
            const int r0 = cls_first[cls], r1 = cls_first[cls + 1];
            if (r1 <= r0) continue;
            int ctas = 0;
            size_t smem = 0;
            for (int r = r0; r < r1; r++) {
                const Plan& P = plans[order[r]];
                ctas += (P.tiles + EV_CTA_TILES - 1) / EV_CTA_TILES * (joint ? P.parts : 1);
                if (cls < 3) smem = std::max(smem, 3 * (2 * (size_t)P.nb + 2) * sizeof(double));
            }
            if (joint) {
                k_ev_joint<<<ctas, EV_THREADS, 0, stream>>>(d_cands + r0, r1 - r0, K);
            } else {
                if (!check(cudaFuncSetAttribute(k_ev_screen, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)EV_STAGE_MAX),
                           "evidence shared memory"))
                    return false;
                k_ev_screen<<<ctas, EV_THREADS, smem, stream>>>(d_cands + r0, r1 - r0, K, d_fault);
            }
            if (!counted(cudaGetLastError(), joint ? "evidence joint" : "evidence screen")) return false;
        }
        return true;
    };
    if (!per_class(false)) return FBLS_ERR_CUDA;
    k_ev_pilot<<<(unsigned)((R + 3) / 4), 128, 0, stream>>>(d_cands, (int)R, K);
    if (!counted(cudaGetLastError(), "evidence pilot")) return FBLS_ERR_CUDA;
    if (!per_class(true)) return FBLS_ERR_CUDA;

    // Results: every candidate's tile records and pilot word and the fault
    // word, one copy, one synchronisation.
    const size_t down = total - o_first;
    std::vector<unsigned char> host(down);
    if (!check(cudaMemcpyAsync(host.data(), ws + o_first, down, cudaMemcpyDeviceToHost, stream), "evidence download") ||
        !check(cudaStreamSynchronize(stream), "evidence"))
        return FBLS_ERR_CUDA;
    uint32_t fault = 0;
    std::memcpy(&fault, host.data() + (o_fault - o_first), sizeof(uint32_t));
    if (fault) {
        message = "evidence: staging copies did not complete";
        return FBLS_ERR_CUDA;
    }

    for (size_t r = 0; r < R; r++) {
        const size_t i = order[r];
        const Plan& P = plans[i];
        EvidenceCandidate& E = cands[i];
        const double* pil = reinterpret_cast<const double*>(host.data() + (P.o_pilot - o_first));
        if (pil[3] == 0.0) continue;  // below the threshold: no rows
        const double* rec = reinterpret_cast<const double*>(host.data() + (P.o_rec - o_first));
        const int tiles = P.tiles * P.parts;  // records: (tile, part)
        const uint64_t nb = (uint64_t)P.nb;
        fbls_evidence_row rows[2];
        std::vector<double> sp(tiles), sb(tiles);
        for (int t = 0; t < tiles; t++) {
            sp[t] = rec[(size_t)t * EV_REC + 20];
            sb[t] = rec[(size_t)t * EV_REC + 21];
        }
        const double lp = host_logsumexp(sp) - P.log_mass;
        const double lb = host_logsumexp(sb) - P.log_mass;
        const double joint = params[3] + lp - log_add(params[5], params[4] + lb);
        for (int sel = 0; sel < 2; sel++) {
            auto value = [&](int t, int k) { return rec[(size_t)t * EV_REC + sel * 10 + k]; };
            double mx = neg_inf();
            for (int t = 0; t < tiles; t++) mx = rmax(mx, value(t, 1));
            double key = __builtin_huge_val();
            for (int t = 0; t < tiles; t++)
                if (value(t, 1) == mx) key = rmin(key, value(t, 0));
            int tile = 0;
            for (int t = 0; t < tiles; t++)
                if (value(t, 1) == mx && value(t, 0) == key) {
                    tile = t;
                    break;
                }
            const uint64_t decoded = mx > neg_inf() ? as_u64(key) : 0;
            const size_t j = (size_t)(decoded % nb);
            const size_t di = (size_t)((decoded / nb) % (uint64_t)P.nd);
            const size_t si = (size_t)(decoded / (nb * (uint64_t)P.nd));
            const double width = rmax(std::floor(P.durations[di] * P.scale + 0.5), 1.0);
            fbls_evidence_row& row = rows[sel];
            row.period = E.period;
            row.epoch = ((double)j + width / 2.0) / P.scale + E.r.origin;
            row.duration = width / P.scale;
            row.snr = mx > neg_inf() ? value(tile, 2) : neg_inf();
            row.depth = value(tile, 3);
            row.planet_log_odds = joint;
            row.log_bf_planet_noise = lp;
            row.log_bf_binary_noise = lb;
            row.binary_secondary_ratio = value(tile, 4);
            row.binary_secondary_phase = value(tile, 5);
            row.binary_odd_even_ratio = value(tile, 6);
            row.binary_period_days = value(tile, 7) * E.period;
            row.ingress_fraction = cfg.ingress_fractions[std::min(si, (size_t)(P.ns - 1))];
            row.selection_flags = sel == 0 ? 1u : 2u;
        }
        const bool hit0 = std::isfinite(rows[0].snr), hit1 = std::isfinite(rows[1].snr);
        const bool same = hit0 && hit1 && rows[0].period == rows[1].period && rows[0].epoch == rows[1].epoch &&
                          rows[0].duration == rows[1].duration && rows[0].snr == rows[1].snr &&
                          rows[0].depth == rows[1].depth && rows[0].ingress_fraction == rows[1].ingress_fraction;
        uint32_t out = 0;
        if (hit0) {
            E.rows[out] = rows[0];
            if (same) E.rows[out].selection_flags = 3;
            out++;
        }
        if (hit1 && !same) E.rows[out++] = rows[1];
        E.n_rows = out;
    }
    return 0;
}

}  // namespace fbls
