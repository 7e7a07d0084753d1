// Joint planet / binary / noise evidence at one trial period on sm_100a.
// Semantics follow src/search/evidence.rs: the two-period fold keeps cycle
// parity (template at phase j paired with its odd counterpart at j + nb),
// each local model integrates a positive depth with a half-normal prior and
// sums discrete scenario masses (secondary eclipses at quarter phases,
// alternating primaries at twice the period), and the phase / duration /
// shape sums are log-sum-exp'd per tile.
//
// Device work: the two-period fold runs on the deterministic fold kernel
// (fold.cu) with one period and 2 nb bins, k_prefix_fields scans the three
// fields, k_screen and k_joint evaluate one 64-phase tile per CTA.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "evidence.h"
#include "kernels.h"

namespace fbls {

namespace {

struct EvArgs {
    const double* cum;  // 3 x (nb2 + 1), field-major
    const double* durations;
    const double* rho;
    const double* dlm;
    const double* shapes;  // ns x layers x 3
    const double* priors;  // ns x 2
    const double* params;  // NPARAM
    const double* orbit;   // nd x NORB x 4
    const double* floors;  // 3
    double scale;
    double baseline;
    double threshold;
    double n;
    int nb2, nd, ns, layers;
};

__device__ __forceinline__ double circular_sum(const double* __restrict__ cum, size_t row, size_t start, size_t width,
                                               size_t nb2) {
    size_t j = start % nb2;
    size_t end = j + width;
    double left = cum[row + j];
    double right = cum[row + (end < nb2 ? end : nb2)];
    double wrap = cum[row + (end > nb2 ? end - nb2 : 0)];
    return right - left + wrap;
}

__device__ __forceinline__ double layered_sum(const EvArgs& a, size_t row, size_t start, size_t width, int si,
                                              bool squared) {
    const size_t nb2 = (size_t)a.nb2;
    double value = 0.0;
    for (int layer = 0; layer < a.layers; layer++) {
        const double* sh = a.shapes + ((size_t)si * a.layers + layer) * 3;
        uint64_t inner = as_u64(floor((double)width * sh[0] + 0.5));
        if (inner < 1) inner = 1;
        value += sh[squared ? 2 : 1] * circular_sum(a.cum, row, start + (width - inner) / 2, inner, nb2);
    }
    return value;
}

// Maximum over the 64 lanes of the CTA (every lane gets it).
__device__ __forceinline__ double tile_max(double v, double* s2) {
    for (int off = 16; off > 0; off >>= 1) v = rmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) s2[threadIdx.x >> 5] = v;
    __syncthreads();
    return rmax(s2[0], s2[1]);
}

}  // namespace

// Exclusive prefix over 2nb bins per field (evidence.rs:96-144), one CTA of
// 256 threads per field with the reference's association: per segment a
// block-wide Hillis-Steele scan (strides 1 .. 128) plus the running carry.
__global__ void __launch_bounds__(256) k_prefix_fields(const double* __restrict__ hist, double* __restrict__ cum,
                                                       int nb2) {
    __shared__ double scan[256];
    const int lane = threadIdx.x, field = blockIdx.x;
    const double* h = hist + (size_t)field * nb2;
    double* out = cum + (size_t)field * (nb2 + 1);
    if (lane == 0) out[0] = 0.0;
    double carry = 0.0;
    for (int seg = 0; seg < nb2; seg += 256) {
        const int b = seg + lane;
        scan[lane] = b < nb2 ? h[b] : 0.0;
        __syncthreads();
        for (int stride = 1; stride < 256; stride <<= 1) {
            const double add = lane >= stride ? scan[lane - stride] : 0.0;
            __syncthreads();
            if (lane >= stride) scan[lane] = __dadd_rn(scan[lane], add);
            __syncthreads();
        }
        if (b < nb2) out[b + 1] = __dadd_rn(scan[lane], carry);
        carry = __dadd_rn(carry, scan[255]);
        __syncthreads();
    }
}

// Amplitude screen (evidence.rs:151-273): per tile the maximum score, the
// planet and binary evidence lower bounds of the best-merit template and its
// key. The screen buffer is zeroed by the caller; a tile without a usable
// template leaves its entry at zero, as the reference's does.
__global__ void __launch_bounds__(EV_TILE) k_screen(EvArgs a, double* __restrict__ screen) {
    __shared__ double s_best[EV_TILE], s_merit[EV_TILE];
    __shared__ int s_chosen;
    __shared__ double s_max, s_bmax;
    const int lane = threadIdx.x, tile = blockIdx.x;
    const size_t nb2 = (size_t)a.nb2, nb = nb2 / 2;
    const size_t j = (size_t)tile * EV_TILE + lane;
    const size_t jj = j < nb - 1 ? j : nb - 1;
    const double c = a.baseline;
    double best = neg_inf(), bound_merit = neg_inf();
    double best_a = 0.0, best_q = 1.0, best_null = 0.0, best_ps = 0.0, best_bs = 0.0;
    uint64_t best_key = 0;
    for (int di = 0; di < a.nd; di++) {
        uint64_t raw_k = template_width(a.durations[di], a.scale);
        uint64_t k = raw_k < nb2 / 8 - 1 ? raw_k : nb2 / 8 - 1;
        double r = a.rho[di];
        double count = circular_sum(a.cum, 2 * (nb2 + 1), jj, k, nb2) + circular_sum(a.cum, 2 * (nb2 + 1), jj + nb, k, nb2);
        bool usable = j < nb && raw_k < nb2 / 8 && count >= 3.0 && count <= a.n - 3.0;
        for (int si = 0; si < a.ns; si++) {
            double av = layered_sum(a, 0, jj, k, si, false) + layered_sum(a, 0, jj + nb, k, si, false);
            double pe = layered_sum(a, nb2 + 1, jj, k, si, false);
            double po = layered_sum(a, nb2 + 1, jj + nb, k, si, false);
            double ne = layered_sum(a, nb2 + 1, jj, k, si, true);
            double no = layered_sum(a, nb2 + 1, jj + nb, k, si, true);
            double qe = ne - pe * pe / c, qo = no - po * po / c, qeo = -pe * po / c;
            double q = qe + qo + 2.0 * qeo;
            double score = av / sqrt(rmax(q * (r * r), 1e-300));
            bool score_valid = usable && av > 0.0 && q > 0.0;
            double merit = 0.5 * score * score + a.dlm[di] + a.priors[si * 2];
            if (score_valid && merit > bound_merit) {
                best_a = av / (r * r);
                best_q = q / (r * r);
                best_null = a.dlm[di];
                best_ps = a.priors[si * 2];
                best_bs = a.priors[si * 2 + 1];
                best_key = (uint64_t)(si * a.nd + di) * nb + jj;
                bound_merit = merit;
            }
            if (score_valid && score > best) best = score;
        }
    }
    s_best[lane] = best;
    s_merit[lane] = bound_merit;
    __syncthreads();
    if (lane == 0) {
        double maximum = neg_inf(), bound_maximum = neg_inf();
        int chosen = EV_TILE;
        for (int l = 0; l < EV_TILE; l++) {
            if (s_best[l] > maximum) maximum = s_best[l];
            if (s_merit[l] > bound_maximum) {
                bound_maximum = s_merit[l];
                chosen = l;
            }
        }
        s_chosen = chosen;
        s_max = maximum;
        s_bmax = bound_maximum;
    }
    __syncthreads();
    if (lane == s_chosen) {
        double lower_p = positive_amplitude_evidence(best_a, best_q, a.params[0]) + log(0.75) + best_null + best_ps;
        double lower_b = log_add(positive_amplitude_evidence(best_a, best_q, a.params[1]),
                                 positive_amplitude_evidence(best_a, best_q, a.params[2])) +
                         log(0.025) + best_null + best_bs;
        double* out = screen + (size_t)tile * 4;
        out[0] = s_max;
        out[1] = s_bmax > neg_inf() ? lower_p : neg_inf();
        out[2] = s_bmax > neg_inf() ? lower_b : neg_inf();
        out[3] = (double)best_key;
    }
}

// Evidence of every ephemeris in a tile (evidence.rs:280-632). pilot != 0:
// every lane evaluates the single template floors[2] and the output gives
// the floors of the full pass.
__global__ void __launch_bounds__(EV_TILE) k_joint(EvArgs a, int pilot, double* __restrict__ parts) {
    __shared__ double s_red[2];
    __shared__ double s_val[EV_TILE], s_sum[EV_TILE];
    __shared__ unsigned long long s_key[EV_TILE];
    __shared__ double s_out[4];
    const int lane = threadIdx.x, tile = blockIdx.x;
    const size_t nb2 = (size_t)a.nb2, nb = nb2 / 2;
    const int nd = a.nd;
    const uint64_t pilot_key = as_u64(a.floors[2]);
    const size_t j = pilot ? (size_t)(pilot_key % nb) : (size_t)tile * EV_TILE + lane;
    const size_t jj = j < nb - 1 ? j : nb - 1;
    const double c = a.baseline;
    const double tau_p = a.params[0], tau_b = a.params[1], tau_d = a.params[2];
    const double floor_p = pilot ? neg_inf() : a.floors[0];
    const double floor_b = pilot ? neg_inf() : a.floors[1];

    double best_joint = neg_inf(), best_signal = neg_inf();
    uint64_t joint_key = KEY_MAX, signal_key = KEY_MAX;
    double j_out[9], s_outv[9];
    for (int i = 0; i < 9; i++) j_out[i] = s_outv[i] = 0.0;
    double sum_p = neg_inf(), sum_b = neg_inf();
    uint32_t omitted = 0;

    int di_begin = 0, di_end = nd;
    if (pilot) {
        di_begin = (int)((pilot_key / nb) % (uint64_t)nd);
        di_end = di_begin + 1;
    }
    for (int di = di_begin; di < di_end; di++) {
        const uint64_t raw_k = template_width(a.durations[di], a.scale);
        const uint64_t k = raw_k < nb2 / 8 - 1 ? raw_k : nb2 / 8 - 1;
        const double rho2 = a.rho[di] * a.rho[di];
        const double dlm = a.dlm[di];
        const double count =
            circular_sum(a.cum, 2 * (nb2 + 1), jj, k, nb2) + circular_sum(a.cum, 2 * (nb2 + 1), jj + nb, k, nb2);
        const bool usable = j < nb && raw_k < nb2 / 8 && count >= 3.0 && count <= a.n - 3.0;
        int si_begin = 0, si_end = a.ns;
        if (pilot) {
            si_begin = (int)(pilot_key / ((uint64_t)nb * (uint64_t)nd));
            si_end = si_begin + 1;
        }
        for (int si = si_begin; si < si_end; si++) {
            const double ae = layered_sum(a, 0, jj, k, si, false);
            const double ao = layered_sum(a, 0, jj + nb, k, si, false);
            const double pe = layered_sum(a, nb2 + 1, jj, k, si, false);
            const double po = layered_sum(a, nb2 + 1, jj + nb, k, si, false);
            const double ne = layered_sum(a, nb2 + 1, jj, k, si, true);
            const double no = layered_sum(a, nb2 + 1, jj + nb, k, si, true);
            const double qe = ne - pe * pe / c, qo = no - po * po / c, qeo = -pe * po / c;
            const double ap = ae + ao, qp = qe + qo + 2.0 * qeo;
            const double snr = ap / sqrt(rmax(qp * rho2, 1e-300));
            const double depth = ap / rmax(qp, 1e-300);
            const bool valid = usable && ap > 0.0 && qp > 0.0 && snr >= a.threshold;
            if (!(raw_k < nb2 / 8)) continue;
            double lp = neg_inf(), lb = neg_inf(), component_best = neg_inf();
            double sec_ratio = 0.0, sec_phase = 0.5, odd_ratio = 1.0, binary_multiple = 1.0;
            double omitted_upper = neg_inf();
            for (int phase_index = 0; phase_index < NORB; phase_index++) {
                const double* ob = a.orbit + ((size_t)di * NORB + phase_index) * 4;
                const double phase = ob[0], duration_ratio = ob[1], logwp = ob[2], logwb = ob[3];
                const int64_t offset = (int64_t)floor(phase * (double)nb + 0.5);
                int64_t sk64 = (int64_t)floor((double)k * duration_ratio + 0.5);
                if (sk64 < 1) sk64 = 1;
                if (sk64 > (int64_t)nb - 1) sk64 = (int64_t)nb - 1;
                const size_t sk = (size_t)sk64;
                const size_t s0 = (size_t)((int64_t)jj + offset + (int64_t)floor(((double)k - (double)sk) / 2.0));
                const size_t s1 = s0 + nb;
                const double ass = layered_sum(a, 0, s0, sk, si, false) + layered_sum(a, 0, s1, sk, si, false);
                const double ps = layered_sum(a, nb2 + 1, s0, sk, si, false) + layered_sum(a, nb2 + 1, s1, sk, si, false);
                const double nsum = layered_sum(a, nb2 + 1, s0, sk, si, true) + layered_sum(a, nb2 + 1, s1, sk, si, true);
                const double qs = nsum - ps * ps / c;
                const double qps = -(pe + po) * ps / c;
                const double pa = ap / rho2, pb = ass / rho2, pq = qp / rho2, pr = qs / rho2, px = qps / rho2;
                const double cu = 1e-6;
                const double su = subspace_upper(pa, pb, pq, pr, px, 1.0);
                const double pu = su + logwp + cu;
                const double bu = su + logwb + cu;
                double upper = rmax(pu - floor_p, bu - floor_b) + dlm;
                if (!(logwp > neg_inf() || logwb > neg_inf())) upper = neg_inf();
                const double raw_upper = logwb > neg_inf() ? bu : neg_inf();
                const double tmax = tile_max(j < nb ? upper : neg_inf(), s_red);
                if (tmax >= 0.0) {
                    for (int ri = 0; ri < 5; ri++) {
                        const double ratio = a.params[6 + ri * 3];
                        const double wp = a.params[7 + ri * 3], wb = a.params[8 + ri * 3];
                        const double aa = pa + ratio * pb;
                        const double qq = pq + 2.0 * ratio * px + ratio * ratio * pr;
                        const double ep = positive_amplitude_evidence(aa, qq, tau_p) + log(wp) + logwp;
                        const double diluted = positive_amplitude_evidence(aa, qq, tau_d);
                        const double eb =
                            log_add(positive_amplitude_evidence(aa, qq, tau_b), diluted) + log(0.25 * wb) + logwb;
                        lp = log_add(lp, ep);
                        lb = log_add(lb, eb);
                        if (eb > component_best) {
                            sec_ratio = ratio;
                            sec_phase = phase;
                            component_best = eb;
                        }
                    }
                } else {
                    omitted += 1;
                    if (raw_upper > omitted_upper) omitted_upper = raw_upper;
                }
            }
            const double ba = ae / rho2, bb = ao / rho2, bq = qe / rho2, br = qo / rho2, bx = qeo / rho2;
            const double alias_mass = k < nb2 / 8 ? 0.0 : neg_inf();
            const double raw_upper = subspace_upper(ba, bb, bq, br, bx, 1.0) + 1e-6 + alias_mass;
            const double upper = raw_upper + dlm;
            const double tmax = tile_max(j < nb ? upper : neg_inf(), s_red);
            if (tmax >= floor_b) {
                for (int ri = 0; ri < 7; ri++) {
                    const double ratio = a.params[21 + ri];
                    const double aa = ba + ratio * bb;
                    const double qq = bq + 2.0 * ratio * bx + ratio * ratio * br;
                    const double diluted = positive_amplitude_evidence(aa, qq, tau_d);
                    const double eb =
                        log_add(positive_amplitude_evidence(aa, qq, tau_b), diluted) + alias_mass + log(0.25 / 7.0);
                    lb = log_add(lb, eb);
                    if (eb > component_best) {
                        sec_ratio = 0.0;
                        sec_phase = 0.5;
                        odd_ratio = ratio;
                        binary_multiple = 2.0;
                        component_best = eb;
                    }
                }
            } else {
                omitted += 1;
                if (raw_upper > omitted_upper) omitted_upper = raw_upper;
            }
            if (!(component_best > omitted_upper)) {
                sec_ratio = sec_phase = odd_ratio = binary_multiple = __longlong_as_double(0x7ff8000000000000ll);
            }
            lp += a.priors[si * 2] + dlm;
            lb += a.priors[si * 2 + 1] + dlm;
            if (j < nb) {
                sum_p = log_add(sum_p, lp);
                sum_b = log_add(sum_b, lb);
            }
            const double joint = lp;
            const uint64_t key = (uint64_t)(si * nd + di) * nb + jj;
            const bool bj = valid && (joint > best_joint || (joint == best_joint && key < joint_key));
            const bool bs = valid && (snr > best_signal || (snr == best_signal && key < signal_key));
            const double vals[9] = {snr, depth, lp, lb, sec_ratio, sec_phase, odd_ratio, binary_multiple, joint};
            if (bj) {
                for (int i = 0; i < 9; i++) j_out[i] = vals[i];
                best_joint = joint;
                joint_key = key;
            }
            if (bs) {
                for (int i = 0; i < 9; i++) s_outv[i] = vals[i];
                best_signal = snr;
                signal_key = key;
            }
        }
    }
    for (int selection = 0; selection < 2; selection++) {
        s_val[lane] = selection == 0 ? best_joint : best_signal;
        s_key[lane] = selection == 0 ? joint_key : signal_key;
        s_sum[lane] = selection == 0 ? sum_p : sum_b;
        __syncthreads();
        if (lane == 0) {
            double maximum = neg_inf();
            for (int l = 0; l < EV_TILE; l++)
                if (s_val[l] > maximum) maximum = s_val[l];
            unsigned long long best_key = KEY_MAX;
            int chosen = EV_TILE;
            for (int l = 0; l < EV_TILE; l++)
                if (s_val[l] == maximum && s_key[l] < best_key) {
                    best_key = s_key[l];
                    chosen = l;
                }
            double high = neg_inf();
            for (int l = 0; l < EV_TILE; l++)
                if (s_sum[l] > high) high = s_sum[l];
            double log_sum = high;
            if (high > neg_inf()) {
                double acc = 0.0;
                for (int l = 0; l < EV_TILE; l++) acc += exp(s_sum[l] - high);
                log_sum = high + log(acc);
            }
            s_out[0] = (double)best_key;
            s_out[1] = maximum;
            s_out[2] = (double)chosen;
            s_out[3] = log_sum;
        }
        __syncthreads();
        const int chosen = (int)s_out[2];
        double* out = parts + ((size_t)tile * 2 + selection) * EV_PART;
        if (lane == (chosen < EV_TILE - 1 ? chosen : EV_TILE - 1)) {
            const double* vals = selection == 0 ? j_out : s_outv;
            out[0] = s_out[0];
            out[1] = s_out[1];
            out[2] = selection == 0 ? vals[0] : best_signal;
            out[3] = vals[1];
            for (int i = 0; i < 6; i++) out[4 + i] = vals[2 + i];
            out[10] = selection == 0 ? best_joint : vals[8];
            out[13] = (double)omitted;
        }
        if (lane == 0) out[11 + selection] = s_out[3];
        __syncthreads();
    }
    if (lane == 0) {
        double* out0 = parts + (size_t)tile * 2 * EV_PART;
        const double sp = out0[11];
        const double sb = out0[EV_PART + 12];
        out0[12] = sb;
        out0[EV_PART + 11] = sp;
    }
}

// ---------------------------------------------------------------------------
// Host side of compare_search (evidence.rs:655-1003).
// ---------------------------------------------------------------------------

namespace {

double host_logsumexp(const std::vector<double>& v) {
    double high = neg_inf();
    for (double x : v) high = rmax(high, x);
    if (high == neg_inf()) return high;
    double s = 0.0;
    for (double x : v) s += std::exp(x - high);
    return high + std::log(s);
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

int compare_search(cudaStream_t stream, void*, size_t, const EvidenceReady& r, const double* durations_in,
                   const double* rho_in, uint32_t nd_in, double period, const fbls_config& cfg,
                   fbls_evidence_row* rows_out, uint32_t* n_rows, std::string& message,
                   const std::function<void*(size_t)>& workspace) {
    *n_rows = 0;
    std::vector<std::pair<double, double>> ds;
    for (uint32_t i = 0; i < nd_in; i++)
        if (durations_in[i] < period / 4.0) ds.push_back({durations_in[i], rho_in[i]});
    std::stable_sort(ds.begin(), ds.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    if (ds.empty()) return 0;
    const int nd = (int)ds.size();
    const int ns = (int)cfg.n_ingress;
    const int layers = (int)cfg.shape_layers;
    if (ns < 1 || layers < 1) {
        message = "invalid shape bank";
        return FBLS_ERR_ARGUMENT;
    }
    std::vector<double> durations(nd), rho(nd);
    for (int i = 0; i < nd; i++) {
        durations[i] = ds[i].first;
        rho[i] = ds[i].second;
    }
    const double dmin = durations[0];
    uint64_t nb = 4 * as_u64(std::ceil((double)cfg.phase_oversample * period / dmin / 4.0));
    if (nb < 8) nb = 8;
    const uint64_t nb2 = 2 * nb;
    if (nb2 > (1ull << 26)) {
        message = "evidence phase grid too large";
        return FBLS_ERR_ARGUMENT;
    }
    const double scale = (double)nb / period;
    if (std::floor(r.t_last * scale) >= 4294967295.0 - 2.0 * (double)nb2 - 2.0) {
        message = "phase cell exceeds 32 bits";
        return FBLS_ERR_ARGUMENT;
    }
    const double n = (double)r.n;
    std::vector<double> dlm(nd);
    for (int i = 0; i < nd; i++) {
        const double rr = rho[i];
        dlm[i] = -0.5 * ((n - 1.0) * std::log(rr * rr) + r.residual_energy / (rr * rr));
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
    std::vector<double> priors(2 * ns);
    for (int s = 0; s < ns; s++) {
        priors[2 * s] = lpl[s] - lp0;
        priors[2 * s + 1] = lbl[s] - lb0;
    }
    std::vector<double> shapes;
    for (int s = 0; s < ns; s++) {
        double previous = 0.0;
        for (int layer = 0; layer < layers; layer++) {
            const double fraction = 1.0 - 2.0 * cfg.ingress_fractions[s] * (double)layer / (double)(std::max(layers, 2) - 1);
            const double inc = 1.0 / (double)layers;
            shapes.push_back(fraction);
            shapes.push_back(inc);
            shapes.push_back(inc * (2.0 * previous + inc));
            previous += inc;
        }
    }
    double params[NPARAM];
    evidence_parameters(cfg, params);
    // Orbit bank: secondary phases 0.25, 0.5, 0.75 (evidence.rs:751-789).
    const double phases[3] = {0.25, 0.5, 0.75};
    const double logw[3] = {std::log(0.1), std::log(0.8), std::log(0.1)};
    std::vector<double> lp_bank((size_t)nd * NORB, neg_inf()), lb_bank((size_t)nd * NORB, neg_inf());
    size_t valid_count = 0;
    for (int di = 0; di < nd; di++) {
        const double k = rmax(std::floor(durations[di] * scale + 0.5), 1.0);
        if (k < (double)(nb / 4)) valid_count++;
        for (int o = 0; o < NORB; o++) {
            const double ks = rmax(std::floor(k + 0.5), 1.0);
            const double shift = std::floor(phases[o] * (double)nb + 0.5);
            const double start = shift + std::floor((k - ks) / 2.0);
            const bool valid = k < (double)(nb / 4) && ks < (double)(nb / 2) && start >= k && start + ks <= (double)nb;
            if (valid) {
                lp_bank[(size_t)di * NORB + o] = logw[o];
                lb_bank[(size_t)di * NORB + o] = logw[o];
            }
        }
    }
    const double count = std::log((double)valid_count);
    const double norm_p = count - host_logsumexp(lp_bank);
    const double norm_b = count - host_logsumexp(lb_bank);
    std::vector<double> orbit;
    for (int di = 0; di < nd; di++)
        for (int o = 0; o < NORB; o++) {
            orbit.push_back(phases[o]);
            orbit.push_back(1.0);
            orbit.push_back(lp_bank[(size_t)di * NORB + o] + norm_p);
            orbit.push_back(lb_bank[(size_t)di * NORB + o] + norm_b);
        }

    // Workspace: constants | floors | hist 3 nb2 | cum 3 (nb2+1) | screen | parts.
    const int tiles = (int)((nb + EV_TILE - 1) / EV_TILE);
    std::vector<double> consts;
    auto put = [&](const std::vector<double>& v) {
        size_t at = consts.size();
        consts.insert(consts.end(), v.begin(), v.end());
        return at;
    };
    const size_t o_dur = put(durations), o_rho = put(rho), o_dlm = put(dlm), o_shapes = put(shapes),
                 o_priors = put(priors), o_params = put(std::vector<double>(params, params + NPARAM)),
                 o_orbit = put(orbit), o_floors = put(std::vector<double>(3, 0.0)),
                 o_scale = put(std::vector<double>(1, scale));
    // Fold shape and chunks (ints, packed into the double workspace).
    FoldShape shape = fold_group_shape((int)nb2, 1, 1);
    std::vector<int> chunks((size_t)r.n + 2);
    const int nchunks = fold_chunks(r.time_host, (int)r.n, scale, (int)nb2, shape.span_cap, shape.chunk_cap,
                                    chunks.data(), (int)chunks.size());
    if (nchunks < 1) {
        message = "fold chunking failed";
        return FBLS_ERR_ARGUMENT;
    }
    std::vector<double> packed(((size_t)nchunks + 2) / 2 + 1, 0.0);
    std::memcpy(packed.data(), chunks.data(), ((size_t)nchunks + 1) * sizeof(int));
    const size_t o_chunks = put(packed);
    const bool fold_smem = shape.hist_in_smem;
    const size_t o_fscratch = consts.size();
    const size_t o_hist = o_fscratch + (fold_smem ? 0 : 3 * (size_t)shape.row_stride);
    const size_t o_cum = o_hist + 3 * nb2;
    const size_t o_screen = o_cum + 3 * (nb2 + 1);
    const size_t o_parts = o_screen + (size_t)tiles * 4;
    const size_t o_fault = o_parts + (size_t)tiles * 2 * EV_PART;
    const size_t total = o_fault + 1;
    double* ws = static_cast<double*>(workspace(total * sizeof(double)));
    if (!ws) {
        message = "evidence workspace allocation failed";
        return FBLS_ERR_CUDA;
    }
    auto check = [&](cudaError_t e, const char* where) {
        if (e != cudaSuccess) message = std::string(where) + ": " + cudaGetErrorString(e);
        return e == cudaSuccess;
    };
    if (!check(cudaMemcpyAsync(ws, consts.data(), consts.size() * sizeof(double), cudaMemcpyHostToDevice, stream),
               "evidence upload"))
        return FBLS_ERR_CUDA;
    if (!check(cudaMemsetAsync(ws + o_hist, 0, (o_parts - o_hist) * sizeof(double), stream), "evidence zero") ||
        !check(cudaMemsetAsync(ws + o_fault, 0, sizeof(double), stream), "evidence zero"))
        return FBLS_ERR_CUDA;
    // fold_two (evidence.rs:75-92): bin = floor(t * scale) mod 2 nb.
    FoldArgs fa{};
    fa.time = r.time;
    fa.v = r.v;
    fa.w = r.w;
    fa.scales = ws + o_scale;
    fa.n = (int)r.n;
    fa.nb = (int)nb2;
    fa.periods = 1;
    fa.group = 1;
    fa.hist_global = fold_smem ? nullptr : ws + o_fscratch;
    fa.hist_out = ws + o_hist;
    fa.chunks = reinterpret_cast<const int*>(ws + o_chunks);
    fa.nchunks = nchunks;
    fa.stage_field = shape.stage_field;
    fa.window = shape.window;
    fa.row_stride = shape.row_stride;
    fa.fault = reinterpret_cast<uint32_t*>(ws + o_fault);
    if (!check(launch_fold(fa, shape, stream), "evidence fold")) return FBLS_ERR_CUDA;
    k_prefix_fields<<<3, 256, 0, stream>>>(ws + o_hist, ws + o_cum, (int)nb2);
    EvArgs ea;
    ea.cum = ws + o_cum;
    ea.durations = ws + o_dur;
    ea.rho = ws + o_rho;
    ea.dlm = ws + o_dlm;
    ea.shapes = ws + o_shapes;
    ea.priors = ws + o_priors;
    ea.params = ws + o_params;
    ea.orbit = ws + o_orbit;
    ea.floors = ws + o_floors;
    ea.scale = scale;
    ea.baseline = r.baseline_norm;
    ea.threshold = cfg.threshold;
    ea.n = n;
    ea.nb2 = (int)nb2;
    ea.nd = nd;
    ea.ns = ns;
    ea.layers = layers;
    k_screen<<<tiles, EV_TILE, 0, stream>>>(ea, ws + o_screen);
    if (!check(cudaGetLastError(), "evidence screen")) return FBLS_ERR_CUDA;
    std::vector<double> screen((size_t)tiles * 4);
    uint32_t fault = 0;
    if (!check(cudaMemcpyAsync(screen.data(), ws + o_screen, screen.size() * sizeof(double), cudaMemcpyDeviceToHost,
                               stream),
               "evidence screen download") ||
        !check(cudaMemcpyAsync(&fault, ws + o_fault, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream),
               "evidence fault download") ||
        !check(cudaStreamSynchronize(stream), "evidence screen"))
        return FBLS_ERR_CUDA;
    if (fault) {
        message = "evidence fold: staging copies did not complete";
        return FBLS_ERR_CUDA;
    }
    double maximum = neg_inf();
    for (int t = 0; t < tiles; t++) maximum = rmax(maximum, screen[(size_t)t * 4]);
    if (!(maximum >= cfg.threshold * (1.0 - 1e-12))) return 0;
    int winner = 0;  // Iterator::max_by keeps the last maximum
    for (int t = 1; t < tiles; t++)
        if (screen[(size_t)t * 4 + 1] >= screen[(size_t)winner * 4 + 1]) winner = t;
    const double pilot_key = screen[(size_t)winner * 4 + 3];
    const double margin = cfg.evidence_rtol > 0.0
                              ? std::log(cfg.evidence_rtol) - std::log((double)((NORB + 1) * nb * (uint64_t)nd * ns))
                              : neg_inf();
    double floors0[3] = {neg_inf(), neg_inf(), pilot_key};
    if (!check(cudaMemcpyAsync(ws + o_floors, floors0, sizeof(floors0), cudaMemcpyHostToDevice, stream), "floors"))
        return FBLS_ERR_CUDA;
    k_joint<<<1, EV_TILE, 0, stream>>>(ea, 1, ws + o_parts);
    double pilot[2 * EV_PART];
    if (!check(cudaMemcpyAsync(pilot, ws + o_parts, sizeof(pilot), cudaMemcpyDeviceToHost, stream), "pilot") ||
        !check(cudaStreamSynchronize(stream), "pilot"))
        return FBLS_ERR_CUDA;
    double floors[3] = {pilot[11] + margin, pilot[12] + margin, pilot_key};
    if (!check(cudaMemcpyAsync(ws + o_floors, floors, sizeof(floors), cudaMemcpyHostToDevice, stream), "floors"))
        return FBLS_ERR_CUDA;
    k_joint<<<tiles, EV_TILE, 0, stream>>>(ea, 0, ws + o_parts);
    std::vector<double> parts((size_t)tiles * 2 * EV_PART);
    if (!check(cudaMemcpyAsync(parts.data(), ws + o_parts, parts.size() * sizeof(double), cudaMemcpyDeviceToHost,
                               stream),
               "parts") ||
        !check(cudaStreamSynchronize(stream), "joint"))
        return FBLS_ERR_CUDA;

    std::vector<double> in_bank;
    for (int i = 0; i < nd; i++)
        if (rmax(std::floor(durations[i] * scale + 0.5), 1.0) < (double)(nb / 4)) in_bank.push_back(dlm[i]);
    const double log_mass = std::log((double)nb) + host_logsumexp(in_bank);
    fbls_evidence_row rows[2];
    for (int selection = 0; selection < 2; selection++) {
        auto value = [&](int t, int i) { return parts[((size_t)t * 2 + selection) * EV_PART + i]; };
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
        std::vector<double> s11(tiles), s12(tiles);
        for (int t = 0; t < tiles; t++) {
            s11[t] = value(t, 11);
            s12[t] = value(t, 12);
        }
        const double lp = host_logsumexp(s11) - log_mass;
        const double lb = host_logsumexp(s12) - log_mass;
        const double joint = params[3] + lp - log_add(params[5], params[4] + lb);
        const uint64_t decoded = mx > neg_inf() ? as_u64(key) : 0;
        const size_t j = (size_t)(decoded % nb);
        const size_t di = (size_t)((decoded / nb) % (uint64_t)nd);
        const size_t si = (size_t)(decoded / (nb * (uint64_t)nd));
        const double width = rmax(std::floor(durations[di] * scale + 0.5), 1.0);
        fbls_evidence_row& row = rows[selection];
        row.period = period;
        row.epoch = ((double)j + width / 2.0) / scale + r.origin;
        row.duration = width / scale;
        row.snr = mx > neg_inf() ? value(tile, 2) : neg_inf();
        row.depth = value(tile, 3);
        row.planet_log_odds = joint;
        row.log_bf_planet_noise = lp;
        row.log_bf_binary_noise = lb;
        row.binary_secondary_ratio = value(tile, 6);
        row.binary_secondary_phase = value(tile, 7);
        row.binary_odd_even_ratio = value(tile, 8);
        row.binary_period_days = value(tile, 9) * period;
        row.ingress_fraction = cfg.ingress_fractions[std::min(si, (size_t)(ns - 1))];
        row.selection_flags = selection == 0 ? 1u : 2u;
    }
    const bool hit0 = std::isfinite(rows[0].snr), hit1 = std::isfinite(rows[1].snr);
    const bool same = hit0 && hit1 && rows[0].period == rows[1].period && rows[0].epoch == rows[1].epoch &&
                      rows[0].duration == rows[1].duration && rows[0].snr == rows[1].snr &&
                      rows[0].depth == rows[1].depth && rows[0].ingress_fraction == rows[1].ingress_fraction;
    uint32_t out = 0;
    if (hit0) {
        rows_out[out] = rows[0];
        if (same) rows_out[out].selection_flags = 3;
        out++;
    }
    if (hit1 && !same) rows_out[out++] = rows[1];
    *n_rows = out;
    return 0;
}

}  // namespace fbls
