"""The precision of the phase-bin index, on the CPU: the reference's bin is
floor(t * scale) of one correctly rounded f64 product (kernels.rs:314-327,
scale = nb / P from scan.rs:204). On the 13-sector workload's times, an f32
product gives another bin for about 0.2 % of (observation, period) pairs,
while a double-single product (Dekker's split and two-product in f32, the
value hi + lo floored with the sign of lo at integers) agreed with f64 on
every pair sampled; the library keeps the bin in f64 (the fold is bound by
its shared-memory pipe, not by f64 throughput, so f64 costs nothing there).

    python -c "import sys; sys.path[:0] = ['.', 'tests']; import test_precision_bins as t; print(t.bin_mismatches(400))"

reproduces the larger sample (every band's periods thinned to about 400 per
band, 601,451,136 pairs).

The prefix sums: box sums a = cum[j + k] - cum[j] of the precision-weighted
deficit v over random (phase, width) windows, from an f32 prefix and from the
(hi, lo) f32 pairs the scan pre-ranks with (hi = f32(cum), lo = f32(cum - hi),
a = (hi_b - hi_a) + (lo_b - lo_a), kernels.rs:51-146), against f64: the plain
f32 prefix loses to cancellation over long prefixes, the pairs do not. On the
13-sector star, 8 periods per band and 2,000 windows each (prefix_errors(8)):
relative error median 2.6e-7 and 99th percentile 2.0e-5 for the plain f32
prefix, 2.3e-8 and 8.3e-8 for the pairs."""
import numpy as np

from fbls_b200 import api, synth

F32 = np.float32


def _split(a):
    c = (a * F32(4097.0)).astype(F32)
    hi = (c - (c - a)).astype(F32)
    return hi, (a - hi).astype(F32)


def _two_prod(a, b):
    p = (a * b).astype(F32)
    ah, al = _split(a)
    bh, bl = _split(b)
    return p, ((((ah * bh - p) + ah * bl) + al * bh) + al * bl).astype(F32)


def _ds_floor(t_hi, t_lo, s_hi, s_lo):
    """floor of the double-single product (t_hi + t_lo)(s_hi + s_lo)."""
    p, e = _two_prod(t_hi, s_hi)
    e = (e + (t_hi * s_lo + t_lo * s_hi)).astype(F32)
    hi = (p + e).astype(F32)
    lo = (e - (hi - p)).astype(F32)
    f = np.floor(hi).astype(np.float64)
    return f - ((f == hi) & (lo < 0))


def bin_mismatches(per_band: int):
    """(pairs, f32 mismatches, double-single mismatches) against the f64 bins
    over about `per_band` periods of every band of the 13-sector workload."""
    c, cfg = synth.multi_sector(), synth.multi_sector_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    _, bands = api.band_plan(st, cfg)
    t = st.time
    t_hi = t.astype(F32)
    t_lo = (t - t_hi.astype(np.float64)).astype(F32)
    pairs = m32 = mds = 0
    for b in bands:
        for period in b["periods"][:: max(1, len(b["periods"]) // per_band)]:
            scale = b["nb"] / period
            ref = np.floor(t * scale)
            f32 = np.floor((t_hi * F32(scale)).astype(F32)).astype(np.float64)
            s_hi = F32(scale)
            ds = _ds_floor(t_hi, t_lo, s_hi, F32(scale - np.float64(s_hi)))
            pairs += t.size
            m32 += int((f32 != ref).sum())
            mds += int((ds != ref).sum())
    return pairs, m32, mds


def test_f32_bins_are_not_exact_and_double_single_bins_agree_on_the_sample():
    pairs, m32, mds = bin_mismatches(4)
    assert pairs > 5_000_000
    assert m32 / pairs > 1e-3  # an f32 bin index is not the reference's
    assert mds == 0


def prefix_errors(per_band: int, windows: int = 2000, seed: int = 0):
    """(median, 99th percentile) of the relative box-sum error for the plain
    f32 prefix and for the (hi, lo) pairs, over about `per_band` periods of
    every band of the 13-sector workload at the band's nb."""
    c, cfg = synth.multi_sector(), synth.multi_sector_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    _, bands = api.band_plan(st, cfg)
    rng = np.random.default_rng(seed)
    e32, ec = [], []
    for b in bands:
        nb = b["nb"]
        for period in b["periods"][:: max(1, len(b["periods"]) // per_band)]:
            bins = np.floor(st.time * (nb / period)).astype(np.int64) % nb
            h = np.bincount(bins, weights=st.v, minlength=nb)
            h2 = np.concatenate([h, h])
            cum = np.concatenate([[0.0], np.cumsum(h2)])
            c32 = np.concatenate([[F32(0.0)], np.cumsum(h2.astype(F32), dtype=F32)])
            hi = cum.astype(F32)
            lo = (cum - hi.astype(np.float64)).astype(F32)
            j = rng.integers(0, nb, windows)
            k = rng.integers(1, nb // 2, windows)
            exact = cum[j + k] - cum[j]
            denom = np.maximum(np.abs(exact), 1e-300)
            e32.append(np.abs((c32[j + k] - c32[j]).astype(np.float64) - exact) / denom)
            ec.append(np.abs(((hi[j + k] - hi[j]) + (lo[j + k] - lo[j])).astype(np.float64) - exact) / denom)
    e32, ec = np.concatenate(e32), np.concatenate(ec)
    return (np.median(e32), np.percentile(e32, 99)), (np.median(ec), np.percentile(ec, 99))


def test_compensated_pairs_keep_box_sums_that_a_plain_f32_prefix_loses():
    (m32, p32), (mc, pc) = prefix_errors(4)
    assert pc < 5e-7 and mc < 1e-7
    assert p32 > 100 * pc
