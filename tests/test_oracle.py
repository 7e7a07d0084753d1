"""The oracle against the reference's own known-answer tests that need code
(noise model, transit mask; the tabulated ones, erfc and the period grid, are
in test_golden.py), and brute-force identities of the fold / prefix /
interval arithmetic. CPU only."""
import math

import numpy as np
import pytest

import oracle
from fbls_b200 import synth


def test_noise_model_normalizes_and_inflates():
    # curve.rs:636-661.
    n = 500
    t = 1000.0 + np.arange(n) * 0.01
    f = 2000.0 + 3.0 * np.sin(np.arange(n) * 1.7)
    e = np.ones(n)
    time, deficit, variance, origin, inflation, segments = oracle.fit_segment_noise(t, f, e, 0.75)
    assert origin == 1000.0
    assert time[0] == 0.0
    median = np.sort(f)[(n - 1) // 2]
    assert abs(deficit[0] - (1.0 - f[0] / median)) < 1e-12
    assert inflation > 2.0
    assert segments == 1


def test_transit_mask_and_cycles():
    # curve.rs:663-673.
    t = np.arange(1000) * 0.01
    m = oracle.transit_mask(t, 2.0, 1.0, 0.2, 0.0)
    direct = sum(1 for x in t if abs(math.fmod(x - 1.0 + 1.0, 2.0) - 1.0) <= 0.1)
    assert m.sum() == direct
    assert 100 <= direct <= 110


def test_log_add_and_evidence_limits():
    assert oracle.log_add(-math.inf, -math.inf) == -math.inf
    assert abs(oracle.log_add(0.0, 0.0) - math.log(2.0)) < 1e-15
    # No data: the normalized half-normal prior integrates the likelihood ratio 1 to log 1 = 0.
    assert oracle.positive_amplitude_evidence(0.0, 0.0, 0.01) == 0.0
    # Continuity across the asymptotic branch at z = -26.
    tau, q = 1.0, 0.0
    lo = oracle.positive_amplitude_evidence(-26.0 - 1e-9, q, tau)
    hi = oracle.positive_amplitude_evidence(-26.0 + 1e-9, q, tau)
    assert abs(lo - hi) < 1e-6
    assert oracle.subspace_upper(-1.0, -1.0, 1.0, 1.0, 0.0, 1.0) == pytest.approx(1e-6)


@pytest.fixture(scope="module")
def small_state():
    c = synth.small_curve()
    cfg = synth.small_config()
    return oracle.family_state(c.time, c.flux, c.flux_err, cfg.durations_days()), cfg, c


def test_prefix_matches_direct_box_sums(small_state):
    """fold + doubled prefix + interval difference == direct per-observation sums,
    including windows that wrap around phase zero."""
    st, cfg, _ = small_state
    nb = 97
    scale = nb / 1.2345
    folded, cum, cum32 = oracle.fold_prefix(st, scale, nb)
    rng = np.random.default_rng(0)
    for _ in range(200):
        j = int(rng.integers(0, nb))
        k = int(rng.integers(1, nb // 2 + 1))
        direct = oracle.box_direct(st, scale, nb, j, k)
        via = [cum[f, j + k] - cum[f, j] for f in (0, 1, 2)]
        assert via[2] == direct[2]
        assert abs(via[0] - direct[0]) <= 1e-9 * np.abs(st.v).sum()
        assert abs(via[1] - direct[1]) <= 1e-12 * st.w.sum()
    # (hi, lo) pairs represent the f64 prefix to f32 x f32 precision.
    rec = cum32[..., 0].astype(np.float64) + cum32[..., 1].astype(np.float64)
    assert np.all(np.abs(rec - cum) <= 1e-13 * np.abs(cum).max())
    # Second copy = first + the row total (the carry of the segment scan).
    total = cum[:, nb:nb + 1]
    assert np.all(np.abs(cum[:, nb + 1:] - (cum[:, 1:nb + 1] + total)) <= 4e-16 * np.abs(cum).max())


def test_winner_is_the_f64_argmax_in_f64_mode(small_state):
    """In f64-only mode each period's record is the argmax of the exact score
    over every (phase, duration) box template (shapes gated off here)."""
    st, cfg, _ = small_state
    periods = np.array([0.77, 1.3, 2.2])
    nb = 60
    d = np.array(sorted(cfg.durations_days()))
    rec, score, depth, flags, _ = oracle.scan_bank(st, periods, nb, d, st.rho, ingress=(0.0,), shape_gate=1e9, mode=1)
    for i, p in enumerate(periods):
        scale = nb / p
        best = (-math.inf, None)
        for di, dur in enumerate(d):
            raw_k = max(1, math.floor(dur * scale + 0.5))
            k = min(raw_k, nb // 2)
            if raw_k >= nb // 2:
                continue
            for j in range(nb):
                a, hp, cnt = oracle.box_direct(st, scale, nb, j, k)
                if not (3 <= cnt <= st.n - 3 and a > 0):
                    continue
                q = hp - hp * hp / st.baseline_norm
                s = (a / st.rho[di]) / math.sqrt(q)
                if s > best[0] * (1 + 1e-12):
                    best = (s, (j, k))
        assert (int(rec[i, 2]), int(rec[i, 3])) == best[1]
        assert score[i] == pytest.approx(best[0], rel=1e-9)


def test_oracle_recovers_injected_signal(small_state):
    st, cfg, c = small_state
    rows, grid, stats = oracle.signal_search(st, cfg)
    assert len(rows) > 0
    best = rows[np.argmax(rows[:, 3])]
    assert abs(best[0] / c.period - 1.0) < 0.01
    phase = ((best[1] - c.epoch) / c.period + 0.5) % 1.0 - 0.5
    assert abs(phase * c.period) < c.duration


def test_mixed_and_f64_modes_agree_on_winners(small_state):
    st, cfg, _ = small_state
    periods = oracle.period_grid(0.5, 1.0, float(st.time[-1]), 0.75 / 24, 3.0)
    d = np.array(sorted(cfg.durations_days()))[:3]
    r0 = oracle.scan_bank(st, periods, 64, d, st.rho[:3], mode=0)
    r1 = oracle.scan_bank(st, periods, 64, d, st.rho[:3], mode=1)
    same = (r0[0][:, 2:4] == r1[0][:, 2:4]).all(axis=1) & (r0[0][:, 7] == r1[0][:, 7])
    assert same.mean() > 0.99
    ok = np.isfinite(r0[1])
    assert np.allclose(r0[1][ok & same], r1[1][ok & same], rtol=1e-12)


def test_erfc_against_arbitrary_precision():
    """Beyond the reference's 16-value table: Cody's approximation as the
    reference evaluates it stays within 2e-15 of the exact value (mpmath at
    50 digits) on [-6, XBIG), is exactly 0 from XBIG = 26.543 on (the
    reference returns 0 there; the exact value is subnormal), and keeps
    erfc(-x) = 2 - erfc(x)."""
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.dps = 50
    xs = np.concatenate([np.linspace(-6.0, 26.54, 4001), [0.46875, 0.46876, 4.0, 4.0000001, 26.5429]])
    worst = max(abs(oracle.erfc(x) - float(mpmath.erfc(x))) / float(mpmath.erfc(x)) for x in xs)
    assert worst < 2e-15, worst
    assert all(oracle.erfc(x) == 0.0 for x in (26.543, 26.6, 30.0, 1e300))
    assert all(oracle.erfc(-x) == 2.0 - oracle.erfc(x) for x in (0.5, 1.0, 3.0, 10.0))


def test_log_add_against_arbitrary_precision():
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.dps = 50
    vals = [-700.0, -50.0, -3.5, -1e-3, 0.0, 2.0, 40.0, 700.0]
    for a in vals:
        for b in vals:
            exact = float(mpmath.log(mpmath.exp(a) + mpmath.exp(b)))
            assert abs(oracle.log_add(a, b) - exact) <= 4e-16 * max(1.0, abs(exact)), (a, b)


def test_positive_amplitude_evidence_is_the_half_normal_integral():
    """math.rs:112-139: log of the integral over depths x >= 0 of a
    half-normal prior of scale tau times exp(a x - q x^2 / 2), in closed form
    -ln(1 + tau^2 q) / 2 + z^2 / 2 + ln erfc(-z / sqrt 2); the reference's
    asymptotic series below z = -26 included."""
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.dps = 60
    rng = np.random.default_rng(6)
    cases = [(a, q, tau) for a, q, tau in zip(rng.normal(0.0, 30.0, 300), np.exp(rng.uniform(-3, 8, 300)),
                                              np.exp(rng.uniform(-6, 1, 300)))]
    cases += [(-2000.0, 100.0, 1.0), (-5000.0, 1e4, 0.5), (-30.0, 0.0, 1.0), (0.0, 1.0, 0.1), (5.0, -3.0, 0.2)]
    seen_series = False
    for a, q, tau in cases:
        qq = max(q, 0.0)
        precision = 1 + mpmath.mpf(tau) ** 2 * qq
        z = mpmath.mpf(tau) * a / mpmath.sqrt(precision)
        seen_series |= z < -26
        exact = -mpmath.log(precision) / 2 + z * z / 2 + mpmath.log(mpmath.erfc(-z / mpmath.sqrt(2)))
        got = oracle.positive_amplitude_evidence(a, q, tau)
        assert abs(got - float(exact)) <= 1e-11 * max(1.0, abs(float(exact))), (a, q, tau, got, float(exact))
    assert seen_series


def test_subspace_upper_bounds_every_positive_mixture():
    """math.rs:141-177: an upper bound of (a x + b y - [x y] M [x y]^T / 2) / rho^2
    over depths x, y >= 0 (M = [[q, c], [c, r]]), within its 1e-6 margins."""
    rng = np.random.default_rng(7)
    for _ in range(300):
        q, r = np.exp(rng.uniform(-2, 3, 2))
        c = rng.uniform(-0.95, 0.95) * math.sqrt(q * r)
        a, b = rng.normal(0.0, 5.0, 2)
        rho2 = rng.uniform(1.0, 3.0)
        upper = oracle.subspace_upper(a, b, q, r, c, rho2)
        xs = np.abs(rng.normal(0.0, 3.0, (400, 2)))
        grid = np.stack(np.meshgrid(np.linspace(0, 6, 61), np.linspace(0, 6, 61)), -1).reshape(-1, 2)
        x, y = np.vstack([xs, grid]).T
        value = (a * x + b * y - 0.5 * (q * x * x + 2 * c * x * y + r * y * y)) / rho2
        assert value.max() <= upper + 1e-9, (a, b, q, r, c, rho2, value.max(), upper)
    assert oracle.subspace_upper(-1.0, -2.0, 1.0, 1.0, 0.0, 1.0) == pytest.approx(1e-6)  # no positive gain


def test_single_event_rows_are_every_box_template_over_the_threshold():
    """The oracle's single-event scan (events.rs:18-153, scan_all
    kernels.rs:851-921) with the box shape only, against a brute-force
    enumeration: one trial period baseline + 2 x longest duration + 1e-6 d,
    nb = max(8, ceil(phase_oversample x trial / shortest duration)), every
    (phase, duration) window from direct per-observation sums that is usable
    (raw width below nb / 2, 3 ... n - 3 observations, a > 0, q > 0) and
    reaches the threshold."""
    import dataclasses as dc
    c = synth.small_curve()
    cfg = dc.replace(synth.small_config(), ingress_fractions=[0.0], threshold=4.0)
    st = oracle.family_state(c.time, c.flux, c.flux_err, cfg.durations_days())
    rows, stats = oracle.single_event_search(st, cfg)
    order = np.argsort(st.durations, kind="stable")
    d, rho = st.durations[order], st.rho[order]
    trial = float(st.time[-1]) + 2.0 * d[-1] + 1e-6
    nb = max(8, math.ceil(cfg.phase_oversample * trial / d[0]))
    scale = nb / trial
    want = {}
    for di in range(len(d)):
        raw_k = max(1, math.floor(d[di] * scale + 0.5))
        if raw_k >= nb // 2:
            continue
        k = raw_k
        for j in range(nb):
            a, hp, cnt = oracle.box_direct(st, scale, nb, j, k)
            q = hp - hp * hp / st.baseline_norm
            if not (3 <= cnt <= st.n - 3 and a > 0 and q > 0):
                continue
            score = (a / rho[di]) / math.sqrt(q)
            if score >= cfg.threshold:
                want[(j, k, di)] = (score, a / q)
    got = {}
    for r in rows:
        j = round((r[1] - st.origin) * scale - (r[2] * scale) / 2.0)
        k = round(r[2] * scale)
        di = next(i for i in range(len(d)) if max(1, math.floor(d[i] * scale + 0.5)) == k and (j, k, i) not in got)
        got[(j, k, di)] = (r[3], r[4])
    assert len(want) > 20 and stats["threshold_survivors"] == len(rows)
    near = {key for key, (s, _) in want.items() if abs(s - cfg.threshold) <= 1e-9 * cfg.threshold}
    assert set(got) ^ set(want) <= near
    for key in set(got) & set(want):
        assert got[key][0] == pytest.approx(want[key][0], rel=1e-9)
        assert got[key][1] == pytest.approx(want[key][1], rel=1e-9)
