"""Peak selection (src/select/peaks.rs) on the CPU: the oracle's rescoring
sums against a literal loop restatement of the reference kernels
(kernels.rs:936-1042), the host helpers, and select_peaks / select_events
driven by an oracle-backed rescorer."""
import math

import numpy as np
import pytest

import oracle
from fbls_b200 import api, select, synth


def _lanes_then_tree(values_by_lane):
    """The reference's 256-lane tree: red[l] += red[l + s], s = 128 ... 1."""
    red = list(values_by_lane)
    s = 128
    while s > 0:
        for l in range(s):
            red[l] = red[l] + red[l + s]
        s //= 2
    return red[0]


def _rescore_loop(t, v, w, ex, row, origin):
    period, epoch, duration = row
    inverse = 1.0 / period
    half = duration / 2.0
    parts = []
    for lane in range(256):
        a = hp = norm = 0.0
        for i in range(lane, len(t), 256):
            if ex[i]:
                continue
            x = (t[i] + origin - epoch) * inverse + 0.5
            phase = (x - math.floor(x) - 0.5) * period
            if abs(phase) <= half:
                a += v[i]
                hp += w[i]
                norm += w[i]
        parts.append((a, hp, norm))
    return tuple(_lanes_then_tree([p[k] for p in parts]) for k in range(3))


def _count_loop(t, ex, row):
    period, epoch, duration = row
    inverse = 1.0 / period
    half = duration / 2.0
    tot, uns = [0] * 256, [0] * 256
    for lane in range(256):
        for i in range(lane, len(t), 256):
            x = (t[i] - epoch) * inverse + 0.5
            phase = (x - math.floor(x) - 0.5) * period
            if abs(phase) <= half:
                tot[lane] += 1
                uns[lane] += 0 if ex[i] else 1
    return _lanes_then_tree(tot), _lanes_then_tree(uns)


def test_oracle_rescore_matches_the_kernel_loops():
    rng = np.random.default_rng(4)
    n = 2100
    t = np.sort(rng.uniform(0.0, 27.0, n))
    v, w = rng.normal(size=n), rng.uniform(0.5, 2.0, n)
    ex = (rng.uniform(size=n) < 0.15).astype(np.uint8)
    origin = 2458000.25
    rows = np.array([[3.1, origin + 2.0, 0.2], [1.7, origin + 0.3, 0.1], [13.0, origin + 5.0, 0.3],
                     [0.6, origin - 7.7, 0.9]])
    got = oracle.rescore_rows(t, v, w, ex, rows, origin)
    for r in range(rows.shape[0]):
        assert tuple(got[r]) == _rescore_loop(t, v, w, ex, rows[r], origin)
    ta = t + origin
    cnt = oracle.count_rows(ta, ex, rows)
    for r in range(rows.shape[0]):
        assert tuple(int(x) for x in cnt[r]) == _count_loop(ta, ex, rows[r])


def test_host_helpers():
    rng = np.random.default_rng(1)
    t = np.sort(rng.uniform(-40.0, 60.0, 4000))
    for period, epoch, duration, margin in [(3.1, 2.0, 0.2, 0.0), (1.7, -0.3, 0.1, 0.5), (0.77, 10.0, 0.05, 0.0)]:
        # the oracle's transit_mask is pinned by the reference's test (curve.rs:663-673)
        assert np.array_equal(select.transit_mask(t, period, epoch, duration, margin),
                              oracle.transit_mask(t, period, epoch, duration, margin))
    x = np.array([-2.5, -1.5, -0.5, 0.5, 1.5, 2.5, 0.49999999999999994, -0.49999999999999994])
    assert select.round_half_away(x).tolist() == [-3.0, -2.0, -1.0, 1.0, 2.0, 3.0, 0.0, -0.0]
    a = np.array([True, True, False, True])
    assert select.overlap(a, np.array([True, False, True, False])) == pytest.approx(1.0 / 3.0)
    assert select.overlap(np.zeros(4, bool), a) == 0.0
    # three epochs of 3+ points, one of 2 points
    tt = np.concatenate([e + np.array([-0.01, 0.0, 0.01]) for e in (1.0, 3.0, 5.0)] + [np.array([6.99, 7.01])])
    assert select.event_count(tt, 2.0, 1.0, 0.05, 3) == 3
    assert select.event_count(tt, 2.0, 1.0, 0.05, 2) == 4


class _OracleGpu:
    """A CPU stand-in for the rescoring calls (test infrastructure)."""

    class _Dev:
        def __init__(self, state):
            self.state = state
            self.n = state.n

        def free(self):
            pass

    def upload(self, state):
        return self._Dev(state)

    def rescore_rows(self, dev, excluded, rows):
        s = dev.state
        return oracle.rescore_rows(s.time, s.v, s.w, excluded, rows, s.origin)

    def count_rows(self, time, excluded, rows):
        return oracle.count_rows(time, excluded, rows)


def _families():
    c, cfg = synth.small_curve(), synth.small_config()
    full = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    st = oracle.family_state(c.time, c.flux, c.flux_err, cfg.durations_days(), cfg.correlated_noise)
    return c, cfg, full, st


def test_select_peaks_accepts_the_injected_signal_on_cpu():
    c, cfg, full, st = _families()
    rows, _, _ = oracle.signal_search(st, cfg)
    assert rows.shape[0] > 0
    time_all = np.unique(full.time + full.origin)
    family = np.zeros(rows.shape[0], dtype=np.int64)
    sel = select.select_peaks(_OracleGpu(), rows, family, [full], time_all, cfg.threshold, 5, 2, [],
                              np.zeros(time_all.shape[0], bool), 1)
    assert len(sel.accepted) >= 1
    best = sel.accepted[0]
    assert best.snr_folded == rows[:, 3].max()
    assert abs(best.period_days - c.period) / c.period < 0.01
    assert sel.excluded.any() and len(sel.masks) == len(sel.accepted)
    # accepted ephemerides overlap earlier masks by less than half
    for k in range(1, len(sel.accepted)):
        p = sel.accepted[k]
        m = select.transit_mask(time_all, p.period_days, p.epoch_bjd, p.duration_hours / 24.0, 0.0)
        assert all(select.overlap(m, other) < 0.5 for other in sel.masks[:k])


def test_select_events_suppresses_overlaps():
    t = np.arange(0.0, 10.0, 0.01)
    table = np.array([[0.0, 2.0, 0.1, 9.0, 1e-3], [0.0, 2.02, 0.1, 8.0, 1e-3], [0.0, 6.0, 0.2, 7.5, 2e-3],
                      [0.0, 8.0, 0.01, 7.2, 1e-3]])
    ev = select.select_events(table, t, 7.0, 10, [])
    assert [e.epoch_bjd for e in ev] == [2.0, 6.0]  # the second overlaps the first; the last has < 3 points
    assert ev[0].points == int(np.count_nonzero(np.abs(t - 2.0) <= 0.05))
