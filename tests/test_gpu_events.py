"""Single-event scan (src/search/events.rs:18-153, scan_all kernels.rs:851-921)
on the GPU against the oracle: the same rows, bit for bit, in (phase,
duration, shape) order, and the same stats."""
import dataclasses

import numpy as np
import pytest

import oracle
from fbls_b200 import api, synth

pytestmark = pytest.mark.gpu


def _single_event_curve(days, cadence_s, seed):
    """A curve with one deep transit-like dip (a single event) and noise."""
    rng = np.random.default_rng(seed)
    t = synth.T0 + np.arange(int(days * 86400 / cadence_s)) * cadence_s / 86400.0
    flux = rng.normal(0.0, 1e-3, t.shape[0])
    mid = synth.T0 + 0.37 * days
    flux[np.abs(t - mid) <= 0.06] -= 4e-3
    return t, flux, np.full_like(t, 1e-3), mid


@pytest.mark.parametrize("days,cadence_s,hours", [(6.0, 600.0, None), (27.0, 120.0, None),
                                                 (60.0, 600.0, [0.5, 1.0, 2.5])])
def test_single_event_search_matches_the_oracle(gpu, days, cadence_s, hours):
    """nb 770, 3,500 (the walking fold) and 11,600 (the staged fold)."""
    t, flux, err, mid = _single_event_curve(days, cadence_s, 3)
    cfg = synth.small_config()
    if hours:
        cfg = dataclasses.replace(cfg, durations_hours=hours)
    st = api.family_state(t, flux, err, cfg.durations_days())
    ost = oracle.family_state(t, flux, err, cfg.durations_days())
    rows, stats = gpu.single_event_search(st, cfg)
    want, wstats = oracle.single_event_search(ost, cfg)
    assert stats == wstats
    assert rows.shape[0] > 0
    assert np.array_equal(rows, want)
    best = rows[np.argmax(rows[:, 3])]
    assert abs(best[1] - mid) < 0.1 and np.isinf(best[0])


def test_single_event_overflow_drops_rows(gpu):
    t, flux, err, _ = _single_event_curve(6.0, 600.0, 4)
    cfg = synth.small_config()
    st = api.family_state(t, flux, err, cfg.durations_days())
    rows, stats = gpu.single_event_search(st, cfg)
    assert stats["threshold_survivors"] > 2
    small, sstats = gpu.single_event_search(st, cfg, capacity=2)
    assert small.shape[0] == 0 and sstats["overflow"] and sstats["threshold_survivors"] == stats["threshold_survivors"]
