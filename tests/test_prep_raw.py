"""Raw-mode preparation (src/prep/curve.rs:89-198, :202-250, :332-425) on the
CPU: the reference's own known-answer tests (noise model, detrending
windows, segment edges, smooth-trend removal) against the library and the
oracle, and the library's noise model with sector groups and bins against the
oracle's restatement."""
import numpy as np
import pytest

import oracle
from fbls_b200 import api, synth


def test_reference_noise_model_kat():
    # curve.rs:636-661
    n = 500
    t = 1000.0 + np.arange(n) * 0.01
    f = 2000.0 + 3.0 * np.sin(np.arange(n) * 1.7)
    m = api.fit_segment_noise(t, f, np.ones(n), None, 0.0, 0.75)
    assert m.origin == 1000.0 and m.time[0] == 0.0
    median = np.sort(f)[(n - 1) // 2]
    assert abs(m.deficit[0] - (1.0 - f[0] / median)) < 1e-12
    assert m.inflation > 2.0 and m.segments == 1


def test_reference_windows_and_edges_kat():
    # curve.rs:609-622
    d = [0.5 / 24.0, 1.0 / 24.0, 2.0 / 24.0, 12.0 / 24.0, 40.0 / 24.0]
    w = api.detrending_windows(d, 0.4, 3.0, 3.5)
    assert w[0] == (0.4, [0, 1, 2]) and w[1][0] == 1.5 and w[2][0] == 3.5
    assert api.segment_edges([0.0, 1.0, 2.0, 10.0, 10.2], 1.5).tolist() == [0.0, 1.0, 0.0, 0.0, 0.0]


def test_reference_biweight_trend_kat():
    # curve.rs:624-634, on the oracle's forms of the reference
    t = np.arange(2000) * 0.01
    trend = 0.01 * np.sin(t / 5.0)
    for sorted_medians in (False, True):
        flat = oracle.biweight_flatten(t, trend, 0.5, 0.5, 5.0, 10, sorted_medians=sorted_medians)
        assert np.abs(flat[100:1900]).max() < 5e-5


def _raw(seed=2, sectors=2, cadence_s=600.0):
    rng = np.random.default_rng(seed)
    t = synth.sector_times(sectors, cadence_s)
    sec = np.floor((t - t[0]) / synth.SECTOR_DAYS).astype(np.int64) + 17
    level = 1.2e4 * (1.0 + 0.05 * (sec - 17))
    flux = level * (1.0 + 2e-3 * np.sin(t / 1.7) + rng.normal(0.0, 8e-4, t.shape[0]))
    err = np.full(t.shape[0], 8e-4) * level
    flux[rng.integers(0, t.shape[0], 10)] = np.nan
    return t, flux, err, sec


@pytest.mark.parametrize("bin_minutes,with_err", [(0.0, True), (30.0, True), (20.0, False)])
def test_noise_model_with_groups_and_bins_matches_the_oracle(bin_minutes, with_err):
    t, flux, err, sec = _raw()
    e = err if with_err else None
    got = api.fit_segment_noise(t, flux, e, sec, bin_minutes, 0.75)
    want = oracle.fit_segment_noise_raw(t, flux, e, sec, bin_minutes, 0.75)
    assert np.array_equal(got.time, want[0])
    assert np.array_equal(got.deficit, want[1])
    assert np.array_equal(got.variance, want[2])
    assert np.array_equal(got.group, want[3])
    assert (got.origin, got.inflation, got.segments) == want[4:]
    assert got.segments >= 2  # the sector boundary and the mid-sector gaps
