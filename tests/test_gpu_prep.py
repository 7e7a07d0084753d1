"""Biweight detrending on the GPU (fbls_biweight_flatten) against the
oracle's form of the reference's kernel, bit for bit."""
import numpy as np
import pytest

import oracle
from fbls_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed,window,iterations,ties", [(1, 0.5, 10, False), (2, 1.5, 3, True), (3, 0.05, 10, False)])
def test_biweight_matches_the_oracle(gpu, seed, window, iterations, ties):
    rng = np.random.default_rng(seed)
    n = 3000
    t = np.sort(np.concatenate([rng.uniform(0.0, 5.0, n // 2), rng.uniform(5.7, 11.0, n - n // 2)]))
    f = 0.004 * np.sin(1.3 * t) + rng.normal(0.0, 1e-3, n)
    f[rng.integers(0, n, 20)] += 0.03
    if ties:
        f = np.round(f, 4)
    got = gpu.biweight_flatten(t, f, window, gap=0.5, iterations=iterations)
    want = oracle.biweight_flatten(t, f, window, gap=0.5, iterations=iterations)
    assert np.array_equal(got, want)


def test_biweight_on_a_sector(gpu):
    """A TESS-like sector at 10-minute cadence with a 0.75 d window."""
    c = synth.small_curve(days=27.0, cadence_s=600.0)
    t = c.time - c.time[0]
    got = gpu.biweight_flatten(t, c.flux, 0.75)
    want = oracle.biweight_flatten(t, c.flux, 0.75)
    assert np.array_equal(got, want)


def test_biweight_removes_a_smooth_trend(gpu):
    # the reference's known-answer test, curve.rs:624-634
    t = np.arange(2000) * 0.01
    flat = gpu.biweight_flatten(t, 0.01 * np.sin(t / 5.0), 0.5, 0.5, 5.0, 10)
    assert np.abs(flat[100:1900]).max() < 5e-5


def test_prepare_families_matches_the_oracle(gpu):
    """Raw flux of two sectors with their own levels, NaNs and a sector label
    each, binned to 30 minutes: every detrended family equal to the oracle's."""
    from fbls_b200.config import SearchConfig
    rng = np.random.default_rng(2)
    t = synth.sector_times(2, 600.0)
    sec = np.floor((t - t[0]) / synth.SECTOR_DAYS).astype(np.int64) + 17
    level = 1.2e4 * (1.0 + 0.05 * (sec - 17))
    flux = level * (1.0 + 2e-3 * np.sin(t / 1.7) + rng.normal(0.0, 8e-4, t.shape[0]))
    flux[rng.integers(0, t.shape[0], 40)] *= 1.02  # positive outliers to clip
    err = np.full(t.shape[0], 8e-4) * level
    cfg = SearchConfig(bin_minutes=30.0, durations_hours=[0.5, 1.0, 2.0, 6.0, 14.0])
    got = gpu.prepare_families(t, flux, err, sec, cfg)
    want = oracle.prepare_families(t, flux, err, sec, cfg.durations_days(), cfg)
    assert len(got) == len(want) >= 3
    for g, w in zip(got, want):
        assert np.array_equal(g.time, w[0]) and np.array_equal(g.flux, w[1]) and np.array_equal(g.sigma, w[2])
        assert (g.window_days, g.clipped, g.indices.tolist()) == (w[3], w[4], w[5])
    assert any(g.clipped > 0 for g in got)
