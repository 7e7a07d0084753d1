"""Biweight detrending (src/prep/curve.rs:202-329, kernels.rs:1051-1110) on
the CPU: the oracle's two forms of the reference (bisection medians as its
GPU kernel, sorted medians as its CPU function) agree, and the detrend
removes a smooth trend."""
import numpy as np

import oracle


def _curve(seed, n=1200, ties=False):
    rng = np.random.default_rng(seed)
    t = np.sort(np.concatenate([rng.uniform(0.0, 4.0, n // 2), rng.uniform(4.8, 9.0, n - n // 2)]))
    f = 0.004 * np.sin(1.3 * t) + rng.normal(0.0, 1e-3, n)
    f[rng.integers(0, n, 15)] += 0.03
    if ties:
        f = np.round(f, 4)
    return t, f


def test_bisection_and_sorted_medians_agree():
    for seed, ties in ((1, False), (2, True)):
        t, f = _curve(seed, ties=ties)
        a = oracle.biweight_flatten(t, f, 0.5, gap=0.5, iterations=5)
        b = oracle.biweight_flatten(t, f, 0.5, gap=0.5, iterations=5, sorted_medians=True)
        assert np.array_equal(a, b)


def test_detrend_removes_the_trend():
    t, f = _curve(3)
    out = oracle.biweight_flatten(t, f, 0.5, gap=0.5, iterations=5)
    clean = np.abs(out) < 0.02
    assert np.std(out[clean]) < 1.5e-3 < np.std(f)
    const = oracle.biweight_flatten(t, np.zeros_like(t), 0.5)
    assert np.all(const == 0.0)
