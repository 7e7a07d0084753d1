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
