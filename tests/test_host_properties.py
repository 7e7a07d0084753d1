"""Property tests (hypothesis) of the library's host-side code on the CPU:
random arguments through the native period grid, segment edges, detrending
windows and prepared family state must keep the reference's invariants and
equal the oracle where it has the function, and NPY members of random
shapes, dtypes and byte orders must round-trip through the reader."""
import io as pyio
import math

import numpy as np
import pytest

hypothesis = pytest.importorskip("hypothesis")
from hypothesis import given, settings, strategies as st  # noqa: E402

import oracle  # noqa: E402
from fbls_b200 import api, io, select  # noqa: E402

SETTINGS = settings(max_examples=60, deadline=None, derandomize=True)


@SETTINGS
@given(pmin=st.floats(0.05, 5.0), span=st.floats(1.0, 40.0), baseline=st.floats(1.0, 400.0),
       dmin=st.floats(0.005, 0.5), os_=st.floats(0.5, 10.0))
def test_period_grid_drift_bound_and_oracle(pmin, span, baseline, dmin, os_):
    pmax = pmin * span
    g = api.period_grid(pmin, pmax, baseline, dmin, os_)
    assert np.array_equal(g, oracle.period_grid(pmin, pmax, baseline, dmin, os_))
    assert g[0] == pmin and g[-1] == pmax
    assert np.all(np.diff(g) > 0)
    assert np.all(baseline * (g[1:] / g[:-1] - 1.0) <= dmin / os_ * (1.0 + 1e-9))


@SETTINGS
@given(steps=st.lists(st.floats(0.0, 3.0), min_size=1, max_size=60), gap=st.floats(0.1, 2.0))
def test_segment_edges_invariants(steps, gap):
    t = np.cumsum(np.array([0.0] + steps))
    e = api.segment_edges(t, gap)
    assert np.array_equal(e, oracle.segment_edges_py(t, gap))
    assert np.all(e >= 0.0)
    starts = np.concatenate([[0], np.nonzero(np.diff(t) > gap)[0] + 1])
    ends = np.concatenate([starts[1:] - 1, [t.shape[0] - 1]])
    assert np.all(e[starts] == 0.0) and np.all(e[ends] == 0.0)


@SETTINGS
@given(d=st.lists(st.floats(1e-3, 3.0), min_size=1, max_size=24), lo=st.floats(0.05, 1.0),
       factor=st.floats(0.5, 6.0), extra=st.floats(0.0, 5.0))
def test_detrending_windows_invariants(d, lo, factor, extra):
    hi = lo + extra
    w = api.detrending_windows(d, lo, factor, hi)
    windows = [x for x, _ in w]
    assert windows == sorted(set(windows))
    assert all(lo - 1e-6 <= x <= hi + 1e-6 for x in windows)
    members = sorted(i for _, idx in w for i in idx)
    assert members == list(range(len(d)))
    for x, idx in w:
        for i in idx:  # Rust's f64::round: halves away from zero (curve.rs:349-370)
            assert x == select.round_half_away(np.array([min(max(factor * d[i], lo), hi) * 1e6]))[0] / 1e6


@SETTINGS
@given(seed=st.integers(0, 2**31 - 1), n=st.integers(8, 400), cadence=st.floats(1e-3, 0.05),
       gaps=st.integers(0, 3), nan_frac=st.floats(0.0, 0.3), nd=st.integers(1, 6))
def test_family_state_matches_the_oracle_on_random_curves(seed, n, cadence, gaps, nan_frac, nd):
    rng = np.random.default_rng(seed)
    t = 2458000.0 + np.cumsum(rng.uniform(0.5, 1.5, n) * cadence)
    for j in rng.integers(1, n, gaps):
        t[j:] += rng.uniform(0.5, 3.0)
    flux = rng.normal(0.0, 1e-3, n)
    err = rng.uniform(5e-4, 2e-3, n)
    flux[rng.uniform(size=n) < nan_frac] = np.nan
    durations = np.sort(rng.uniform(0.02, 0.5, nd))
    try:
        want = oracle.family_state(t, flux, err, durations)
    except ValueError as e:
        with pytest.raises(api.FblsError, match=str(e)):
            api.family_state(t, flux, err, durations)
        return
    got = api.family_state(t, flux, err, durations)
    for k in ("time", "v", "w", "rho"):
        assert np.array_equal(getattr(got, k), getattr(want, k)), k
    assert got.baseline_norm == want.baseline_norm and got.origin == want.origin
    assert np.all(np.diff(got.time) >= 0) and got.time[0] == 0.0


_DTYPES = ["<f8", ">f8", "<f4", ">f4", "<i8", ">i8", "<i4", ">i4", "<i2", ">i2", "|u1", "|b1"]


@SETTINGS
@given(dtype=st.sampled_from(_DTYPES), shape=st.lists(st.integers(0, 5), min_size=0, max_size=3),
       seed=st.integers(0, 2**31 - 1))
def test_npy_round_trip(dtype, shape, seed):
    rng = np.random.default_rng(seed)
    size = int(math.prod(shape))
    if dtype.endswith("b1"):
        a = rng.integers(0, 2, size).astype(bool)
    elif "f" in dtype:
        a = rng.normal(size=size).astype(np.dtype(dtype))
    else:
        info = np.iinfo(np.dtype(dtype).newbyteorder("="))
        a = rng.integers(info.min, info.max, size, endpoint=True, dtype=np.int64).astype(np.dtype(dtype))
    a = a.reshape(shape)
    buf = pyio.BytesIO()
    np.save(buf, a)
    got = io.parse_npy(buf.getvalue())
    assert got.shape == tuple(shape)
    assert np.array_equal(got.data, a.astype(np.float64).reshape(-1))


def test_detrending_window_halves_round_away_from_zero():
    # 1.03125 x 0.25 d = 0.2578125 d: 257812.5 micro-days rounds to 257813, as Rust's f64::round does
    assert api.detrending_windows([0.25], 0.25, 1.03125, 1.25)[0][0] == 0.257813


@SETTINGS
@given(seed=st.integers(0, 2**31 - 1), n=st.integers(2, 600), sectors=st.integers(1, 3),
       bin_minutes=st.sampled_from([0.0, 0.0, 2.0, 10.0, 30.0]), with_err=st.booleans(),
       nan_frac=st.floats(0.0, 0.2), gap=st.floats(0.1, 1.5))
def test_noise_fit_matches_the_oracle_on_random_raw_curves(seed, n, sectors, bin_minutes, with_err, nan_frac, gap):
    rng = np.random.default_rng(seed)
    t = 1000.0 + np.cumsum(rng.uniform(0.2, 1.8, n) * (2.0 / 1440.0))
    sec = np.sort(rng.integers(0, sectors, n)).astype(np.int64) + 5
    t += (sec - 5) * 30.0
    level = 1e4 * (1.0 + 0.1 * (sec - 5))
    flux = level * (1.0 + rng.normal(0.0, 1e-3, n))
    flux[rng.uniform(size=n) < nan_frac] = np.nan
    err = level * rng.uniform(5e-4, 2e-3, n) if with_err else None
    try:
        want = oracle.fit_segment_noise_raw(t, flux, err, sec, bin_minutes, gap)
    except ValueError as e:
        with pytest.raises(api.FblsError, match=str(e)):
            api.fit_segment_noise(t, flux, err, sec, bin_minutes, gap)
        return
    got = api.fit_segment_noise(t, flux, err, sec, bin_minutes, gap)
    assert np.array_equal(got.time, want[0])
    assert np.array_equal(got.deficit, want[1])
    assert np.array_equal(got.variance, want[2])
    assert np.array_equal(got.group, want[3])
    assert (got.origin, got.inflation, got.segments) == want[4:]
