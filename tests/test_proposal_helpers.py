"""The proposal path's host helpers on the CPU: log-period bands and their
ranges, the ranges the pruned search gets from the band scores (a period is
searched exactly when its band is among the k best), the map's durations
and covered periods, the features' standardisation, recall and labels."""
import math

import numpy as np
import pytest

hypothesis = pytest.importorskip("hypothesis")
from hypothesis import given, settings, strategies as st  # noqa: E402

from fbls_b200 import proposal as pr  # noqa: E402


def test_bands_partition_the_map_range():
    assert pr.band_range(0)[0] == pytest.approx(pr.PMIN, rel=1e-15)
    assert pr.band_range(pr.BANDS - 1)[1] == pytest.approx(pr.PMAX, rel=1e-12)
    for b in range(pr.BANDS):
        lo, hi = pr.band_range(b)
        assert pr.band_of(math.sqrt(lo * hi)) == b
        if b + 1 < pr.BANDS:
            assert pr.band_range(b + 1)[0] == pytest.approx(hi, rel=1e-15)
    assert pr.band_of(pr.PMIN / 10) == 0 and pr.band_of(pr.PMAX * 10) == pr.BANDS - 1
    periods = pr.map_periods()
    assert periods.shape == (pr.T_IN,) and not periods.flags.writeable
    assert np.all(np.diff([pr.band_of(p) for p in periods]) >= 0)


@settings(max_examples=80, deadline=None, derandomize=True)
@given(seed=st.integers(0, 2**31 - 1), k=st.integers(1, 6))
def test_ranges_cover_exactly_the_k_best_bands(seed, k):
    rng = np.random.default_rng(seed)
    logits = rng.normal(size=pr.BANDS)
    best = set(np.argsort(-logits)[:k].tolist())
    ranges = pr.ranges_for(logits, k)
    assert all(lo < hi for lo, hi in ranges)
    assert all(ranges[i][1] <= ranges[i + 1][0] for i in range(len(ranges) - 1))  # sorted, disjoint
    probes = np.exp(rng.uniform(math.log(pr.PMIN / 4), math.log(pr.PMAX * 4), 400))
    for p in probes:
        inside = any(lo <= p < hi for lo, hi in ranges)
        assert inside == (pr.band_of(p) in best), (p, pr.band_of(p), sorted(best))


class _State:
    def __init__(self, durations, rho, t_last):
        self.durations = np.asarray(durations, dtype=np.float64)
        self.rho = np.asarray(rho, dtype=np.float64)
        self.time = np.array([0.0, t_last])


@pytest.mark.parametrize("nd", [1, 2, 3, 4, 5, 20])
def test_map_bank_takes_the_shortest_inner_and_longest_durations(nd):
    d = np.linspace(0.3, 0.02, nd)  # family order need not be sorted
    rho = 1.0 + d
    md, mr = pr.map_bank(_State(d, rho, 100.0))
    assert md.shape == (pr.MAP_CHANNELS,) and mr.shape == (pr.MAP_CHANNELS,)
    assert md[0] == d.min() and md[-1] == d.max() and np.all(np.diff(md) >= 0)
    assert np.array_equal(mr, 1.0 + md)  # rho travels with its duration


def test_map_range_is_the_searched_periods():
    periods = pr.map_periods()
    s = _State([0.05, 0.2], [1.0, 1.0], 27.0)
    i0, i1 = pr.map_range(s, 13.0)
    lo, hi = max(pr.PMIN, 4 * 0.05 * (1 + 1e-9)), 13.0
    assert np.all(periods[i0:i1] >= lo) and np.all(periods[i0:i1] <= hi)
    assert (i0 == 0 or periods[i0 - 1] < lo) and (i1 == pr.T_IN or periods[i1] > hi)
    keep, d, r = pr.map_plan(s, 13.0)
    assert keep.sum() == i1 - i0 and keep[i0:i1].all()
    assert pr.map_range(_State([0.05], [1.0], 0.1), 13.0)[1] == pr.map_range(_State([0.05], [1.0], 0.1), 13.0)[0]


def test_map_features_standardise_the_covered_periods():
    rng = np.random.default_rng(3)
    keep = np.zeros(pr.T_IN, bool)
    keep[100:3000] = True
    m = rng.uniform(0.0, 20.0, (int(keep.sum()), pr.MAP_CHANNELS))  # the map of the covered periods
    x = pr.map_features(m, keep)
    assert x.dtype == np.float32 and x.shape == (pr.MAP_CHANNELS, pr.T_IN)
    assert np.all(x[:, ~keep] == 0.0)
    assert np.allclose(x[:, keep].mean(axis=1), 0.0, atol=1e-5)
    assert np.all(x[:, keep].std(axis=1) < 1.0) and np.all(x[:, keep].std(axis=1) > 0.99)
    few = np.zeros(pr.T_IN, bool)
    few[:7] = True
    assert not pr.map_features(m[:7], few).any()


def test_recall_and_labels():
    logits = np.array([[0.0, 3.0, 1.0] + [0.0] * (pr.BANDS - 3), [5.0, 0.0, 4.0] + [0.0] * (pr.BANDS - 3)])
    y = np.array([2, 0])
    rec = pr.recall_at(logits, y)
    assert rec[0] == 0.5 and rec[1] == 1.0 and rec[-1] == 1.0
    assert pr.recall_at(logits, np.array([-1, -1])).tolist() == [1.0] * pr.BANDS  # no labelled star
    rows = np.array([[1.3, 0.0, 0.1, 8.0, 1e-3], [7.7, 0.0, 0.1, 9.5, 1e-3]])
    assert pr.top_band(rows) == pr.band_of(7.7) and pr.top_band(np.zeros((0, 5))) == -1
