"""Property tests (hypothesis) of the peak-selection host helpers on the
CPU: transit masks against the oracle's C restatement of the reference's
(curve.rs:572-585), f64::round and f64::rem_euclid against exact decimal
arithmetic, and event counts against a literal loop over the observations
(peaks.rs:65-82)."""
from decimal import ROUND_HALF_UP, Decimal
import math

import numpy as np
import pytest

hypothesis = pytest.importorskip("hypothesis")
from hypothesis import given, settings, strategies as st  # noqa: E402

import oracle  # noqa: E402
from fbls_b200 import select  # noqa: E402

SETTINGS = settings(max_examples=80, deadline=None, derandomize=True)
finite = st.floats(-1e6, 1e6, allow_nan=False, allow_infinity=False)


@SETTINGS
@given(seed=st.integers(0, 2**31 - 1), n=st.integers(1, 500), period=st.floats(0.05, 50.0),
       epoch=st.floats(-1e4, 3e6), duration=st.floats(0.0, 2.0), margin=st.floats(0.0, 2.0))
def test_transit_mask_is_the_oracles(seed, n, period, epoch, duration, margin):
    rng = np.random.default_rng(seed)
    t = np.sort(epoch + rng.uniform(-200.0, 200.0, n))
    assert np.array_equal(select.transit_mask(t, period, epoch, duration, margin),
                          oracle.transit_mask(t, period, epoch, duration, margin))


@SETTINGS
@given(x=st.lists(finite, min_size=1, max_size=50))
def test_round_half_away_is_exact(x):
    got = select.round_half_away(np.array(x))
    want = [float(Decimal(v).quantize(Decimal(1), rounding=ROUND_HALF_UP)) for v in x]  # halves away from zero
    assert np.array_equal(got, np.array(want))
    assert np.array_equal(np.signbit(got), np.signbit(np.array(want)))  # round(-0.4) is -0.0, as in Rust


@SETTINGS
@given(x=st.lists(finite, min_size=1, max_size=50), m=st.floats(1e-3, 1e3))
def test_rem_euclid_is_in_range_and_congruent(x, m):
    xs = np.array(x)
    for mm in (m, -m):
        r = select.rem_euclid(xs, mm)
        assert np.all(r >= 0.0) and np.all(r <= abs(mm))
        # the reference's value: fmod, then |m| added to a negative remainder (exactly as f64 arithmetic does)
        want = [math.fmod(v, mm) + abs(mm) if math.fmod(v, mm) < 0 else math.fmod(v, mm) for v in x]
        assert np.array_equal(r, np.array(want))


@SETTINGS
@given(seed=st.integers(0, 2**31 - 1), n=st.integers(0, 300), period=st.floats(0.3, 10.0),
       duration=st.floats(0.01, 0.5), minimum=st.integers(1, 5))
def test_event_count_is_the_loop(seed, n, period, duration, minimum):
    rng = np.random.default_rng(seed)
    t = np.sort(rng.uniform(0.0, 30.0, n))
    epoch = float(rng.uniform(0.0, period))
    per_cycle = {}
    for x in t:
        phase = math.fmod((x - epoch) + period / 2.0, period)
        phase = (phase + period if phase < 0 else phase) - period / 2.0
        if abs(phase) <= duration / 2.0:
            q = (x - epoch) / period
            c = math.trunc(q) + (math.copysign(1.0, q) if abs(q - math.trunc(q)) >= 0.5 else 0.0)
            per_cycle[c] = per_cycle.get(c, 0) + 1
    want = sum(1 for v in per_cycle.values() if v >= minimum)
    assert select.event_count(t, period, epoch, duration, minimum) == want
