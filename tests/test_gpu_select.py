"""Peak-selection rescoring on the GPU (fbls_rescore_rows, fbls_count_rows)
against the oracle, bit for bit, and select_peaks driven by the GPU against
the same selection driven by the oracle."""
import math

import numpy as np
import pytest

import oracle
from fbls_b200 import api, select, synth

pytestmark = pytest.mark.gpu


def _family():
    c, cfg = synth.single_sector(), synth.single_sector_config()
    return c, cfg, api.prepared_family(c.time, c.flux, c.flux_err, cfg)


def _rows(st, table, rng):
    """Search rows, random rows, rows with an observation on a window edge,
    and rows the windowed walk leaves to the full scan."""
    ta = st.time + st.origin
    rand = np.column_stack([np.exp(rng.uniform(np.log(0.3), np.log(30.0), 300)),
                            rng.uniform(ta[0] - 5.0, ta[-1] + 5.0, 300), rng.uniform(0.01, 0.5, 300)])
    edge = []
    for j in rng.integers(0, ta.shape[0], 100):
        period, duration = rng.uniform(0.5, 9.0), rng.uniform(0.02, 0.3)
        edge.append([period, ta[j] - duration / 2.0 - period * rng.integers(-3, 4), duration])
        edge.append([period, ta[j] + duration / 2.0, duration])
    odd = [[0.0, ta[10], 0.1], [-2.0, ta[10], 0.1], [3.0, math.nan, 0.1], [3.0, ta[10], math.nan],
           [1.0, ta[10], 1.5], [2.0, ta[100], 0.0], [0.004, ta[10], 0.001], [5.0, ta[0] - 1e4, 0.2],
           [math.inf, ta[10], 0.2]]
    return np.vstack([table[:, :3], rand, np.array(edge), np.array(odd)])


def test_rescore_and_count_rows_match_the_oracle(gpu):
    c, cfg, st = _family()
    table = gpu.signal_search(st, cfg)[0]
    rng = np.random.default_rng(8)
    rows = _rows(st, table, rng)
    dev = gpu.upload(st)
    for frac in (0.0, 0.2):
        ex = (rng.uniform(size=st.n) < frac).astype(np.uint8)
        got = gpu.rescore_rows(dev, ex, rows)
        want = oracle.rescore_rows(st.time, st.v, st.w, ex, rows, st.origin)
        assert np.array_equal(got, want, equal_nan=True), np.nonzero(~((got == want) | np.isnan(want)))[0][:5]
        ta = st.time + st.origin
        cnt = gpu.count_rows(ta, ex, rows)
        assert np.array_equal(cnt, oracle.count_rows(ta, ex, rows))
    assert (got[:, 2] > 0).sum() > 100
    dev.free()


class _OracleGpu:
    """The rescoring calls on the oracle (test infrastructure)."""

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


def test_select_peaks_on_the_gpu_is_the_oracle_selection(gpu):
    """Two duration families of a sector with two injected signals; the rows
    of both families' searches go through select_peaks twice (three passes'
    worth of acceptances), once rescored on the GPU and once on the oracle."""
    rng = np.random.default_rng(5)
    c, cfg = synth.single_sector(), synth.single_sector_config()
    flux = synth.inject_box(c.time, c.flux, 5.9, c.time[0] + 1.3, 0.11, 9e-4)
    d = cfg.durations_days()
    states = [api.family_state(c.time, flux, c.flux_err, d[: len(d) // 2]),
              api.family_state(c.time, flux, c.flux_err, d[len(d) // 2:])]
    tables, family = [], []
    for k, s in enumerate(states):
        rows = gpu.signal_search(s, cfg)[0]
        tables.append(rows)
        family += [k] * rows.shape[0]
    table = np.vstack(tables)
    family = np.array(family)
    time_all = np.unique(np.concatenate([s.time + s.origin for s in states]))
    excluded = np.zeros(time_all.shape[0], bool)
    excluded[rng.integers(0, time_all.shape[0], 50)] = True
    got = select.select_peaks(gpu, table, family, states, time_all, cfg.threshold, 10, cfg.min_events, [], excluded, 1)
    want = select.select_peaks(_OracleGpu(), table, family, states, time_all, cfg.threshold, 10, cfg.min_events, [],
                               excluded, 1)
    assert len(got.accepted) >= 2
    assert [p.__dict__ for p in got.accepted] == [p.__dict__ for p in want.accepted]
    assert np.array_equal(got.excluded, want.excluded)
    # the strongest row is the injected sector signal
    assert abs(got.accepted[0].period_days - c.period) / c.period < 0.01
