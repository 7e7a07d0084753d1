"""Parity of the CUDA evidence (model comparison) path with the oracle.

Evidence values are f64 sums of logs of erfc / exp terms; the device's exp
and log differ from the host's by a few ulps, so log-evidences are compared
to 1e-9 absolute and SNR / depth to 1e-9 relative, indices exactly.
"""
import math

import numpy as np
import pytest

import oracle
from fbls_b200 import api, synth

pytestmark = pytest.mark.gpu

LOG_ATOL = 1e-9
RTOL = 1e-9


def _check_rows(g, o):
    assert len(g) == len(o)
    for gr, orr in zip(g, o):
        assert gr["selection_flags"] == orr["selection_flags"]
        for k in ("period", "epoch", "duration", "ingress_fraction"):
            assert gr[k] == orr[k], k
        for k in ("snr", "depth"):
            assert gr[k] == pytest.approx(orr[k], rel=RTOL), k
        for k in ("planet_log_odds", "log_bf_planet_noise", "log_bf_binary_noise"):
            assert abs(gr[k] - orr[k]) <= LOG_ATOL * max(1.0, abs(orr[k])), k
        for k in ("binary_secondary_ratio", "binary_secondary_phase", "binary_odd_even_ratio", "binary_period_days"):
            if math.isnan(orr[k]):
                assert math.isnan(gr[k]), k
            else:
                assert gr[k] == orr[k], k


def _same_rows(a, b):
    """Bit-identical rows (NaN fields equal to NaN)."""
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert x.keys() == y.keys()
        assert np.array_equal(np.array([float(x[k]) for k in x]), np.array([float(y[k]) for k in y]), equal_nan=True)


@pytest.fixture(scope="module")
def small():
    c = synth.small_curve()
    cfg = synth.small_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    ost = oracle.family_state(c.time, c.flux, c.flux_err, cfg.durations_days())
    return c, cfg, st, ost


@pytest.mark.parametrize("period", [1.3, 1.30481313, 0.9, 2.6, 1.95])
def test_compare_search_parity_small(gpu, small, period):
    c, cfg, st, ost = small
    g = gpu.compare_search(st, period, cfg)
    o = oracle.compare_search(ost, period, cfg)
    _check_rows(g, o)


def test_compare_search_finds_the_injected_box(gpu, small):
    c, cfg, st, ost = small
    rows = gpu.compare_search(st, c.period, cfg)
    assert rows, "the injected box must pass the evidence screen"
    r = rows[0]
    assert r["log_bf_planet_noise"] > 10.0
    phase = ((r["epoch"] - c.epoch) / c.period + 0.5) % 1.0 - 0.5
    assert abs(phase * c.period) < c.duration


def test_compare_search_single_sector(gpu):
    c = synth.single_sector()
    cfg = synth.single_sector_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    ost = oracle.family_state(c.time, c.flux, c.flux_err, cfg.durations_days())
    for period in (c.period, 2.0 * c.period, 5.123):
        _check_rows(gpu.compare_search(st, period, cfg), oracle.compare_search(ost, period, cfg))


@pytest.fixture(scope="module")
def multi():
    c = synth.multi_sector()
    cfg = synth.multi_sector_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    ost = oracle.family_state(c.time, c.flux, c.flux_err, cfg.durations_days())
    return c, cfg, st, ost


@pytest.mark.parametrize("factor", [1.0, 2.0, 0.5])
def test_compare_search_parity_thirteen_sectors(gpu, multi, factor):
    # The 13-sector star at its injected 17.3 d period (nb 3,324, 2 nb 6,648,
    # 52 tiles: prefix rows read from global memory), and at 2x and 1/2x.
    c, cfg, st, ost = multi
    period = c.period * factor
    g = gpu.compare_search(st, period, cfg)
    o, diag = oracle.compare_search(ost, period, cfg, diag=True)
    _check_rows(g, o)
    if factor == 1.0:
        assert int(diag["nb"]) == 3324 and int(diag["tiles"]) == 52
        assert g, "the injected box must pass the evidence screen"


def test_compare_batch_equals_one_call_per_candidate(gpu, multi, small):
    # Candidates of three families in one batch (every launch class: staged
    # rows of a few KB, of ~160 KB and rows left in global memory) against one
    # compare_search each and against the oracle.
    c, cfg, st, ost = multi
    cs, cfgs, sst, sost = small
    rows, _, _ = gpu.signal_search(st, cfg)
    order = np.argsort(-rows[:, 3])
    periods = []
    for i in order:
        p = float(rows[i, 0])
        if all(abs(p - q) > 1e-3 * q for q in periods):
            periods.append(p)
        if len(periods) == 12:
            break
    periods += [c.period, 1.7, 3.1]
    cands = [(st, p) for p in periods]
    got = gpu.compare_batch(cands, cfg)
    for (s_, p), g in zip(cands, got):
        _same_rows(g, gpu.compare_search(s_, p, cfg))
        _check_rows(g, oracle.compare_search(ost, p, cfg))
    # the small star has its own config: a second batch with both stars' bands
    got_small = gpu.compare_batch([(sst, 1.3), (sst, 0.9), (sst, 2.6)], cfgs)
    for p, g in zip((1.3, 0.9, 2.6), got_small):
        _check_rows(g, oracle.compare_search(sost, p, cfgs))


def test_compare_batch_on_masked_families(gpu, multi):
    # The pipeline masks the other peaks out of each candidate's family, so a
    # batch holds several families of different lengths.
    c, cfg, st, ost = multi
    rng = np.random.default_rng(11)
    cands, ocands = [], []
    for k in range(4):
        centre = c.time[0] + rng.uniform(0.0, c.time[-1] - c.time[0])
        keep = np.abs(c.time - centre) > 0.5 + 0.5 * k
        s_ = api.prepared_family(c.time[keep], c.flux[keep], c.flux_err[keep], cfg)
        o_ = oracle.family_state(c.time[keep], c.flux[keep], c.flux_err[keep], cfg.durations_days())
        p = c.period * (1.0 + 0.01 * k)
        cands.append((s_, p))
        ocands.append((o_, p))
    got = gpu.compare_batch(cands, cfg)
    for g, (o_, p) in zip(got, ocands):
        _check_rows(g, oracle.compare_search(o_, p, cfg))


def test_compare_search_below_threshold_returns_nothing(gpu, small):
    c, cfg, st, ost = small
    cfg2 = synth.small_config()
    cfg2.threshold = 1e6
    assert gpu.compare_search(st, 1.3, cfg2) == []
    assert oracle.compare_search(ost, 1.3, cfg2) == []
