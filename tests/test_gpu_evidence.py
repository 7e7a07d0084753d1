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


def test_compare_search_below_threshold_returns_nothing(gpu, small):
    c, cfg, st, ost = small
    cfg2 = synth.small_config()
    cfg2.threshold = 1e6
    assert gpu.compare_search(st, 1.3, cfg2) == []
    assert oracle.compare_search(ost, 1.3, cfg2) == []
