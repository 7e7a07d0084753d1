"""The CUDA path against the committed golden fixtures (tests/golden/, the
oracle's frozen outputs on seeded small inputs), through the C ABI: every
band's scan at the coarse and the full phase-bin count in both precision
modes, signal_search, model comparison at five periods, rescoring and
counting of 1,046 rows with and without excluded points, the single-event
scan and the biweight detrend. The same checks pin the oracle to these files
on the CPU (test_golden.py)."""
import pytest

import _golden
from fbls_b200 import api

pytestmark = pytest.mark.gpu

EVIDENCE_RTOL = 1e-9     # SNR and depth, relative (with a 1e-12 absolute floor)
EVIDENCE_LOG_ATOL = 1e-9  # log-evidences, absolute times max(1, |x|)


@pytest.fixture(scope="module")
def golden():
    arrays, meta, cfg = _golden.load()
    st = api.prepared_family(arrays["input_time"], arrays["input_flux"], arrays["input_flux_err"], cfg)
    return arrays, meta, cfg, st


def test_scan_bands_match_the_fixture(gpu, golden):
    arrays, meta, cfg, st = golden
    _golden.check_scan_bands(gpu, st, arrays, meta, cfg)


def test_signal_search_matches_the_fixture(gpu, golden):
    arrays, meta, cfg, st = golden
    _golden.check_signal_search(gpu, st, arrays, meta, cfg)


def test_model_comparison_matches_the_fixture(gpu, golden):
    arrays, meta, cfg, st = golden
    _golden.check_evidence(gpu, st, meta, cfg, rtol=EVIDENCE_RTOL, log_atol=EVIDENCE_LOG_ATOL, atol=1e-12)


def test_rescoring_matches_the_fixture(gpu, golden):
    arrays, meta, cfg, st = golden
    _golden.check_rescore(gpu, st, arrays)


def test_single_events_match_the_fixture(gpu, golden):
    arrays, meta, cfg, st = golden
    est = api.family_state(arrays["event_time"], arrays["event_flux"], arrays["event_flux_err"],
                           cfg.durations_days())
    _golden.check_single_events(gpu, est, arrays, meta, cfg)


def test_detrend_matches_the_fixture(gpu, golden):
    arrays, meta, cfg, st = golden
    _golden.check_detrend(gpu, arrays, meta)
