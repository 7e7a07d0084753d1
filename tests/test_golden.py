"""The golden fixtures on the CPU: the oracle against the reference's own
known-answer values (read from its test sources into
golden/reference_kats.json), the oracle's outputs pinned to the frozen
golden/oracle_small.* (so a change of the oracle fails here before a GPU test
compares the CUDA path with the same files), and the library's host-side
preparation and band planning against the same fixtures."""
import numpy as np
import pytest

import _golden
import oracle
from fbls_b200 import api


@pytest.fixture(scope="module")
def golden():
    return _golden.load()


ERFC = _golden.reference_kats()["erfc"]


def test_erfc_table_is_complete():
    assert len(ERFC["cases"]) == 16 and ERFC["rel_tol"] == 1e-14


@pytest.mark.parametrize("x,want", ERFC["cases"])
def test_erfc_against_the_reference_table(x, want):
    assert abs((oracle.erfc(x) - want) / want) < ERFC["rel_tol"]


def test_period_grid_against_the_reference_property():
    kat = _golden.reference_kats()["period_grid"]
    lo, hi, baseline, dmin, os_ = kat["args"]
    for g in (oracle.period_grid(lo, hi, baseline, dmin, os_), api.period_grid(lo, hi, baseline, dmin, os_)):
        assert g[0] == lo and g[-1] == hi
        assert np.all(baseline * (g[1:] / g[:-1] - 1.0) <= dmin / os_ * (1.0 + kat["drift_slack"]))


def test_segment_edges_and_windows_against_the_reference_cases():
    kat = _golden.reference_kats()
    e = kat["segment_edges"]
    assert api.segment_edges(e["time"], e["gap"]).tolist() == e["want"]
    assert oracle.segment_edges_py(np.array(e["time"]), e["gap"]).tolist() == e["want"]
    w = kat["detrending_windows"]
    got = api.detrending_windows(w["durations"], *w["args"])
    assert got[0] == (w["first"][0], w["first"][1])
    for index, days in w["window_days"]:
        assert got[index][0] == days


def test_fixture_config_is_the_small_workload(golden):
    arrays, meta, cfg = golden
    assert _golden.config_is_the_small_workload(meta)


def test_library_preparation_and_bands_match_the_fixture(golden):
    arrays, meta, cfg = golden
    st = api.prepared_family(arrays["input_time"], arrays["input_flux"], arrays["input_flux_err"], cfg)
    for k in ("time", "v", "w", "durations", "rho"):
        assert np.array_equal(getattr(st, k), arrays["state_" + k]), k
    for k, v in meta["state"].items():
        assert getattr(st, k) == v, k
    grid, bands = api.band_plan(st, cfg)
    assert len(grid) == meta["grid_len"] and len(bands) == len(meta["bands"])
    for b, band in enumerate(bands):
        assert band["nb"] == meta["bands"][b]["nb"]
        for k in ("periods", "durations", "rho"):
            assert np.array_equal(band[k], arrays[f"b{b}_{k}"]), (b, k)


def _oracle_state(arrays, cfg):
    return oracle.family_state(arrays["input_time"], arrays["input_flux"], arrays["input_flux_err"],
                               cfg.durations_days())


def test_oracle_scan_is_pinned(golden):
    arrays, meta, cfg = golden
    st = _oracle_state(arrays, cfg)
    _golden.check_scan_bands(_golden.OracleGpu(), st, arrays, meta, cfg)
    _golden.check_signal_search(_golden.OracleGpu(), st, arrays, meta, cfg)


def test_oracle_evidence_is_pinned(golden):
    arrays, meta, cfg = golden
    _golden.check_evidence(_golden.OracleGpu(), _oracle_state(arrays, cfg), meta, cfg)


def test_oracle_rescoring_events_and_detrend_are_pinned(golden):
    arrays, meta, cfg = golden
    gpu = _golden.OracleGpu()
    _golden.check_rescore(gpu, _oracle_state(arrays, cfg), arrays)
    est = oracle.family_state(arrays["event_time"], arrays["event_flux"], arrays["event_flux_err"],
                              cfg.durations_days())
    _golden.check_single_events(gpu, est, arrays, meta, cfg)
    _golden.check_detrend(gpu, arrays, meta)


def test_a_planted_oracle_change_fails_the_pin(golden):
    """The pin notices a one-ulp change of one score (planted in the fixture
    copy, on the CPU)."""
    arrays, meta, cfg = golden
    bad = dict(arrays)
    key = "b2_nb372_m0_score"
    s = bad[key].copy()
    i = int(np.flatnonzero(np.isfinite(s))[0])
    s[i] = np.nextafter(s[i], np.inf)
    bad[key] = s
    with pytest.raises(AssertionError):
        _golden.check_scan_bands(_golden.OracleGpu(), _oracle_state(arrays, cfg), bad, meta, cfg)
