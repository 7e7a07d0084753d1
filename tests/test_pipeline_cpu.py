"""The search command's host logic (fbls_b200.pipeline) on the CPU, with
every GPU step answered by the oracle (test infrastructure): prepared and
raw inputs of a small curve with one injected signal give a schema-3 report
whose strongest candidate is that signal."""
import dataclasses
import json
import types

import numpy as np
import pytest

import oracle
from fbls_b200 import io, pipeline, synth


class _OracleGpu:
    """The Gpu methods the pipeline calls, on the oracle."""

    class _Dev:
        def __init__(self, state):
            self.state = state
            self.n = state.n

        def free(self):
            pass

    def upload(self, state):
        return self._Dev(state)

    def signal_search(self, state, cfg):
        rows, grid, stats = oracle.signal_search(state, cfg)
        return rows, int(len(grid)), [dict(s) for s in stats]

    def rescore_rows(self, dev, excluded, rows):
        s = dev.state
        return oracle.rescore_rows(s.time, s.v, s.w, excluded, rows, s.origin)

    def count_rows(self, time, excluded, rows):
        return oracle.count_rows(time, excluded, rows)

    def compare_search(self, state, period, cfg):
        return oracle.compare_search(state, period, cfg)

    def compare_batch(self, candidates, cfg, devs=None):
        return [oracle.compare_search(state, period, cfg) for state, period in candidates]

    def single_event_search(self, state, cfg, capacity=131072, dev=None):
        return oracle.single_event_search(state, cfg, capacity)

    def prepare_families(self, time, flux, err, group, cfg):
        return [types.SimpleNamespace(time=t, flux=f, sigma=s, window_days=w, clipped=c, indices=np.array(i))
                for t, f, s, w, c, i in oracle.prepare_families(time, flux, err, group, cfg.durations_days(), cfg)]


def _check(report, c, mode):
    assert report["schema_version"] == 3
    best = report["signal_candidates"][0]
    assert abs(best["period_days"] - c.period) / c.period < 0.01
    assert best["pass"] == 1 and best["events"] >= 2
    assert report["statistics"]["periods_tested"] > 0 and report["statistics"]["passes"]
    assert report["candidates"] and "row" not in best
    text = json.dumps(pipeline._clean(report), default=pipeline._json_default)  # as run_search writes it
    assert json.loads(text)["signal_candidates"][0]["period_days"] == best["period_days"]


def test_prepared_search_on_the_oracle():
    c, cfg = synth.small_curve(), synth.small_config()
    obs = io.Observations(c.time, c.flux, c.flux_err, np.zeros(c.time.shape[0], dtype=np.int64))
    report = pipeline.search_prepared(_OracleGpu(), obs, cfg)
    _check(report, c, "prepared")


def test_raw_search_on_the_oracle():
    c, cfg = synth.small_curve(), synth.small_config()
    cfg = dataclasses.replace(cfg, bin_minutes=0.0)
    flux = 1.0e4 * (1.0 + c.flux)
    obs = io.Observations(c.time, flux, 1.0e4 * c.flux_err, np.zeros(c.time.shape[0], dtype=np.int64))
    report = pipeline.search_transits(_OracleGpu(), obs, cfg)
    _check(report, c, "raw")
    assert report["statistics"]["passes"][0]["families"][0]["window_days"] == 0.4


@pytest.mark.parametrize("argv,message", [
    ([], "usage: python -m fbls_b200 search"),
    (["search"], "--input is required"),
    (["search", "--input", "a.npz", "--output"], "--output needs a value"),
    (["search", "--input", "a.npz", "--pmin", "x"], "could not convert"),
    (["search", "--input", "a.npz", "--bogus"], "unknown argument --bogus"),
    (["search", "--input", "missing.npz"], "missing.npz"),
])
def test_search_command_errors_exit_1_with_a_message(argv, message, capsys, tmp_path, monkeypatch):
    from fbls_b200 import pipeline
    monkeypatch.chdir(tmp_path)
    assert pipeline.main(argv) == 1
    assert message in capsys.readouterr().err


def test_a_search_that_finds_nothing_still_writes_a_schema_3_report():
    """Pure noise under a threshold no row reaches: no candidates, every key
    of the report present, and the JSON writable as run_search writes it."""
    rng = np.random.default_rng(12)
    c, cfg = synth.small_curve(), synth.small_config()
    cfg = dataclasses.replace(cfg, threshold=50.0)
    flux = rng.normal(0.0, 1e-3, c.time.shape[0])
    obs = io.Observations(c.time, flux, c.flux_err, np.zeros(c.time.shape[0], dtype=np.int64))
    report = pipeline.search_prepared(_OracleGpu(), obs, cfg)
    for key in ("schema_version", "software_version", "config", "statistics", "candidates", "signal_candidates",
                "single_events"):
        assert key in report, key
    assert report["schema_version"] == 3
    assert report["signal_candidates"] == [] and report["candidates"] == []
    assert report["statistics"]["periods_tested"] > 0
    text = json.dumps(pipeline._clean(report), default=pipeline._json_default)
    assert json.loads(text)["signal_candidates"] == []


def test_band_plan_of_a_baseline_shorter_than_the_minimum_period_is_empty():
    from fbls_b200 import api
    c, cfg = synth.small_curve(), synth.small_config()
    st = oracle.family_state(c.time[:40], c.flux[:40], c.flux_err[:40], cfg.durations_days())
    assert float(st.time[-1]) < cfg.period_min * 4
    cfg = dataclasses.replace(cfg, period_min=float(st.time[-1]) * 2.0, period_max=float(st.time[-1]) * 4.0,
                              durations_hours=[0.5])
    grid, bands = api.band_plan(st, cfg)
    assert len(grid) == 0 and bands == []
    rows, ogrid, stats = oracle.signal_search(st, cfg)
    assert rows.shape == (0, 5) and len(ogrid) == 0 and stats == []


class _OracleContext(_OracleGpu):
    """api.Gpu's place in run_search: the oracle behind a context manager."""

    def __init__(self, device=0):
        self.device = device

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


@pytest.mark.parametrize("mode", ["raw", "prepared"])
def test_search_command_on_npz_files_with_the_oracle(tmp_path, monkeypatch, mode):
    """run_search end to end on the CPU: NPZ files written by numpy, the
    options, the report and the CSV table; the GPU steps answered by the
    oracle."""
    rng = np.random.default_rng(9)
    t = synth.sector_times(1, 1200.0)
    rel = synth.inject_box(t, rng.normal(0.0, 8e-4, t.shape[0]), 3.3, t[0] + 1.1, 0.15, 4e-3)
    flux = 5.0e3 * (1.0 + 0.002 * np.sin(t / 2.3)) * (1.0 + rel)
    raw, prepared = tmp_path / "star.npz", tmp_path / "prepared.npz"
    np.savez(raw, time_bjd=t, flux=flux, flux_err=np.full(t.shape[0], 4.0), sector=np.full(t.shape[0], 31))
    np.savez(prepared, time_bjd=t, flux=rel, flux_err=np.full(t.shape[0], 8e-4))
    monkeypatch.setattr(pipeline.api, "Gpu", _OracleContext)
    out, table = tmp_path / "report.json", tmp_path / "table.csv"
    args = ["search", "--input", str(raw if mode == "raw" else prepared), "--output", str(out),
            "--save-table", str(table), "--pmax", "6"]
    if mode == "prepared":
        args.append("--prepared")
    assert pipeline.main(args) == 0
    report = json.loads(out.read_text())
    assert report["schema_version"] == 3 and report["input_mode"] == mode
    assert report["input_files"] == [str(raw if mode == "raw" else prepared)]
    assert "period_table" not in report
    best = report["signal_candidates"][0]
    assert abs(best["period_days"] - 3.3) / 3.3 < 0.01
    lines = table.read_text().splitlines()
    assert lines[0] == "period_days,epoch_bjd,duration_days,snr,depth" and len(lines) > 1


def test_candidate_fields_are_the_references():
    # Peak, src/select/peaks.rs:18-45 (`row` is not serialised)
    want = ["period_days", "epoch_bjd", "duration_hours", "snr", "snr_folded", "snr_without_strongest_event",
            "depth", "depth_ppm", "events", "family", "pass", "planet_log_odds", "log_bf_planet_noise",
            "log_bf_binary_noise", "binary_secondary_ratio", "binary_secondary_phase", "binary_odd_even_ratio",
            "binary_period_days", "ingress_fraction", "evidence_epoch_bjd", "evidence_duration_hours",
            "model_preferred", "binary_diagnostics_complete"]
    c, cfg = synth.small_curve(), synth.small_config()
    obs = io.Observations(c.time, c.flux, c.flux_err, np.zeros(c.time.shape[0], dtype=np.int64))
    report = pipeline.search_prepared(_OracleGpu(), obs, cfg)
    assert list(report["signal_candidates"][0].keys()) == want


def test_written_report_keys_are_sorted_at_every_level(tmp_path, monkeypatch):
    """The reference builds the report as a serde_json Value without
    preserve_order (BTreeMap objects), so its file has every object's keys
    in sorted order; run_search writes the same order."""
    c = synth.small_curve()
    path = tmp_path / "p.npz"
    np.savez(path, time_bjd=c.time, flux=c.flux, flux_err=c.flux_err)
    monkeypatch.setattr(pipeline.api, "Gpu", _OracleContext)
    out = tmp_path / "r.json"
    cfg_args = ["--pmin", "0.4", "--pmax", "2.9"]
    assert pipeline.main(["search", "--prepared", "--input", str(path), "--output", str(out)] + cfg_args) == 0
    orders = []
    json.loads(out.read_text(), object_pairs_hook=lambda pairs: orders.append([k for k, _ in pairs]) or dict(pairs))
    assert len(orders) > 5
    assert all(keys == sorted(keys) for keys in orders)


def test_report_config_has_the_reference_fields():
    fields = ["period_min", "period_max", "durations_hours", "threshold"]  # a few, and the whole set below
    c, cfg = synth.small_curve(), synth.small_config()
    obs = io.Observations(c.time, c.flux, c.flux_err, np.zeros(c.time.shape[0], dtype=np.int64))
    report = pipeline.search_prepared(_OracleGpu(), obs, cfg)
    assert all(f in report["config"] for f in fields)
    assert "precision_mode" not in report["config"]  # not a field of the reference's SearchConfig
    assert len(report["config"]) == 36  # config.rs:6-88
    f64 = pipeline.search_prepared(_OracleGpu(), obs, dataclasses.replace(cfg, precision_mode=1))
    assert f64["config"]["precision_mode"] == 1


def test_band_stats_in_the_report_are_the_references_scan_stats():
    from fbls_b200 import _native
    full = _native.ScanStats().as_dict()  # every field the C ABI reports
    assert "tile_rescans" in full
    got = pipeline._scan_stats_json(full)
    assert list(got) == list(pipeline.SCAN_STATS_FIELDS) and "tile_rescans" not in got
