"""The search command end to end (src/pipeline.rs, src/main.rs): raw NPZ
input of two sectors with one injected transit, and the same star as a
prepared curve, through `python -m fbls_b200 search`'s code path."""
import json

import numpy as np
import pytest

from fbls_b200 import pipeline, synth

pytestmark = pytest.mark.gpu


def _raw_star(tmp_path):
    rng = np.random.default_rng(9)
    t = synth.sector_times(2, 600.0)
    sec = np.where(t - t[0] < synth.SECTOR_DAYS, 31, 32)
    rel = synth.inject_box(t, rng.normal(0.0, 8e-4, t.shape[0]), 3.3, t[0] + 1.1, 0.12, 3e-3)
    flux = 5.0e3 * (1.0 + 0.002 * np.sin(t / 2.3)) * (1.0 + rel)
    path = tmp_path / "star.npz"
    np.savez(path, time_bjd=t, flux=flux, flux_err=np.full(t.shape[0], 4.0), sector=sec)
    prepared = tmp_path / "prepared.npz"
    np.savez(prepared, time_bjd=t, flux=rel, flux_err=np.full(t.shape[0], 8e-4))
    return path, prepared


@pytest.mark.parametrize("mode", ["raw", "prepared"])
def test_search_command_finds_the_injected_signal(gpu, tmp_path, mode):
    raw, prepared = _raw_star(tmp_path)
    out, table = tmp_path / "report.json", tmp_path / "table.csv"
    args = ["search", "--input", str(raw if mode == "raw" else prepared), "--output", str(out),
            "--save-table", str(table), "--pmax", "12"]
    if mode == "prepared":
        args.append("--prepared")
    assert pipeline.main(args) == 0
    report = json.loads(out.read_text())
    assert report["schema_version"] == 3 and report["input_mode"] == mode
    assert "period_table" not in report
    best = report["signal_candidates"][0]
    assert abs(best["period_days"] - 3.3) / 3.3 < 0.01
    assert best["events"] >= 2 and best["pass"] == 1
    assert report["statistics"]["periods_tested"] > 0
    assert table.read_text().startswith("period_days,epoch_bjd,duration_days,snr,depth\n")
