"""bench.py's helpers that need no GPU: the proposal network's FLOP count
and the peak lookups' fallbacks."""
import bench
from fbls_b200 import proposal as pr


def test_network_flops_counts_the_convolution_gemms():
    # 4 -> 64 channels at T 8192, then 64 -> 64 at 4096, 2048 and three times
    # at 1024 (pools 2, 2, 2, 1, 1, 1); kernel 7
    want = 2 * 64 * 7 * (4 * 8192 + 64 * 4096 + 64 * 2048 + 3 * 64 * 1024)
    assert bench._network_flops(1) == want == 557_842_432
    assert bench._network_flops(512) == 512 * want
    assert pr.T_IN == 8192 and pr.POOLS == (2, 2, 2, 1, 1, 1)


def test_peaks_fall_back_without_the_measured_file(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench._peaks() == (6650.0, "fallback")
    assert bench._bf16_peak() == (1590.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text('{"hbm_gbs": 7000.0, "bf16_tflops": 1600.0}')
    assert bench._peaks() == (7000.0, "measured")
    assert bench._bf16_peak() == (1600.0, "measured")


def _reference_arm(env_extra, tmp_path):
    import os
    import subprocess
    import sys
    root = bench.ROOT
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, str(root / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup",
                           "1", "--cpu-seconds", "0.5", "--workload", "single_sector"],
                          capture_output=True, text=True, env=env, timeout=600, cwd=tmp_path)


def test_reference_arm_prints_one_contract_line(tmp_path):
    import json
    r = _reference_arm({"RANK": "0", "WORLD_SIZE": "1"}, tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["unit"] == d["unit"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    assert "single_sector" in d["config"]["workload"]


def test_reference_arm_is_silent_on_other_ranks(tmp_path):
    r = _reference_arm({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, tmp_path)
    assert r.returncode == 0 and r.stdout.strip() == ""
