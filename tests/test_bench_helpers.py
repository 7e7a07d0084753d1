"""bench.py's helpers that need no GPU: the proposal network's FLOP count
and the peak lookups' fallbacks."""
import bench
from fbls_b200 import proposal as pr


def test_network_flops_counts_the_convolution_gemms():
    # 4 -> 32 channels at T 4096, then 32 -> 32 at 2048, 1024, 512; kernel 7
    want = 2 * 32 * 7 * (4 * 4096 + 32 * 2048 + 32 * 1024 + 32 * 512)
    assert bench._network_flops(1) == want == 58_720_256
    assert bench._network_flops(512) == 512 * want
    assert pr.T_IN == 4096 and pr.POOLS == (2, 2, 2, 4)


def test_peaks_fall_back_without_the_measured_file(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench._peaks() == (6650.0, "fallback")
    assert bench._bf16_peak() == (1590.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text('{"hbm_gbs": 7000.0, "bf16_tflops": 1600.0}')
    assert bench._peaks() == (7000.0, "measured")
    assert bench._bf16_peak() == (1600.0, "measured")
