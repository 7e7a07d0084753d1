"""The precision forms on the GPU against the FP64 arithmetic.

precision_mode 2 (the f32 form: f32 ranking from the compensated (hi, lo) f32
prefix pairs, the winner's values in f32, no f64 prefix rows) against
precision_mode 1 (f64 ranking, bit-identical to the FP64 oracle): the same
winning template (bin, width, shape, duration) on every period whose score
clears the threshold, and the winner's SNR within 1e-5 and depth within 1e-4
relative of the FP64 values (the f32 form's own tolerance; the run-to-run
report in `bench.py --precision-report` gives the measured errors).

The bin forms: every observation at a sample of periods, the f64 bin of the
fold against the double-single product with its exact fallback (no
mismatch allowed) and against a plain f32 product (which does mismatch).
"""
import numpy as np
import pytest

import oracle
from fbls_b200 import api, synth

pytestmark = pytest.mark.gpu

SNR_RTOL = 1e-5
DEPTH_RTOL = 1e-4


@pytest.fixture(scope="module")
def single(gpu):
    c, cfg = synth.single_sector(), synth.single_sector_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    dev = gpu.upload(st)
    yield c, cfg, st, dev
    dev.free()


def test_f64_ranking_equals_the_oracle(gpu, single):
    c, cfg, st, dev = single
    grid, bands = api.band_plan(st, cfg)
    band = bands[1]
    bank = api.bank_for(band, cfg)
    ost = oracle.family_state(c.time, c.flux, c.flux_err, cfg.durations_days())
    periods = band["periods"][::50]
    got = gpu.scan_bank(dev, periods, bank, band["nb"], precision_mode=1)
    want = oracle.scan_bank(ost, periods, band["nb"], band["durations"], band["rho"], shape_gate=bank.shape_gate, mode=1)
    for g, w in zip(got[:4], want[:4]):
        assert np.array_equal(g, w)


@pytest.mark.parametrize("band_index", [0, 2, 4])
def test_f32_form_against_f64(gpu, single, band_index):
    c, cfg, st, dev = single
    grid, bands = api.band_plan(st, cfg)
    band = bands[band_index]
    bank = api.bank_for(band, cfg)
    for nb in (band["nb"] // 2, band["nb"]):
        ref = gpu.scan_bank(dev, band["periods"], bank, nb, precision_mode=1)
        f32 = gpu.scan_bank(dev, band["periods"], bank, nb, precision_mode=2)
        key = [2, 3, 7, 8]
        top = np.isfinite(ref[1]) & (ref[1] >= bank.threshold)
        same = (f32[0][:, key] == ref[0][:, key]).all(axis=1)
        assert same[top].all()
        ok = np.isfinite(ref[1]) & (ref[1] > 0) & same
        assert (np.abs(f32[1][ok] - ref[1][ok]) / ref[1][ok]).max(initial=0.0) <= SNR_RTOL
        assert (np.abs(f32[2][ok] - ref[2][ok]) / np.abs(ref[2][ok])).max(initial=0.0) <= DEPTH_RTOL
        assert same[np.isfinite(ref[1])].mean() > 0.99


def test_f32_form_signal_search_finds_the_injected_box(gpu, single):
    c, cfg, st, dev = single
    cfg2 = synth.single_sector_config()
    cfg2.precision_mode = 2
    rows, _, _ = gpu.signal_search(st, cfg2, dev=dev)
    ref, _, _ = gpu.signal_search(st, cfg, dev=dev)
    best = rows[int(np.argmax(rows[:, 3]))]
    rbest = ref[int(np.argmax(ref[:, 3]))]
    assert best[0] == rbest[0] and best[1] == rbest[1] and best[2] == rbest[2]
    assert abs(best[3] - rbest[3]) <= SNR_RTOL * rbest[3]


def test_bin_forms(gpu, single):
    c, cfg, st, dev = single
    grid, bands = api.band_plan(st, cfg)
    band = bands[-1]
    scales = band["nb"] / np.asarray(band["periods"][::20])
    counts = gpu.precision_bins(dev, scales, band["nb"])
    assert counts["pairs"] == st.n * scales.shape[0]
    assert counts["fallback_mismatches"] == 0
    assert counts["f32_mismatches"] > 0
    assert counts["fallbacks"] < 1e-4 * counts["pairs"]


def test_precision_mode_out_of_range_is_an_argument_error(gpu, single):
    c, cfg, st, dev = single
    grid, bands = api.band_plan(st, cfg)
    band = bands[0]
    with pytest.raises(api.FblsError, match="precision_mode"):
        gpu.scan_bank(dev, band["periods"][:4], api.bank_for(band, cfg), band["nb"], precision_mode=3)
