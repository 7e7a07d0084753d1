"""Parity of the CUDA scan path with the oracle, through the C ABI.

The fold adds each bin's observations in time order and the prefix sums use
the reference's association (kernels.rs:237-309) on both sides, and every
later operation rounds the same way (no fused multiply-adds), so the device
results must equal the oracle's bit for bit: phase, width, shape and
duration indices, a, norm, d, score and depth. This is stricter than the
path's 1e-6 tolerance on power, which is also asserted explicitly.
"""
import numpy as np
import pytest

import oracle
from fbls_b200 import api, synth

pytestmark = pytest.mark.gpu

RTOL = 1e-6


def _compare_records(g, o):
    grec, gscore, gdepth, gflags = g[:4]
    orec, oscore, odepth, oflags = o[:4]
    assert grec.shape == orec.shape
    finite = np.isfinite(oscore)
    rel = np.abs(gscore[finite] - oscore[finite]) / np.abs(oscore[finite])
    assert rel.max(initial=0.0) <= RTOL, rel.max()
    bad = np.nonzero(~(grec == orec).all(axis=1) | (gscore != oscore) | (gdepth != odepth))[0]
    assert bad.size == 0, (bad[:5], grec[bad[:2]], orec[bad[:2]], gscore[bad[:2]], oscore[bad[:2]])
    assert np.array_equal(gflags & 3, oflags & 3)
    return 0


@pytest.fixture(scope="module")
def small():
    c = synth.small_curve()
    cfg = synth.small_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    ost = oracle.family_state(c.time, c.flux, c.flux_err, cfg.durations_days())
    return c, cfg, st, ost


@pytest.mark.parametrize("mode", [0, 1])
def test_scan_bank_parity_small(gpu, small, mode):
    c, cfg, st, ost = small
    dev = gpu.upload(st)
    grid, bands = api.band_plan(st, cfg)
    for band in bands:
        bank = api.bank_for(band, cfg)
        for nb in (band["nb"] // 2, band["nb"], band["nb"] + 37):
            g = gpu.scan_bank(dev, band["periods"], bank, nb, precision_mode=mode)
            o = oracle.scan_bank(ost, band["periods"], nb, band["durations"], band["rho"], ingress=cfg.ingress_fractions,
                                 layers=cfg.shape_layers, shape_gate=bank.shape_gate, mode=mode)
            _compare_records(g, o)
            stats = g[4]
            assert stats["templates_scanned"] == len(band["periods"]) * len(band["durations"]) * 3 * nb
            assert stats["exact_tile_retries"] == 0  # the reference's flag word never keeps the retry bit


def test_signal_search_parity_small(gpu, small):
    c, cfg, st, ost = small
    rows, glen, stats = gpu.signal_search(st, cfg)
    orows, ogrid, ostats = oracle.signal_search(ost, cfg)
    assert glen == len(ogrid)
    assert np.array_equal(rows, orows)
    for s, o in zip(stats, ostats):
        for key in ("periods", "prescan_survivors", "phase_bins", "templates_scanned"):
            assert s[key] == o[key], key


def test_global_fold_path(gpu, small):
    """Phase grids whose histograms exceed shared memory fold in global memory."""
    c, cfg, st, ost = small
    dev = gpu.upload(st)
    periods = np.array([1.3, 2.1, 2.7])
    d = np.array(sorted(cfg.durations_days()))
    bank = api.Bank(durations=d, rho=st.rho[np.argsort(st.durations, kind="stable")])
    nb = 12000
    g = gpu.scan_bank(dev, periods, bank, nb)
    o = oracle.scan_bank(ost, periods, nb, d, bank.rho)
    _compare_records(g, o)


def test_budget_error_keeps_reference_message(gpu, small):
    c, cfg, st, ost = small
    dev = gpu.upload(st)
    bank = api.Bank(durations=[0.05], rho=[1.0], max_fold_mib=1e-6)
    with pytest.raises(api.FblsError, match="one folded period exceeds max_fold_mib"):
        gpu.scan_bank(dev, [1.0], bank, 64)


def test_launches_of_several_batches_keep_results_and_batch_count(gpu, small):
    """A launch may cover several of the reference's batches; the records do
    not depend on the batch size and ScanStats counts the reference's batches
    (ceil(P / period_batch), scan.rs:190-199)."""
    c, cfg, st, ost = small
    dev = gpu.upload(st)
    grid, bands = api.band_plan(st, cfg)
    band = bands[-1]
    periods = band["periods"]
    whole = gpu.scan_bank(dev, periods, api.bank_for(band, cfg), band["nb"])
    for batch in (7, 64, len(periods)):
        bank = api.bank_for(band, cfg)
        bank.period_batch = batch
        got = gpu.scan_bank(dev, periods, bank, band["nb"])
        for x, y in zip(got[:4], whole[:4]):
            assert np.array_equal(x, y)
        assert got[4]["batches"] == -(-len(periods) // batch)


def test_fold_is_deterministic(gpu, small):
    c, cfg, st, ost = small
    dev = gpu.upload(st)
    grid, bands = api.band_plan(st, cfg)
    band = bands[-1]
    bank = api.bank_for(band, cfg)
    first = gpu.scan_bank(dev, band["periods"], bank, band["nb"])
    for _ in range(3):
        again = gpu.scan_bank(dev, band["periods"], bank, band["nb"])
        for x, y in zip(first[:4], again[:4]):
            assert np.array_equal(x, y)


def _subsample_parity(gpu, curve, cfg, every):
    st = api.prepared_family(curve.time, curve.flux, curve.flux_err, cfg)
    ost = oracle.family_state(curve.time, curve.flux, curve.flux_err, cfg.durations_days())
    assert np.array_equal(st.v, ost.v)
    dev = gpu.upload(st)
    grid, bands = api.band_plan(st, cfg)
    for band in bands:
        sel = band["periods"][::every]
        bank = api.bank_for(band, cfg)
        for nb in (band["nb"] // 2, band["nb"]):
            for mode in (0, 1):
                g = gpu.scan_bank(dev, sel, bank, nb, precision_mode=mode)
                o = oracle.scan_bank(ost, sel, nb, band["durations"], band["rho"], ingress=cfg.ingress_fractions,
                                     layers=cfg.shape_layers, shape_gate=bank.shape_gate, mode=mode)
                _compare_records(g, o)


def test_single_sector_full_size_parity(gpu):
    """~19k points, 12 durations, every 13th period of each band at coarse and full nb."""
    _subsample_parity(gpu, synth.single_sector(), synth.single_sector_config(), every=13)


def test_multi_sector_full_size_parity(gpu):
    """~250k points, 20 durations, nb up to 3840: every 1500th period of each band."""
    _subsample_parity(gpu, synth.multi_sector(), synth.multi_sector_config(), every=1500)


def test_single_sector_recovers_injected_signal(gpu):
    c = synth.single_sector()
    cfg = synth.single_sector_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    rows, glen, stats = gpu.signal_search(st, cfg)
    assert glen == 13065
    best = rows[np.argmax(rows[:, 3])]
    assert abs(best[0] / c.period - 1.0) < 2e-3
    phase = ((best[1] - c.epoch) / c.period + 0.5) % 1.0 - 0.5
    assert abs(phase * c.period) < c.duration / 2
    assert abs(best[2] / c.duration - 1.0) < 0.35
