"""fbls_scan_bank_static: the scan pass for callers that cannot allocate
device memory (their GPU memory is owned by another allocator or a fixed
partition). It must give the same records, scores, depths and flags as the
allocating entry point fbls_scan_bank, on two calls in a row (the second call
reuses the static array the first one left behind), in both precision modes
and when the periods run in several batches with a shorter last one. This
file is collected last so that a run stopping at the first failure has run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

from fbls_b200 import _native as N
from fbls_b200 import api, synth


def _static_scan(state, periods, bank, nb, mode=0, outputs=None):
    lib = N.load()
    t, v, w = (np.ascontiguousarray(x, dtype=np.float64) for x in (state.time, state.v, state.w))
    p = np.ascontiguousarray(periods, dtype=np.float64)
    P = p.shape[0]
    rec, score, depth, flags = outputs if outputs is not None else (
        np.empty((P, 9)), np.empty(P), np.empty(P), np.empty(P, dtype=np.uint32))
    err = C.create_string_buffer(256)
    b, keep = bank._native()
    dp = lambda a: a.ctypes.data_as(N.c_double_p)
    rc = lib.fbls_scan_bank_static(0, dp(t), dp(v), dp(w), t.shape[0], state.baseline_norm, dp(p), P, C.byref(b), nb,
                                   mode, dp(rec), dp(score), dp(depth), flags.ctypes.data_as(N.c_uint32_p), err, 256)
    if rc:
        raise api.FblsError(rc, err.value.decode())
    return rec, score, depth, flags


def _workload(name):
    if name == "small":
        curve, cfg = synth.small_curve(), synth.small_config()
    else:
        curve, cfg = synth.single_sector(), synth.single_sector_config()
    state = api.prepared_family(curve.time, curve.flux, curve.flux_err, cfg)
    grid, bands = api.band_plan(state, cfg)
    return state, bands[-1], cfg


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("workload", ["small", "single_sector"])
def test_static_scan_matches_allocating_scan_twice(gpu, workload, mode):
    state, band, cfg = _workload(workload)
    dev = gpu.upload(state)
    bank = api.bank_for(band, cfg)
    for nb in (band["nb"] // 2, band["nb"]):
        want = gpu.scan_bank(dev, band["periods"], bank, nb, precision_mode=mode)
        for _ in range(2):
            got = _static_scan(state, band["periods"], bank, nb, mode)
            for g, w in zip(got, want[:4]):
                assert np.array_equal(g, w)
    dev.free()


@pytest.mark.gpu
def test_static_scan_with_a_short_last_batch(gpu):
    # single_sector's top band at its full nb does not fit the array in one
    # batch; dropping a few periods leaves a last batch shorter than the rest.
    state, band, cfg = _workload("single_sector")
    periods = band["periods"][:-7]
    dev = gpu.upload(state)
    bank = api.bank_for(band, cfg)
    want = gpu.scan_bank(dev, periods, bank, band["nb"])
    got = _static_scan(state, periods, bank, band["nb"])
    for g, w in zip(got, want[:4]):
        assert np.array_equal(g, w)
    dev.free()


@pytest.mark.gpu
def test_static_scan_rejects_inputs_beyond_its_array(gpu):
    state = api.prepared_family(*(lambda c: (c.time, c.flux, c.flux_err))(synth.small_curve()), synth.small_config())
    bank = api.Bank(durations=[0.05], rho=[1.0])
    with pytest.raises(api.FblsError, match="static scratch"):
        _static_scan(state, [1.0], bank, 2_000_000)


def test_static_scan_with_no_periods_leaves_the_outputs_alone():
    # P = 0 returns before any device work (no GPU needed).
    state, band, cfg = _workload("small")
    bank = api.bank_for(band, cfg)
    outs = (np.full((1, 9), 7.0), np.full(1, 7.0), np.full(1, 7.0), np.full(1, 7, dtype=np.uint32))
    _static_scan(state, np.empty(0), bank, band["nb"], outputs=outs)
    assert all((o == 7).all() for o in outs)


@pytest.mark.parametrize("bad", ["null_durations", "zero_duration", "nan_duration"])
def test_static_scan_rejects_bad_banks_before_touching_a_device(bad):
    # Argument checks come before cudaSetDevice, so they run without a GPU.
    state, band, cfg = _workload("small")
    if bad == "null_durations":
        bank = api.bank_for(band, cfg)
        b, keep = bank._native()
        b.durations = None
        lib = N.load()
        t = np.ascontiguousarray(state.time)
        p = np.ascontiguousarray(band["periods"][:4])
        out = np.empty((4, 9)), np.empty(4), np.empty(4), np.empty(4, dtype=np.uint32)
        err = C.create_string_buffer(256)
        dp = lambda a: a.ctypes.data_as(N.c_double_p)
        rc = lib.fbls_scan_bank_static(0, dp(t), dp(np.ascontiguousarray(state.v)), dp(np.ascontiguousarray(state.w)),
                                       t.shape[0], state.baseline_norm, dp(p), 4, C.byref(b), band["nb"], 0,
                                       dp(out[0]), dp(out[1]), dp(out[2]), out[3].ctypes.data_as(N.c_uint32_p),
                                       err, 256)
        assert rc == 1 and b"null argument" in err.value
        return
    d = 0.0 if bad == "zero_duration" else float("nan")
    bank = api.Bank(durations=[d, 0.1], rho=[1.0, 1.0])
    with pytest.raises(api.FblsError, match="positive and finite"):
        _static_scan(state, band["periods"][:4], bank, band["nb"])
