"""fbls_scan_bank_static: the scan pass for callers that cannot allocate
device memory (their GPU memory is owned by another allocator or a fixed
partition). It must give the same records, scores, depths and flags as the
allocating entry point fbls_scan_bank, on two calls in a row (the second call
reuses the static array the first one left behind). This file is collected
last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from fbls_b200 import _native as N
from fbls_b200 import api, synth

pytestmark = pytest.mark.gpu


def _static_scan(state, periods, bank, nb, mode=0):
    lib = N.load()
    t, v, w = (np.ascontiguousarray(x, dtype=np.float64) for x in (state.time, state.v, state.w))
    p = np.ascontiguousarray(periods, dtype=np.float64)
    P = p.shape[0]
    rec = np.empty((P, 9))
    score = np.empty(P)
    depth = np.empty(P)
    flags = np.empty(P, dtype=np.uint32)
    err = C.create_string_buffer(256)
    b, keep = bank._native()
    dp = lambda a: a.ctypes.data_as(N.c_double_p)
    rc = lib.fbls_scan_bank_static(0, dp(t), dp(v), dp(w), t.shape[0], state.baseline_norm, dp(p), P, C.byref(b), nb,
                                   mode, dp(rec), dp(score), dp(depth), flags.ctypes.data_as(N.c_uint32_p), err, 256)
    if rc:
        raise api.FblsError(rc, err.value.decode())
    return rec, score, depth, flags


@pytest.mark.parametrize("workload", ["small", "single_sector"])
def test_static_scan_matches_allocating_scan_twice(gpu, workload):
    if workload == "small":
        curve, cfg = synth.small_curve(), synth.small_config()
    else:
        curve, cfg = synth.single_sector(), synth.single_sector_config()
    state = api.prepared_family(curve.time, curve.flux, curve.flux_err, cfg)
    dev = gpu.upload(state)
    grid, bands = api.band_plan(state, cfg)
    band = bands[-1]
    bank = api.bank_for(band, cfg)
    for nb in (band["nb"] // 2, band["nb"]):
        want = gpu.scan_bank(dev, band["periods"], bank, nb)
        for _ in range(2):
            got = _static_scan(state, band["periods"], bank, nb)
            for g, w in zip(got, want[:4]):
                assert np.array_equal(g, w)
    dev.free()


def test_static_scan_rejects_inputs_beyond_its_array(gpu):
    state = api.prepared_family(*(lambda c: (c.time, c.flux, c.flux_err))(synth.small_curve()), synth.small_config())
    bank = api.Bank(durations=[0.05], rho=[1.0])
    with pytest.raises(api.FblsError, match="static scratch"):
        _static_scan(state, [1.0], bank, 2_000_000)
