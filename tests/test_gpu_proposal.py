"""Proposal path: the coarse periodogram (fbls_coarse_map) is, per period and
duration, the score of the best box template over all phases, the same value
the f64 scan reports for a one-duration box-only bank at the same nb."""
import math

import numpy as np
import pytest

from fbls_b200 import api, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("workload", ["small", "single_sector"])
def test_coarse_map_matches_the_f64_box_scan(gpu, workload):
    if workload == "small":
        c, cfg = synth.small_curve(), synth.small_config()
        periods = np.geomspace(0.6, 1.15, 257)
    else:
        c, cfg = synth.single_sector(), synth.single_sector_config()
        periods = np.geomspace(2.0, 3.9, 1000)
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    dev = gpu.upload(st)
    pick = [0, len(st.durations) // 3, len(st.durations) - 1]
    durations, rho = st.durations[pick], st.rho[pick]
    oversample = 2.0
    got = gpu.coarse_map(dev, periods, durations, rho, oversample)
    nb = max(8, math.ceil(oversample * periods[-1] / durations.min()))
    for d in range(len(pick)):
        bank = api.Bank(durations=[durations[d]], rho=[rho[d]], ingress=(0.0,), layers=1, shape_gate=0.0)
        rec, score, depth, flags, stats = gpu.scan_bank(dev, periods, bank, nb, precision_mode=1)
        want = np.where(np.isfinite(score) & (score > 0), score, 0.0).astype(np.float32)
        assert np.array_equal(got[:, d], want), (d, np.nonzero(got[:, d] != want)[0][:5])
    assert (got > 0).any()
    dev.free()
