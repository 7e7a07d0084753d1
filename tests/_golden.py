"""The committed golden fixtures (tests/golden/) and the checks that hold a
search path to them. A check takes `gpu`, an object with the library
context's methods (fbls_b200.api.Gpu on a GPU; OracleGpu, the oracle behind
the same methods, on the CPU), so that the GPU tests and the oracle's CPU
pin run the same comparisons on the same files.

Bars: bit for bit for the scan records, scores, depths, tile flags, search
rows, rescoring sums and counts, single events and detrended series; the
model-comparison rows keep indices and flags exact and take `rtol` (with an
`atol` floor) on SNR and depth and `log_atol` (scaled by max(1, |x|)) on
log-evidences, whose exp / log terms differ by ulps between the device and
the host library (all 0 for the oracle itself)."""
from __future__ import annotations

import dataclasses
import json
import math
from pathlib import Path

import numpy as np

import oracle
from fbls_b200 import api
from fbls_b200.config import SearchConfig

GOLDEN = Path(__file__).resolve().parent / "golden"


def load():
    """(arrays, meta, config) of oracle_small.{npz,json}."""
    with np.load(GOLDEN / "oracle_small.npz") as z:
        arrays = {k: z[k] for k in z.files}
    meta = json.loads((GOLDEN / "oracle_small.json").read_text())
    return arrays, meta, SearchConfig(**meta["config"])


def reference_kats() -> dict:
    return json.loads((GOLDEN / "reference_kats.json").read_text())


class OracleGpu:
    """The oracle behind the library context's methods (test infrastructure).
    States are oracle.State objects; `upload` wraps one."""

    class _Dev:
        def __init__(self, state):
            self.state = state
            self.n = state.n

        def free(self):
            pass

    def upload(self, state):
        return self._Dev(state)

    def scan_bank(self, dev, periods, bank, nb, precision_mode=0):
        return oracle.scan_bank(dev.state, periods, nb, bank.durations, bank.rho, ingress=bank.ingress,
                                layers=bank.layers, shape_gate=bank.shape_gate, mode=precision_mode)

    def signal_search(self, state, cfg):
        rows, grid, stats = oracle.signal_search(state, cfg)
        return rows, len(grid), stats

    def compare_search(self, state, period, cfg):
        return oracle.compare_search(state, period, cfg)

    def compare_batch(self, candidates, cfg, devs=None):
        return [oracle.compare_search(state, period, cfg) for state, period in candidates]

    def rescore_rows(self, dev, excluded, rows):
        s = dev.state
        return oracle.rescore_rows(s.time, s.v, s.w, excluded, rows, s.origin)

    def count_rows(self, time, excluded, rows):
        return oracle.count_rows(time, excluded, rows)

    def single_event_search(self, state, cfg):
        return oracle.single_event_search(state, cfg)

    def biweight_flatten(self, time, flux, window, gap=0.5, iterations=10):
        return oracle.biweight_flatten(time, flux, window, gap=gap, iterations=iterations)


def _bank(arrays, meta, cfg, b):
    return api.bank_for({"durations": arrays[f"b{b}_durations"], "rho": arrays[f"b{b}_rho"]}, cfg)


def check_scan_bands(gpu, state, arrays, meta, cfg):
    """Every band at its coarse and full phase-bin count, both precision
    modes: records, score, depth and the tile flags' low bits."""
    dev = gpu.upload(state)
    try:
        for b, band in enumerate(meta["bands"]):
            bank = _bank(arrays, meta, cfg, b)
            assert bank.shape_gate == band["shape_gate"]
            for nb in band["nbs"]:
                for mode in (0, 1):
                    key = f"b{b}_nb{nb}_m{mode}"
                    got = gpu.scan_bank(dev, arrays[f"b{b}_periods"], bank, nb, precision_mode=mode)
                    rec, score, depth, flags = got[:4]
                    assert np.array_equal(rec, arrays[key + "_rec"]), key
                    assert np.array_equal(score, arrays[key + "_score"], equal_nan=True), key
                    assert np.array_equal(depth, arrays[key + "_depth"], equal_nan=True), key
                    assert np.array_equal(np.asarray(flags).astype(np.uint32) & 3, arrays[key + "_flags"]), key
    finally:
        dev.free()


def check_signal_search(gpu, state, arrays, meta, cfg):
    rows, glen, stats = gpu.signal_search(state, cfg)
    assert glen == meta["grid_len"]
    assert np.array_equal(rows, arrays["signal_rows"])
    assert len(stats) == len(meta["signal_stats"])
    for s, want in zip(stats, meta["signal_stats"]):
        for k, v in want.items():
            assert int(s[k]) == v, k


def _close(got, want, tol, scale_floor, floor=0.0):
    return abs(got - want) <= max(tol * max(scale_floor, abs(want)), floor)


def check_evidence(gpu, state, meta, cfg, rtol=0.0, log_atol=0.0, atol=0.0):
    for case in meta["evidence"]:
        got = gpu.compare_search(state, case["period"], cfg)
        want = case["rows"]
        assert len(got) == len(want), case["period"]
        for g, w in zip(got, want):
            assert int(g["selection_flags"]) == w["selection_flags"]
            for k in ("period", "epoch", "duration", "ingress_fraction"):
                assert float(g[k]) == w[k], k
            for k in ("snr", "depth"):
                assert _close(float(g[k]), w[k], rtol, 0.0, atol), (k, g[k], w[k])
            for k in ("planet_log_odds", "log_bf_planet_noise", "log_bf_binary_noise"):
                assert _close(float(g[k]), w[k], log_atol, 1.0), (k, g[k], w[k])
            for k in ("binary_secondary_ratio", "binary_secondary_phase", "binary_odd_even_ratio",
                      "binary_period_days"):
                if math.isnan(w[k]):
                    assert math.isnan(float(g[k])), k
                else:
                    assert float(g[k]) == w[k], k


def check_rescore(gpu, state, arrays):
    dev = gpu.upload(state)
    try:
        rows = arrays["rescore_rows"]
        ta = state.time + state.origin
        for tag, ex in (("none", np.zeros(state.n, np.uint8)), ("excluded", arrays["rescore_excluded"])):
            got = gpu.rescore_rows(dev, ex, rows)
            assert np.array_equal(got, arrays["rescore_sums_" + tag], equal_nan=True), tag
            assert np.array_equal(gpu.count_rows(ta, ex, rows), arrays["count_" + tag]), tag
    finally:
        dev.free()


def check_single_events(gpu, state, arrays, meta, cfg):
    rows, stats = gpu.single_event_search(state, cfg)
    assert json.loads(json.dumps(stats)) == meta["event_stats"]
    assert np.array_equal(rows, arrays["event_rows"])


def check_detrend(gpu, arrays, meta):
    d = meta["detrend"]
    got = gpu.biweight_flatten(arrays["detrend_time"], arrays["detrend_flux"], d["window"], gap=d["gap"],
                               iterations=d["iterations"])
    assert np.array_equal(got, arrays["detrend_out"])


def config_is_the_small_workload(meta) -> bool:
    from fbls_b200 import synth
    return meta["config"] == json.loads(json.dumps(dataclasses.asdict(synth.small_config())))
