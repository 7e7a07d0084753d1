"""The C-ABI library on CPU: it loads, exports every entry point the header
declares, and its host-side code (period grid, prepared-mode family state,
configuration) matches the oracle exactly. No GPU calls."""
import ctypes
import math
import re
from pathlib import Path

import numpy as np
import pytest

import oracle
from fbls_b200 import _native, api, synth
from fbls_b200.config import SearchConfig

HEADER = Path(__file__).resolve().parent.parent / "include" / "fbls_b200.h"


def _declared():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fbls_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    names = _declared()
    assert len(names) >= 12
    for name in names:
        assert hasattr(lib, name), name
        assert name in _native.SIGNATURES, name
    assert lib.fbls_version().decode().startswith("fbls_b200")


def test_period_grid_matches_oracle():
    for args in [(0.5, 20.0, 50.0, 0.02, 3.0), (0.5, 13.7, 26.4, 0.5 / 24, 3.0), (0.3, 10.0, 356.2, 0.5 / 24, 3.0)]:
        assert np.array_equal(api.period_grid(*args), oracle.period_grid(*args))


@pytest.mark.parametrize("maker", [synth.small_curve, synth.single_sector])
def test_family_state_matches_oracle_bit_exactly(maker):
    c = maker()
    cfg = synth.small_config() if maker is synth.small_curve else synth.single_sector_config()
    d = cfg.durations_days()
    a = api.family_state(c.time, c.flux, c.flux_err, d)
    o = oracle.family_state(c.time, c.flux, c.flux_err, d)
    assert a.n == o.n
    for name in ("time", "v", "w", "rho"):
        assert np.array_equal(getattr(a, name), getattr(o, name)), name
    assert a.baseline_norm == o.baseline_norm
    assert a.origin == o.origin
    assert a.residual_energy == o.residual_energy
    assert a.inflation == o.inflation


def test_family_state_errors_keep_the_reference_messages():
    t = np.arange(5.0)
    with pytest.raises(api.FblsError, match="insufficient usable observations"):
        api.family_state(t, np.zeros(5), np.ones(5), [0.1])
    t = np.arange(20.0)
    f = np.full(20, -2.0)  # 1 + flux has a negative median
    with pytest.raises(api.FblsError, match="positive median"):
        api.family_state(t, f, np.ones(20), [0.1])


def test_family_state_drops_nonfinite_and_sorts():
    c = synth.small_curve()
    t = c.time.copy()
    f = c.flux.copy()
    e = c.flux_err.copy()
    f[5] = np.nan
    e[7] = 0.0
    perm = np.random.default_rng(1).permutation(t.shape[0])
    d = synth.small_config().durations_days()
    a = api.family_state(t[perm], f[perm], e[perm], d)
    o = oracle.family_state(t, f, e, d)
    assert a.n == c.time.shape[0] - 2
    assert np.array_equal(a.v, o.v)


def test_config_defaults_and_validation():
    cfg = SearchConfig()
    cfg.validate()
    assert cfg.durations_hours[:3] == [0.5, 0.625, 0.78125]
    assert len(cfg.durations_days()) == 13
    with pytest.raises(ValueError, match="quarter of period_min"):
        SearchConfig(period_min=0.05).validate()
    with pytest.raises(ValueError, match="ingress"):
        SearchConfig(ingress_fractions=[0.5]).validate()


def test_band_plan_matches_oracle():
    c = synth.single_sector()
    cfg = synth.single_sector_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    grid, bands = api.band_plan(st, cfg)
    ost = oracle.family_state(c.time, c.flux, c.flux_err, cfg.durations_days())
    ogrid, obands = oracle.band_plan(ost, cfg)
    assert np.array_equal(grid, ogrid)
    assert len(bands) == len(obands) == 5
    for b, (sel, d, r) in zip(bands, obands):
        assert np.array_equal(b["periods"], sel)
        assert np.array_equal(b["durations"], d)
    # The reference's rule at this configuration: 13,065 periods, nb 192 ... 2631.
    assert grid.shape[0] == 13065
    assert [b["nb"] for b in bands] == [192, 384, 768, 1536, 2631]


def test_period_grid_refuses_infinite_grids_and_keeps_the_reference_edge_cases():
    lib = _native.load()
    # infinite counts: a zero minimum period, a zero minimum duration (zero step), an infinite maximum
    for args in [(0.0, 20.0, 50.0, 0.02, 3.0), (0.5, 20.0, 50.0, 0.0, 3.0), (0.5, math.inf, 50.0, 0.02, 3.0),
                 (1e-9, 1e9, 1e9, 1e-12, 1e6)]:
        assert lib.fbls_period_grid(*args, None, 0) == -1, args
        with pytest.raises(api.FblsError, match="infinite or too large"):
            api.period_grid(*args)
    # a reversed range or a NaN bound gives one period (the reference's saturating count), the maximum
    for args in [(20.0, 0.5, 50.0, 0.02, 3.0), (math.nan, 20.0, 50.0, 0.02, 3.0)]:
        g = api.period_grid(*args)
        assert g.shape == (1,) and g[0] == args[1]


def test_family_state_rejects_null_arrays():
    lib = _native.load()
    err = ctypes.create_string_buffer(64)
    rc = lib.fbls_family_state(None, None, None, 10, None, 0, 1, None, None, None, None, None, None, err, 64)
    assert rc == 1 and err.value == b"null argument"


def test_multi_sector_workload_sizes():
    """The 13-sector benchmark workload under the reference's rules: 247,104
    points, 189,216 periods in 6 octave bands of 11, 14, 18, 20, 20, 20
    durations at nb 192 ... 3840; the dense-grid variants' counts."""
    c, cfg = synth.multi_sector(), synth.multi_sector_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    grid, bands = api.band_plan(st, cfg)
    assert st.n == 247104 and grid.shape[0] == 189216
    assert [len(b["durations"]) for b in bands] == [11, 14, 18, 20, 20, 20]
    assert [b["nb"] for b in bands] == [192, 384, 768, 1536, 3072, 3840]
    assert sum(len(b["periods"]) for b in bands) == grid.shape[0]
    dense = SearchConfig(**{**cfg.__dict__, "period_oversample": 19.0})
    assert api.band_plan(st, dense)[0].shape[0] == 1198347
    s1, c1 = synth.single_sector(), synth.single_sector_config()
    st1 = api.prepared_family(s1.time, s1.flux, s1.flux_err, c1)
    assert st1.n == 19008
    assert api.band_plan(st1, SearchConfig(**{**c1.__dict__, "period_oversample": 6.9}))[0].shape[0] == 30044


def test_host_entry_points_are_safe_to_call_from_many_threads():
    """ctypes releases the GIL, so these calls overlap in the library: family
    state, period grids and noise fits from 8 threads equal the sequential
    results (the host code keeps no shared state)."""
    from concurrent.futures import ThreadPoolExecutor
    curves = [synth.small_curve(seed=s) for s in range(8)]
    cfg = synth.small_config()

    def work(c):
        st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
        g = api.period_grid(0.3, 9.0, float(st.time[-1]), 0.02, 3.0)
        m = api.fit_segment_noise(c.time, 1e4 * (1.0 + c.flux), None, None, 10.0, 0.75)
        return st.v, g, m.deficit

    want = [work(c) for c in curves]
    with ThreadPoolExecutor(8) as pool:
        for _ in range(3):
            got = list(pool.map(work, curves))
            for (v, g, d), (wv, wg, wd) in zip(got, want):
                assert np.array_equal(v, wv) and np.array_equal(g, wg) and np.array_equal(d, wd)


def test_oracle_search_does_not_depend_on_its_thread_count():
    c, cfg = synth.small_curve(), synth.small_config()
    st = oracle.family_state(c.time, c.flux, c.flux_err, cfg.durations_days())
    one = oracle.signal_search(st, cfg, threads=1)
    many = oracle.signal_search(st, cfg, threads=8)
    assert np.array_equal(one[0], many[0]) and np.array_equal(one[1], many[1])


def test_tuning_table_round_trip_and_limits():
    from fbls_b200 import autotune
    try:
        table = {"fold_group_max": {"10": 4, "11": 2}, "fold_threads": {"10": 512, "11": 256},
                 "lockstep_min": {"10": 7}, "fold_pair": {"9": 1}, "launch_periods": 8192, "fold_steal": 1,
                 "fused_scan": 1,
                 "map_lockstep_min": 3, "map_threads": 512, "map_group_max": 64, "batch_no_fill": 1}
        autotune.apply(table)
        assert autotune.current() == table
        with pytest.raises(ValueError):
            autotune.apply({"fold_group_max": {"10": 3}})  # not a power of two
        with pytest.raises(ValueError):
            autotune.apply({"fold_group_max": {"10": 256}})  # above the largest group
        with pytest.raises(ValueError):
            autotune.apply({"map_group_max": 256})
        with pytest.raises(ValueError):
            autotune.apply({"map_threads": 640})
        with pytest.raises(ValueError):
            autotune.apply({"batch_no_fill": 2})
        with pytest.raises(ValueError):
            autotune.apply({"fold_threads": {"10": 384}})  # not a walking-fold CTA size
        with pytest.raises(ValueError):
            autotune.apply({"lockstep_min": {"10": 5000}})
    finally:
        autotune.reset()
    assert autotune.current() == {"fold_group_max": {}, "fold_threads": {}, "lockstep_min": {}, "fold_pair": {},
                                  "launch_periods": 16384,
                                  "fold_steal": 0, "fused_scan": 0, "map_lockstep_min": 0, "map_threads": 0,
                                  "map_group_max": 0, "batch_no_fill": 0}
