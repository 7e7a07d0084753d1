"""The mixed-precision scan pinned by two independent readings of the
reference: the oracle (C++, oracle/) and a literal NumPy restatement of
kernels.rs (tests/_scan_literal.py, no shared code). On seeded small curves
built to reach every branch of scan_tiles' f32 pre-ranking (exact near ties,
an unsafe merit, the sensitivity flag, the tile shape gate open and closed,
the invalid key nb + 1 + j, the f64 rescan) both give the same records,
scores, depths and flags bit for bit, and the GPU gives them too. A literal
reading of the evidence screen (tests/_screen_literal.py) picks the oracle's
screen maximum and pilot template.
"""
import math
from collections import Counter

import numpy as np
import pytest

import _scan_literal as L
import _screen_literal as S
import oracle
from fbls_b200 import synth


def _periodic_case():
    """A pattern repeating every 0.05 d folded at multiples of it: the
    histogram repeats, so boxes at phases a quarter cycle apart tie exactly
    (near-tie retries)."""
    t = synth.T0 + np.arange(2400) * (0.05 / 25)
    phase = (np.arange(2400) % 25)
    flux = np.where(phase < 3, -2e-3, 0.0) + np.where(phase == 12, 5e-4, 0.0)
    d = [0.004, 0.006, 0.010]
    st = oracle.family_state(t, flux, np.full(t.shape[0], 1e-3), d)
    return st, [0.2, 0.3, 0.15, 0.25], d, [1.0, 1.0, 1.0]


def _heavy_case():
    """Three observations carry almost all of the weight: a box holding them
    has c norm - hp^2 below 1e-3 c norm (unsafe merit, whole-tile rescan)."""
    rng = np.random.default_rng(7)
    t = synth.T0 + np.sort(rng.uniform(0.0, 3.0, 900))
    sigma = np.full(t.shape[0], 1e-3)
    heavy = [300, 301, 302]
    sigma[heavy] = 1e-7
    flux = rng.normal(0.0, 1e-3, t.shape[0])
    flux[heavy] = 0.0
    flux[290:320] -= 3e-3
    d = [0.02, 0.05]
    st = oracle.family_state(t, flux, sigma, d, correlated=False)
    return st, [0.7, 0.9, 1.1, 1.3], d, [1.0, 1.0]


def _twin_durations_case():
    """Two durations one part in 1e7 apart share every width: equal merits in
    one lane (the sensitivity flag)."""
    c = synth.small_curve(seed=9)
    d = [0.03, 0.03 * (1 + 1e-7), 0.08]
    st = oracle.family_state(c.time, c.flux, c.flux_err, d)
    return st, list(np.linspace(0.5, 2.5, 9)), d, [1.0, 1.0, 1.1]


def _noise_case(gate):
    c = synth.small_curve(seed=4, depth=0.0)
    d = [0.02, 0.05, 0.1]
    st = oracle.family_state(c.time, c.flux, c.flux_err, d)
    return st, list(np.linspace(0.45, 2.9, 7)), d, list(st.rho)


CASES = {
    "periodic": (_periodic_case, 0.6 * 7.1, 160),
    "heavy": (_heavy_case, 0.6 * 7.1, 150),
    "twins": (_twin_durations_case, 0.0, 200),
    "noise_gate_closed": (lambda: _noise_case(100.0), 100.0, 260),
    "noise_gate_open": (lambda: _noise_case(0.0), 0.0, 96),
}


def _run(name):
    make, gate, nb = CASES[name]
    st, periods, d, rho = make()
    lit = L.scan_bank_literal(st.time, st.v, st.w, st.baseline_norm, periods, nb, d, rho, gate=gate)
    orc = oracle.scan_bank(st, periods, nb, d, rho, shape_gate=gate, mode=0)
    return st, periods, d, rho, gate, nb, lit, orc


def test_literal_prefix_rows_equal_the_oracle():
    st, periods, d, rho = _twin_durations_case()
    for nb in (96, 300, 700):
        scale = nb / periods[3]
        cum, hi, lo = L.prefix_block(L.fold(st.time, st.v, st.w, scale, nb), nb)
        _, ocum, ocum32 = oracle.fold_prefix(st, scale, nb)
        assert np.array_equal(cum, ocum)
        assert np.array_equal(hi, ocum32[..., 0]) and np.array_equal(lo, ocum32[..., 1])


@pytest.mark.parametrize("name", sorted(CASES))
def test_literal_scan_equals_the_oracle(name):
    *_, lit, orc = _run(name)
    rec, score, depth, flags, _ = lit
    orec, oscore, odepth, oflags, _ = orc
    assert np.array_equal(rec, orec)
    assert np.array_equal(score, oscore)
    assert np.array_equal(depth, odepth)
    assert np.array_equal(flags, oflags)


def test_every_branch_is_exercised():
    total = Counter()
    for name in CASES:
        total.update(_run(name)[-2][-1])
    print("branch counts:", dict(total))
    for branch in ("retry_near_tie", "retry_unsafe", "retry_sensitive", "rescans", "gate_open", "gate_closed",
                   "invalid_key_lanes", "unsafe_lanes"):
        assert total[branch] > 0, branch


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_scan_equals_the_literal_restatement(gpu, name):
    from fbls_b200 import api
    st, periods, d, rho, gate, nb, lit, _ = _run(name)
    state = api.FamilyState(time=st.time, v=st.v, w=st.w, baseline_norm=st.baseline_norm, origin=st.origin,
                            residual_energy=st.residual_energy, durations=np.asarray(d), rho=np.asarray(rho))
    dev = gpu.upload(state)
    bank = api.Bank(durations=d, rho=rho, shape_gate=gate)
    rec, score, depth, flags, _ = gpu.scan_bank(dev, periods, bank, nb, precision_mode=0)
    dev.free()
    assert np.array_equal(rec, lit[0])
    assert np.array_equal(score, lit[1])
    assert np.array_equal(depth, lit[2])
    # The device's flag word adds bit 2 (this tile ran its f64 rescan), which
    # the library counts as tile_rescans; bits 0 and 1 are the reference's.
    assert np.array_equal(flags & 3, lit[3])


# -- the evidence screen ------------------------------------------------------

@pytest.mark.parametrize("period", [1.3, 0.9, 1.95, 2.6])
def test_literal_screen_picks_the_oracles_pilot(period):
    # The screen's maximum (the threshold test) and the pilot key (the
    # template the floors come from) of a literal reading of evidence.rs
    # against the oracle's compare_search diagnostics on the small curve.
    c, cfg = synth.small_curve(), synth.small_config()
    st = oracle.family_state(c.time, c.flux, c.flux_err, cfg.durations_days())
    maximum, key, s = S.pilot(st, period, cfg)
    _, diag = oracle.compare_search(st, period, cfg, diag=True)
    assert int(diag["nb"]) == s["nb"]
    assert maximum == diag["screen_max"]
    if maximum >= cfg.threshold * (1.0 - 1e-12):
        assert key == diag["pilot_key"]
