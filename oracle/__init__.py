"""CPU oracle of the FBLS search path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
import this package, and only to check or time against it. The product
(fbls_b200) never calls it.

The arithmetic lives in fbls_oracle.cpp (a C++ restatement of the
reference's src/search/{grid,scan,kernels,evidence,math}.rs, the
prepared-mode preparation in src/prep/{curve,stats}.rs, the rescoring and
single-event kernels and both forms of the biweight detrend); this module
binds it with ctypes and restates in Python the host orchestration of
scan_periods (src/search/scan.rs:363-408), signal_search
(src/search/scan.rs:413-473), single_event_search (src/search/events.rs) and
the raw-mode preparation (src/prep/curve.rs:89-198, :332-425).

Parity status: pinned by the reference's erfc table (math.rs:183-210), grid
property (grid.rs:34-42), noise-model / transit-mask tests
(curve.rs:636-673) and biweight trend test (curve.rs:624-634). The reference
has no golden vectors for the fold, prefix, tile-scan, evidence, rescoring,
single-event or detrend outputs; those are checked here by brute-force
identities and literal loop restatements only (parity unpinned against
reference output). The oracle's own outputs on seeded small inputs are frozen
in tests/golden/ (tests/golden/make_golden.py), where the CPU tests pin the
oracle and the GPU tests hold the CUDA path to the same files.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from pathlib import Path
from typing import List, Optional, Sequence

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

_dp = C.POINTER(C.c_double)
_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def _load():
    global _lib
    if _lib is not None:
        return _lib
    src = HERE / "fbls_oracle.cpp"
    if not LIB.exists() or (src.exists() and src.stat().st_mtime > LIB.stat().st_mtime):
        build()
    lib = C.CDLL(str(LIB))
    sig = {
        "orc_erfc": (C.c_double, [C.c_double]),
        "orc_log_add": (C.c_double, [C.c_double, C.c_double]),
        "orc_positive_amplitude_evidence": (C.c_double, [C.c_double, C.c_double, C.c_double]),
        "orc_subspace_upper": (C.c_double, [C.c_double] * 6),
        "orc_period_grid": (C.c_int64, [C.c_double] * 5 + [_dp, C.c_int64]),
        "orc_median_lower": (C.c_double, [_dp, C.c_int64]),
        "orc_family_state": (C.c_int, [_dp, _dp, _dp, C.c_int64, _dp, C.c_int, C.c_int, C.POINTER(C.c_int64),
                                       _dp, _dp, _dp, _dp, _dp, _dp]),
        "orc_fit_segment_noise": (C.c_int, [_dp, _dp, _dp, C.c_int64, C.c_double, C.POINTER(C.c_int64), _dp, _dp,
                                            _dp, _dp]),
        "orc_transit_mask": (C.c_int64, [_dp, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double,
                                         C.POINTER(C.c_uint8)]),
        "orc_rescore_rows": (None, [_dp, _dp, _dp, C.POINTER(C.c_uint8), C.c_int64, _dp, C.c_int64, C.c_double,
                                    _dp]),
        "orc_count_rows": (None, [_dp, C.POINTER(C.c_uint8), C.c_int64, _dp, C.c_int64, C.POINTER(C.c_uint32)]),
        "orc_biweight_flatten": (None, [_dp, _dp, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                        _dp]),
        "orc_single_event_scan": (C.c_int64, [_dp, _dp, _dp, C.c_int64, C.c_double, C.c_double, C.c_int, _dp, _dp,
                                              C.c_int, _dp, C.c_int, C.c_int, C.c_double, C.c_int64, _dp]),
        "orc_scan_bank": (C.c_int64, [_dp, _dp, _dp, C.c_int64, C.c_double, _dp, C.c_int64, C.c_int, _dp, _dp,
                                      C.c_int, _dp, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, _dp, _dp, _dp,
                                      C.POINTER(C.c_uint32)]),
        "orc_fold_prefix": (None, [_dp, _dp, _dp, C.c_int64, C.c_double, C.c_int, _dp, _dp, C.POINTER(C.c_float)]),
        "orc_box_direct": (None, [_dp, _dp, _dp, C.c_int64, C.c_double, C.c_int, C.c_int64, C.c_int64, _dp]),
        "orc_evidence_parameters": (None, [_dp, _dp]),
        "orc_compare_search": (C.c_int, [_dp, _dp, _dp, C.c_int64, C.c_double, C.c_double, C.c_double, _dp, _dp,
                                         C.c_int, _dp, C.c_int, C.c_double, _dp, _dp, _dp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _f(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


# -- scalar math (math.rs) ----------------------------------------------------

def erfc(x: float) -> float:
    return _load().orc_erfc(x)


def log_add(x: float, y: float) -> float:
    return _load().orc_log_add(x, y)


def positive_amplitude_evidence(a: float, q: float, tau: float) -> float:
    return _load().orc_positive_amplitude_evidence(a, q, tau)


def subspace_upper(a, b, q, r, cross, rho2) -> float:
    return _load().orc_subspace_upper(a, b, q, r, cross, rho2)


# -- grid and preparation -----------------------------------------------------

def period_grid(minimum, maximum, baseline, minimum_duration, oversample) -> np.ndarray:
    lib = _load()
    n = lib.orc_period_grid(minimum, maximum, baseline, minimum_duration, oversample, None, 0)
    out = np.empty(n)
    lib.orc_period_grid(minimum, maximum, baseline, minimum_duration, oversample, _p(out), n)
    return out


def median_lower(v) -> float:
    a = _f(v)
    return _load().orc_median_lower(_p(a), a.shape[0])


class State:
    """Oracle family state (Ready fields + rho), prepared mode."""

    def __init__(self, time, v, w, deficit, baseline_norm, origin, residual_energy, inflation, segments,
                 durations, rho):
        self.time, self.v, self.w, self.deficit = time, v, w, deficit
        self.baseline_norm, self.origin, self.residual_energy = baseline_norm, origin, residual_energy
        self.inflation, self.segments = inflation, segments
        self.durations, self.rho = durations, rho

    @property
    def n(self) -> int:
        return int(self.time.shape[0])


_STATUS = {1: "insufficient usable observations", 2: "mission flux must have a positive median",
           3: "no adjacent observations available for noise estimation", 4: "invalid baseline precision"}


def family_state(time, flux, sigma, durations_days, correlated=True) -> State:
    lib = _load()
    t, f, s, d = _f(time), _f(flux), _f(sigma), _f(durations_days)
    n_in = t.shape[0]
    n = C.c_int64(0)
    to, vo, wo, do = (np.empty(max(n_in, 1)) for _ in range(4))
    sc = np.empty(5)
    rho = np.empty(max(len(d), 1))
    rc = lib.orc_family_state(_p(t), _p(f), _p(s), n_in, _p(d), len(d), int(correlated), C.byref(n), _p(to), _p(vo),
                              _p(wo), _p(do), _p(sc), _p(rho))
    if rc:
        raise ValueError(_STATUS.get(rc, f"status {rc}"))
    k = n.value
    return State(to[:k].copy(), vo[:k].copy(), wo[:k].copy(), do[:k].copy(), sc[0], sc[1], sc[2], sc[3], int(sc[4]),
                 d.copy(), rho[:len(d)].copy())


def fit_segment_noise(time, flux, err, gap_days=0.75):
    """(time, deficit, variance, origin, inflation, segments) of curve.rs:89-198 at bin 0."""
    lib = _load()
    t, f, e = _f(time), _f(flux), _f(err)
    n = C.c_int64(0)
    to, do, vo = (np.empty(max(t.shape[0], 1)) for _ in range(3))
    sc = np.empty(3)
    rc = lib.orc_fit_segment_noise(_p(t), _p(f), _p(e), t.shape[0], gap_days, C.byref(n), _p(to), _p(do), _p(vo),
                                   _p(sc))
    if rc:
        raise ValueError(_STATUS.get(rc, f"status {rc}"))
    k = n.value
    return to[:k].copy(), do[:k].copy(), vo[:k].copy(), sc[0], sc[1], int(sc[2])


def transit_mask(time, period, epoch, duration, margin) -> np.ndarray:
    t = _f(time)
    m = np.zeros(t.shape[0], dtype=np.uint8)
    _load().orc_transit_mask(_p(t), t.shape[0], period, epoch, duration, margin,
                             m.ctypes.data_as(C.POINTER(C.c_uint8)))
    return m.astype(bool)


def biweight_flatten(time, relative_flux, window: float, gap: float = 0.5, c: float = 5.0, iterations: int = 10,
                     sorted_medians: bool = False) -> np.ndarray:
    """Biweight detrend: the reference's GPU form (bisection medians,
    kernels.rs:1051-1110) or, with sorted_medians, its CPU form
    (curve.rs:202-250)."""
    t, f = _f(time), _f(relative_flux)
    out = np.empty_like(t)
    _load().orc_biweight_flatten(_p(t), _p(f), t.shape[0], float(window), float(gap), float(c), int(iterations),
                                 int(sorted_medians), _p(out))
    return out


# -- raw-mode preparation (curve.rs:89-198, :332-425), restated in Python ------

def _median_lower_py(v) -> float:
    v = np.sort(np.asarray(v, dtype=np.float64)[np.isfinite(v)])
    return float(v[(v.shape[0] - 1) // 2]) if v.shape[0] else math.nan


def _mad_scale_py(v) -> float:
    v = np.asarray(v, dtype=np.float64)
    m = _median_lower_py(v)
    return 1.4826 * _median_lower_py(np.abs(v - m))


def _round_half_away(y: float) -> float:
    r = math.trunc(y)
    return r + math.copysign(1.0, y) if abs(y - r) >= 0.5 else float(r)


def fit_segment_noise_raw(time, flux, err=None, group=None, bin_minutes: float = 0.0, gap_days: float = 0.75):
    """fit_segment_noise (curve.rs:89-198) with groups and bins: (time,
    deficit, variance, group, origin, inflation, segments)."""
    t_in, f_in = _f(time), _f(flux)
    n = t_in.shape[0]
    e_in = np.ones(n) if err is None else _f(err)
    g_in = np.zeros(n, dtype=np.int64) if group is None else np.asarray(group, dtype=np.int64)
    keep = np.flatnonzero(np.isfinite(t_in) & np.isfinite(f_in) & np.isfinite(e_in) & (e_in > 0.0))
    keep = keep[np.argsort(t_in[keep], kind="stable")]
    t, f, e, sec = t_in[keep].copy(), f_in[keep].copy(), e_in[keep].copy(), g_in[keep].copy()
    if t.shape[0] < 6:
        raise ValueError("insufficient usable observations")
    for label in np.unique(sec):
        idx = np.flatnonzero(sec == label)
        m = _median_lower_py(f[idx])
        if not m > 0.0:
            raise ValueError("mission flux must have a positive median")
        f[idx] = f[idx] / m - 1.0
        e[idx] = e[idx] / m
    origin = float(t[0])
    t = t - origin
    if bin_minutes > 0.0:
        width = bin_minutes / 1440.0
        keys = list(zip(np.floor(t / width).astype(np.int64).tolist(), sec.tolist()))
        uniq = sorted(set(keys))
        at = {k: i for i, k in enumerate(uniq)}
        m = len(uniq)
        den, st, sf = [0.0] * m, [0.0] * m, [0.0] * m
        for i, k in enumerate(keys):  # in observation order, as the reference
            j = at[k]
            w = 1.0 / (e[i] * e[i])
            den[j] += w
            st[j] += t[i] * w
            sf[j] += f[i] * w
        den, st, sf = np.array(den), np.array(st), np.array(sf)
        tb, fb, eb = st / den, sf / den, 1.0 / np.sqrt(den)
        sb = np.array([k[1] for k in uniq], dtype=np.int64)
        o = np.argsort(tb, kind="stable")
        t, f, e, sec = tb[o], fb[o], eb[o], sb[o]
    adj = (np.diff(t) < gap_days) & (sec[1:] == sec[:-1])
    deltas = (f[1:] - f[:-1])[adj]
    if deltas.shape[0] == 0:
        raise ValueError("no adjacent observations available for noise estimation")
    standardized = deltas / np.sqrt(e[1:][adj] * e[1:][adj] + e[:-1][adj] * e[:-1][adj])
    ms = _mad_scale_py(standardized)
    inflation = ms if ms > 1.0 else 1.0
    if err is not None:
        variance = (e * inflation) ** 2
    else:
        md = _median_lower_py(deltas)
        white = max(1.4826 / math.sqrt(2.0) * _median_lower_py(np.abs(deltas - md)), 1e-12)
        variance = np.full(t.shape[0], white * white)
    segments = 1 + int(np.count_nonzero((np.diff(t) > gap_days) | (sec[1:] != sec[:-1])))
    return t, -f, variance, sec, origin, inflation, segments


def segment_edges_py(t, gap: float) -> np.ndarray:
    out = np.zeros(len(t))
    start = 0
    for i in range(1, len(t) + 1):
        if i == len(t) or t[i] - t[i - 1] > gap:
            for j in range(start, i):
                out[j] = min(t[j] - t[start], t[i - 1] - t[j])
            start = i
    return out


def prepare_families(time, flux, err, group, durations, cfg):
    """prepare_families (curve.rs:384-425) on the oracle: [(time absolute,
    flux, sigma, window, clipped, indices)] per detrending window."""
    t, deficit, variance, _, origin, _, _ = fit_segment_noise_raw(time, flux, err, group, cfg.bin_minutes, 0.75)
    sigma = np.sqrt(variance)
    edge = segment_edges_py(t, 0.5)
    relative = -deficit
    win = []
    for d in durations:
        x = min(max(cfg.window_factor * d, cfg.window_days), cfg.window_max_days)
        win.append(_round_half_away(x * 1e6) / 1e6)
    out = []
    for w in sorted(set(win)):
        flat = biweight_flatten(t, relative, w, 0.5, 5.0, 10)
        scale = _mad_scale_py(flat)
        keep = np.isfinite(flat) & (flat <= cfg.clip_sigma * scale) & (edge >= cfg.edge_trim_windows * w)
        out.append((t[keep] + origin, flat[keep], sigma[keep], w, int(flat.shape[0] - keep.sum()),
                    [i for i, x in enumerate(win) if x == w]))
    return out


def rescore_rows(time, v, w, excluded, rows, origin: float) -> np.ndarray:
    """(R, 3) box sums a, hp, norm per row (kernels.rs:936-990)."""
    t, vv, ww = _f(time), _f(v), _f(w)
    ex = np.ascontiguousarray(excluded, dtype=np.uint8)
    r = _f(rows).reshape(-1, 3)
    out = np.zeros((r.shape[0], 3))
    _load().orc_rescore_rows(_p(t), _p(vv), _p(ww), ex.ctypes.data_as(C.POINTER(C.c_uint8)), t.shape[0], _p(r),
                             r.shape[0], float(origin), _p(out))
    return out


def count_rows(time, excluded, rows) -> np.ndarray:
    """(R, 2) in-transit and not-excluded in-transit counts per row (kernels.rs:993-1042)."""
    t = _f(time)
    ex = np.ascontiguousarray(excluded, dtype=np.uint8)
    r = _f(rows).reshape(-1, 3)
    out = np.zeros((r.shape[0], 2), dtype=np.uint32)
    _load().orc_count_rows(_p(t), ex.ctypes.data_as(C.POINTER(C.c_uint8)), t.shape[0], _p(r), r.shape[0],
                           out.ctypes.data_as(C.POINTER(C.c_uint32)))
    return out


# -- scan path ------------------------------------------------------------------

def scan_bank(state: State, periods, nb: int, durations, rho, ingress=(0.0, 0.2, 0.45), layers=4,
              shape_gate=0.6 * 7.1, mode: int = 0, threads: Optional[int] = None):
    """Every period's winner at nb bins: (records Px9, score, depth, flags_or, rescans)."""
    lib = _load()
    p, d, r, g = _f(periods), _f(durations), _f(rho), _f(ingress)
    P = p.shape[0]
    rec = np.empty((P, 9))
    score = np.empty(P)
    depth = np.empty(P)
    flags = np.zeros(P, dtype=np.uint32)
    threads = threads or min(os.cpu_count() or 1, 64)
    rescans = lib.orc_scan_bank(_p(state.time), _p(state.v), _p(state.w), state.n, state.baseline_norm, _p(p), P, nb,
                                _p(d), _p(r), len(d), _p(g), len(g), layers, shape_gate, mode, threads, _p(rec),
                                _p(score), _p(depth), flags.ctypes.data_as(C.POINTER(C.c_uint32)))
    return rec, score, depth, flags, int(rescans)


def _rows(state: State, rec, score, depth, idx) -> np.ndarray:
    out = np.empty((len(idx), 5))
    for o, i in enumerate(idx):
        r = rec[i]
        out[o] = (r[0], (r[2] + r[3] / 2.0) / r[1] + state.origin, r[3] / r[1], score[i], depth[i])
    return out


def scan_periods(state: State, periods, durations, rho, cfg, threads=None):
    """scan_periods (scan.rs:363-408): rows at or above the threshold and stats."""
    periods = _f(periods)
    stats = {"periods": len(periods), "prescan_survivors": 0, "phase_bins": 0, "templates_scanned": 0}
    if len(periods) == 0 or len(durations) == 0:
        return np.zeros((0, 5)), stats
    gate = cfg.shape_gate_fraction * cfg.threshold if cfg.ingress_fractions[0] == 0.0 else 0.0
    mode = int(getattr(cfg, "precision_mode", 0))
    dmin = min(durations)
    nb = max(8, int(math.ceil(cfg.phase_oversample * periods[-1] / dmin)))
    ns = len(cfg.ingress_fractions)
    kw = dict(ingress=cfg.ingress_fractions, layers=cfg.shape_layers, shape_gate=gate, mode=mode, threads=threads)
    survivors = periods
    if cfg.prescan_factor > 1 and nb // cfg.prescan_factor >= 8:
        nbc = nb // cfg.prescan_factor
        rec, score, depth, flags, _ = scan_bank(state, periods, nbc, durations, rho, **kw)
        if np.any(flags & 2):
            raise ValueError("nonpositive template precision; inspect noise model")
        stats["phase_bins"] = nbc
        stats["templates_scanned"] += len(periods) * len(durations) * ns * nbc
        keep = np.isfinite(score) & (score >= cfg.prescan_fraction * cfg.threshold)
        survivors = rec[keep, 0].copy()
        stats["prescan_survivors"] = int(keep.sum())
    rows = np.zeros((0, 5))
    if len(survivors):
        rec, score, depth, flags, _ = scan_bank(state, survivors, nb, durations, rho, **kw)
        if np.any(flags & 2):
            raise ValueError("nonpositive template precision; inspect noise model")
        stats["phase_bins"] = nb
        stats["templates_scanned"] += len(survivors) * len(durations) * ns * nb
        keep = np.nonzero(np.isfinite(score) & (score >= cfg.threshold))[0]
        rows = _rows(state, rec, score, depth, keep)
    return rows, stats


def band_plan(state: State, cfg):
    order = np.argsort(state.durations, kind="stable")
    ds, rs = state.durations[order], state.rho[order]
    baseline = float(state.time[-1])
    maximum = min(cfg.period_max, baseline)
    minimum = max(cfg.period_min, 4.0 * ds[0] * (1.0 + 1e-9))
    if maximum <= minimum:
        return np.zeros(0), []
    grid = period_grid(minimum, maximum, baseline, float(ds[0]), cfg.period_oversample)
    bands = []
    lo = grid[0]
    while lo <= grid[-1]:
        hi = lo * 2.0
        sel = grid[(grid >= lo) & (grid < hi)]
        ch = ds < lo / 4.0
        if sel.size and ch.any():
            bands.append((sel, ds[ch], rs[ch]))
        lo = hi
    return grid, bands


def signal_search(state: State, cfg, threads=None):
    """signal_search (scan.rs:413-473): (rows, grid, per-band stats)."""
    grid, bands = band_plan(state, cfg)
    rows, stats = [], []
    for sel, d, r in bands:
        rr, st = scan_periods(state, sel, d, r, cfg, threads=threads)
        rows.append(rr)
        stats.append(st)
    return (np.concatenate(rows) if rows else np.zeros((0, 5))), grid, stats


def fold_prefix(state: State, scale: float, nb: int):
    lib = _load()
    folded = np.empty((nb, 3))
    cum = np.empty((3, 2 * nb + 1))
    cum32 = np.empty((3, 2 * nb + 1, 2), dtype=np.float32)
    lib.orc_fold_prefix(_p(state.time), _p(state.v), _p(state.w), state.n, scale, nb, _p(folded), _p(cum),
                        cum32.ctypes.data_as(C.POINTER(C.c_float)))
    return folded, cum, cum32


def single_event_search(state: State, cfg, capacity: int = 131072):
    """events.rs:18-153: rows (period inf, epoch, duration, score, depth) of
    every template above threshold at one trial period longer than the
    baseline, in (phase, duration, shape) order, and the stats
    (templates_scanned, threshold_survivors, overflow)."""
    order = np.argsort(np.asarray(state.durations), kind="stable")
    d = _f(np.asarray(state.durations)[order])
    r = _f(np.asarray(state.rho)[order])
    baseline = float(state.time[-1])
    trial = baseline + 2.0 * float(d[-1]) + 1e-6
    nb = max(8, int(math.ceil(cfg.phase_oversample * trial / float(d[0]))))
    scale = nb / trial
    ing = _f(cfg.ingress_fractions)
    rec = np.empty((capacity, 4))
    count = _load().orc_single_event_scan(_p(state.time), _p(state.v), _p(state.w), state.n, state.baseline_norm,
                                          scale, nb, _p(d), _p(r), d.shape[0], _p(ing), ing.shape[0],
                                          cfg.shape_layers, cfg.threshold, capacity, _p(rec))
    stats = {"templates_scanned": nb * d.shape[0] * ing.shape[0], "threshold_survivors": int(count),
             "overflow": bool(count > capacity)}
    if count > capacity:
        return np.empty((0, 5)), stats
    rec = rec[:count]
    rows = np.column_stack([np.full(count, np.inf), (rec[:, 0] + rec[:, 1] / 2.0) / scale + state.origin,
                            rec[:, 1] / scale, rec[:, 2], rec[:, 3]])
    return rows, stats


def box_direct(state: State, scale: float, nb: int, j: int, k: int):
    out = np.empty(3)
    _load().orc_box_direct(_p(state.time), _p(state.v), _p(state.w), state.n, scale, nb, j, k, _p(out))
    return out


# -- evidence -------------------------------------------------------------------

EVIDENCE_FIELDS = ("period", "epoch", "duration", "snr", "depth", "planet_log_odds", "log_bf_planet_noise",
                   "log_bf_binary_noise", "binary_secondary_ratio", "binary_secondary_phase", "binary_odd_even_ratio",
                   "binary_period_days", "ingress_fraction", "selection_flags")


def _evidence_cfg(cfg) -> np.ndarray:
    srs = math.nan if cfg.stellar_radius_solar is None else cfg.stellar_radius_solar
    return np.array([cfg.target_flux_fraction, cfg.planet_depth_scale, cfg.binary_depth_scale,
                     cfg.diluted_binary_depth_scale, cfg.planet_prior, cfg.binary_prior, srs,
                     cfg.planet_radius_scale_rj, cfg.threshold, cfg.evidence_rtol, float(cfg.phase_oversample),
                     float(cfg.shape_layers)])


def evidence_parameters(cfg) -> np.ndarray:
    c = _evidence_cfg(cfg)
    p = np.empty(30)
    _load().orc_evidence_parameters(_p(c), _p(p))
    return p


def compare_search(state: State, period: float, cfg, diag: bool = False):
    """compare_search (evidence.rs:693-1003): list of row dicts."""
    lib = _load()
    c = _evidence_cfg(cfg)
    g = _f(cfg.ingress_fractions)
    out = np.zeros(28)
    dg = np.zeros(8)
    n = lib.orc_compare_search(_p(state.time), _p(state.v), _p(state.w), state.n, state.baseline_norm, state.origin,
                               state.residual_energy, _p(_f(state.durations)), _p(_f(state.rho)), len(state.durations),
                               _p(g), len(g), float(period), _p(c), _p(out), _p(dg))
    rows = [dict(zip(EVIDENCE_FIELDS, out[14 * i:14 * (i + 1)])) for i in range(n)]
    for r in rows:
        r["selection_flags"] = int(r["selection_flags"])
    if diag:
        return rows, dict(zip(("nb", "nd", "tiles", "screen_max", "pilot_key", "floor_p", "floor_b", "log_mass"), dg))
    return rows
