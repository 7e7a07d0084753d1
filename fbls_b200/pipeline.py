"""The search around the hot path (src/pipeline.rs, src/main.rs:145-229):
raw or prepared observations to families, passes of signal search and peak
selection with each pass's leading signal masked, Bayesian evidence for the
strongest peaks, single events, and the schema-3 JSON report.

    python -m fbls_b200 search --input a.npz b.fits [--prepared] [--output report.json]
        [--save-table table.csv] [--device 0] [--pmin P] [--pmax P] [--prescan K] [--threshold T]

Every GPU step is this library's (fbls_prepare_families, fbls_signal_search,
fbls_rescore_rows / fbls_count_rows through select_peaks, fbls_compare_search,
fbls_single_event_search); the rest is host logic restated from the
reference.
"""
from __future__ import annotations

import dataclasses
import json
import math
import sys
import time as _time
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import api, select
from .config import SearchConfig
from .io import Observations, read_inputs

SCHEMA_VERSION = 3
CANDIDATE_CAPACITY = 131072  # pipeline.rs:14


@dataclasses.dataclass
class Curve:
    """A family's detrended curve (PreparedCurve, curve.rs:35-43)."""
    time: np.ndarray   # absolute
    flux: np.ndarray
    sigma: np.ndarray
    window_days: float = math.nan
    clipped: int = 0


@dataclasses.dataclass
class Family:
    curve: Curve
    durations: np.ndarray   # days
    indices: List[int]
    state: api.FamilyState


def family_state(curve: Curve, durations, indices, correlated: bool) -> Family:
    """family_state (curve.rs:541-569)."""
    st = api.family_state(curve.time, curve.flux, curve.sigma, durations, correlated)
    return Family(curve, np.asarray(durations, dtype=np.float64), list(indices), st)


def mask_curve(curve: Curve, period: float, epoch: float, duration: float, margin: float) -> Curve:
    """The curve without the observations of one ephemeris (curve.rs:587-606)."""
    keep = ~select.transit_mask(curve.time, period, epoch, duration, margin)
    return Curve(curve.time[keep], curve.flux[keep], curve.sigma[keep], curve.window_days, curve.clipped)


def merged_time(families: Sequence[Family]) -> np.ndarray:
    """Every family's times, sorted, duplicates dropped (pipeline.rs:16-24)."""
    return np.unique(np.concatenate([f.curve.time for f in families]))


def search_transits(gpu: api.Gpu, obs: Observations, cfg: SearchConfig, device: int = 0) -> dict:
    """Raw mission flux: normalised, binned and detrended per duration family
    on the GPU, then searched (pipeline.rs:26-37)."""
    start = _time.perf_counter()
    d = cfg.durations_days()
    fams = []
    for pc in gpu.prepare_families(obs.time, obs.flux, obs.err, obs.group, cfg):
        fams.append((Curve(pc.time, pc.flux, pc.sigma, pc.window_days, pc.clipped), [int(i) for i in pc.indices]))
    return search_families(gpu, fams, d, cfg, device, start)


def search_prepared(gpu: api.Gpu, obs: Observations, cfg: SearchConfig, device: int = 0) -> dict:
    """Detrended fractional flux with per-observation errors, searched as one
    family with every duration (pipeline.rs:39-68)."""
    if obs.err is None:
        raise ValueError("prepared input requires flux_err")
    ok = np.isfinite(obs.time) & np.isfinite(obs.flux) & np.isfinite(obs.err) & (obs.err > 0.0)
    keep = np.flatnonzero(ok)
    keep = keep[np.argsort(obs.time[keep], kind="stable")]
    curve = Curve(obs.time[keep], obs.flux[keep], obs.err[keep])
    d = cfg.durations_days()
    return search_families(gpu, [(curve, list(range(len(d))))], d, cfg, device, _time.perf_counter())


def _finite(x: float) -> Optional[float]:
    return float(x) if math.isfinite(x) else None


# ScanStats as the reference serialises it (scan.rs:24-37); the library's
# fbls_scan_stats adds tile_rescans, which the schema-3 report leaves out.
SCAN_STATS_FIELDS = ("periods", "prescan_survivors", "phase_bins", "batches", "templates_scanned",
                     "exact_tile_retries", "seconds", "seconds_fold", "seconds_cumulative", "seconds_scan")


def _scan_stats_json(stats: dict) -> dict:
    return {k: stats[k] for k in SCAN_STATS_FIELDS if k in stats}


def _config_json(cfg: SearchConfig) -> dict:
    """SearchConfig as the reference serialises it (config.rs:5-88): its
    fields only; this library's precision_mode appears only when a run asks
    for f64 ranking, which the reference does not have."""
    out = dataclasses.asdict(cfg)
    if out.get("precision_mode", 0) == 0:
        out.pop("precision_mode", None)
    return out


def _peak_json(p: select.Peak) -> dict:
    """The fields in the reference's order (Peak, peaks.rs:18-45), `pass_`
    written as "pass" in its place and `row` left out (not serialised there)."""
    return {("pass" if k == "pass_" else k): v for k, v in dataclasses.asdict(p).items() if k != "row"}


def search_families(gpu: api.Gpu, fams: List[Tuple[Curve, List[int]]], durations: Sequence[float],
                    cfg: SearchConfig, device: int, start: float) -> dict:
    """pipeline.rs:70-290."""
    durations = np.asarray(durations, dtype=np.float64)
    states = [family_state(c, durations[idx], idx, cfg.correlated_noise) for c, idx in fams]
    original = list(states)
    preparation_seconds = _time.perf_counter() - start
    time_all = merged_time(states)
    if time_all.shape[0] < 6:
        raise ValueError("at least six usable observations are required")
    baseline = float(time_all[-1] - time_all[0])
    search_start = _time.perf_counter()
    peaks: List[select.Peak] = []
    masks: List[np.ndarray] = []
    excluded = np.zeros(time_all.shape[0], dtype=bool)
    pass_stats, first_table = [], np.empty((0, 5))
    periods_tested = 0
    seconds_scan = seconds_select = 0.0
    for pass_ in range(cfg.passes):
        scan_start = _time.perf_counter()
        tables, family, band_stats = [], [], []
        for k, fam in enumerate(states):
            rows, grid_len, stats = gpu.signal_search(fam.state, cfg)
            if pass_ == 0:
                periods_tested += grid_len
            band_stats.append({
                "family": k, "window_days": _finite(fam.curve.window_days), "observations": int(fam.curve.time.shape[0]),
                "clipped": fam.curve.clipped, "error_inflation": fam.state.inflation, "segments": fam.state.segments,
                "durations_hours": (fam.durations * 24.0).tolist(), "periods": grid_len,
                "rho": fam.state.rho.tolist(), "bands": [_scan_stats_json(b) for b in stats]})
            family += [k] * rows.shape[0]
            tables.append(rows)
        table = np.vstack(tables) if tables else np.empty((0, 5))
        if pass_ == 0:
            first_table = table.copy()
        seconds_scan += _time.perf_counter() - scan_start
        select_start = _time.perf_counter()
        sel = select.select_peaks(gpu, table, np.array(family, dtype=np.int64), [f.state for f in states], time_all,
                                  cfg.threshold, cfg.max_candidates - len(peaks), cfg.min_events, masks, excluded,
                                  pass_ + 1)
        masks, excluded = sel.masks, sel.excluded
        seconds_select += _time.perf_counter() - select_start
        pass_stats.append({"pass": pass_ + 1, "rows": int(table.shape[0]), "accepted": len(sel.accepted),
                           "families": band_stats})
        if not sel.accepted:
            break
        lead = sel.accepted[0]
        peaks += sel.accepted
        if pass_ + 1 < cfg.passes:
            # The next pass searches every family with the leading signal
            # masked; a family left with too few observations fails, as in
            # the reference (pipeline.rs:145-163).
            states = [family_state(mask_curve(f.curve, lead.period_days, lead.epoch_bjd, lead.duration_hours / 24.0,
                                              0.5), f.durations, f.indices, cfg.correlated_noise) for f in states]
            if any(f.curve.time.shape[0] < 6 for f in states):
                break

    evidence_seconds = 0.0
    if cfg.model_comparison and peaks:
        ev_start = _time.perf_counter()
        order = sorted(range(len(peaks)), key=lambda i: -peaks[i].snr)
        # Every candidate's family (the others' transits masked), then one
        # batched evidence call for all of them (fbls_compare_batch); the rows
        # are those of one compare_search per peak (pipeline.rs:169-192).
        chosen, cands = [], []
        for index in order[:cfg.evidence_candidates]:
            peak = peaks[index]
            base = original[peak.family]
            curve = base.curve
            for other in peaks:
                if (other.row, other.pass_, other.family) != (peak.row, peak.pass_, peak.family):
                    curve = mask_curve(curve, other.period_days, other.epoch_bjd, other.duration_hours / 24.0, 0.5)
            if curve.time.shape[0] < 6:
                continue
            state = family_state(curve, base.durations, base.indices, cfg.correlated_noise)
            chosen.append(peak)
            cands.append((state.state, peak.period_days))
        results = gpu.compare_batch(cands, cfg) if cands else []
        for peak, rows in zip(chosen, results):
            row = next((r for r in rows if int(r["selection_flags"]) & 1), rows[0] if rows else None)
            if row is None:
                continue
            p = peak
            p.planet_log_odds = _finite(row["planet_log_odds"])
            p.log_bf_planet_noise = _finite(row["log_bf_planet_noise"])
            p.log_bf_binary_noise = _finite(row["log_bf_binary_noise"])
            p.binary_secondary_ratio = _finite(row["binary_secondary_ratio"])
            p.binary_secondary_phase = _finite(row["binary_secondary_phase"])
            p.binary_odd_even_ratio = _finite(row["binary_odd_even_ratio"])
            p.binary_period_days = _finite(row["binary_period_days"])
            p.ingress_fraction = _finite(row["ingress_fraction"])
            p.evidence_epoch_bjd = float(row["epoch"])
            p.evidence_duration_hours = 24.0 * float(row["duration"])
            p.model_preferred = bool(row["planet_log_odds"] >= cfg.planet_log_odds_min)
            p.binary_diagnostics_complete = all(math.isfinite(row[k]) for k in (
                "binary_secondary_ratio", "binary_secondary_phase", "binary_odd_even_ratio", "binary_period_days"))
        evidence_seconds = _time.perf_counter() - ev_start

    events: List[select.SingleEvent] = []
    event_stats = {}
    events_start = _time.perf_counter()
    if cfg.single_events:
        all_rows = []
        for k, fam in enumerate(states):
            table, stats = gpu.single_event_search(fam.state, cfg, CANDIDATE_CAPACITY)
            event_stats[str(k)] = stats
            for e in select.select_events(table, time_all, cfg.threshold, cfg.max_candidates, masks):
                all_rows.append([math.inf, e.epoch_bjd, e.duration_hours / 24.0, e.snr, e.depth])
        all_rows.sort(key=lambda r: -r[3])
        events = select.select_events(np.array(all_rows).reshape(-1, 5), time_all, cfg.threshold,
                                      cfg.max_candidates, masks)
    seconds_events = _time.perf_counter() - events_start

    by_signal = sorted(peaks, key=lambda p: -p.snr)

    def model_key(p):
        evidence = p.log_bf_planet_noise if p.model_preferred else None
        value = evidence if evidence is not None else p.planet_log_odds
        return (0 if p.model_preferred else 1, -(value if value is not None else -math.inf))

    by_model = sorted(peaks, key=model_key) if cfg.model_comparison else by_signal
    search_seconds = _time.perf_counter() - search_start
    table_rows = [dict(zip(api.ROW_FIELDS, map(float, r))) for r in first_table]
    return {
        "schema_version": SCHEMA_VERSION,
        "software_version": "fbls_b200 0.1",
        "config": _config_json(cfg),
        "statistics": {
            "device": f"cuda:{device}", "observations": int(time_all.shape[0]), "baseline_days": baseline,
            "periodic_period_max_days": min(cfg.period_max, baseline), "periods_tested": periods_tested,
            "qualifying_periods": int(first_table.shape[0]), "resolved_peaks": len(peaks),
            "single_events": len(events), "seconds_preparation": preparation_seconds,
            "seconds_search": search_seconds, "evidence": {"seconds_search": evidence_seconds},
            "seconds_scan": seconds_scan, "seconds_select": seconds_select, "seconds_single_events": seconds_events,
            "seconds_total": preparation_seconds + search_seconds, "passes": pass_stats,
            "single_event_scan": event_stats,
        },
        "candidates": [_peak_json(p) for p in by_model[:cfg.max_candidates]],
        "signal_candidates": [_peak_json(p) for p in by_signal[:cfg.max_candidates]],
        "single_events": [dataclasses.asdict(e) for e in events[:cfg.max_candidates]],
        "period_table": table_rows,
    }


def _json_default(x):
    if isinstance(x, (np.floating,)):
        return float(x)
    if isinstance(x, (np.integer,)):
        return int(x)
    if isinstance(x, np.ndarray):
        return x.tolist()
    raise TypeError(type(x))


def _clean(x):
    """Non-finite floats as null, as serde_json writes them."""
    if isinstance(x, float):
        return x if math.isfinite(x) else None
    if isinstance(x, dict):
        return {k: _clean(v) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [_clean(v) for v in x]
    return x


def run_search(argv: Sequence[str]) -> int:
    """`fbls search` (main.rs:145-229)."""
    inputs: List[str] = []
    output, table_path, prepared, device = "-", None, False, 0
    cfg = SearchConfig()
    i = 0
    while i < len(argv):
        a = argv[i]
        if a == "--input":
            i += 1
            while i < len(argv) and not argv[i].startswith("--"):
                inputs.append(argv[i])
                i += 1
            continue
        if a == "--prepared":
            prepared = True
        elif a in ("--output", "--save-table", "--device", "--pmin", "--pmax", "--prescan", "--threshold"):
            if i + 1 >= len(argv):
                raise ValueError(f"{a} needs a value")  # the reference indexes past the end and panics
            v = argv[i + 1]
            i += 1
            if a == "--output":
                output = v
            elif a == "--save-table":
                table_path = v
            elif a == "--device":
                device = int(v)
            elif a == "--pmin":
                cfg = dataclasses.replace(cfg, period_min=float(v))
            elif a == "--pmax":
                cfg = dataclasses.replace(cfg, period_max=float(v))
            elif a == "--prescan":
                cfg = dataclasses.replace(cfg, prescan_factor=int(v))
            else:
                cfg = dataclasses.replace(cfg, threshold=float(v))
        else:
            raise ValueError(f"unknown argument {a}")
        i += 1
    if not inputs:
        raise ValueError("--input is required")
    cfg.validate()
    obs = read_inputs(inputs)
    with api.Gpu(device) as gpu:
        report = (search_prepared if prepared else search_transits)(gpu, obs, cfg, device)
    report["input_files"] = list(inputs)
    report["input_mode"] = "prepared" if prepared else "raw"
    if table_path:
        with open(table_path, "w") as fh:
            fh.write("period_days,epoch_bjd,duration_days,snr,depth\n")
            for r in report["period_table"]:
                fh.write(f"{r['period']},{r['epoch']},{r['duration']},{r['score']},{r['depth']}\n")
    report.pop("period_table")
    # serde_json without preserve_order keeps every object in a BTreeMap, so the
    # reference writes all keys sorted (main.rs:221, to_string_pretty).
    text = json.dumps(_clean(report), indent=2, sort_keys=True, default=_json_default)
    if output == "-":
        print(text)
    else:
        with open(output, "w") as fh:
            fh.write(text)
    return 0


def main(argv: Optional[Sequence[str]] = None) -> int:
    args = list(sys.argv[1:] if argv is None else argv)
    try:
        if args and args[0] == "search":
            return run_search(args[1:])
        raise ValueError("usage: python -m fbls_b200 search --input FILE... [options]")
    except (ValueError, OSError, api.FblsError) as e:
        print(f"fbls: {e}", file=sys.stderr)
        return 1
