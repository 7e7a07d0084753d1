#!/usr/bin/env python
"""Writes the golden fixtures of this directory. Run it from the repository
root where the reference's sources are present:

    python tests/golden/make_golden.py --reference <path to the reference's source tree>

reference_kats.json
    The known-answer values of the reference's own unit tests, read from its
    Rust test sources as text (nothing of the reference is run): the erfc
    table (src/search/math.rs:183-210), the period-grid property test's
    arguments (src/search/grid.rs:34-42), the segment-edge and
    detrending-window cases (src/prep/curve.rs:609-622). Each entry records
    the file and lines it was read from.

oracle_small.json / oracle_small.npz
    Seeded small inputs (the 821-point curve with one injected box, a 6-day
    curve with one single event, a 3,000-point detrending series) and the
    oracle's outputs on them: the prepared family, every band's records at
    the coarse and the full phase-bin count in both precision modes, the
    signal_search rows and stats, model-comparison rows at five periods,
    rescoring sums and counts of 1,000 rows with and without excluded points,
    the single-event rows and stats, and the biweight-detrended series. The
    oracle's outputs are frozen here so that a change of the oracle shows up
    as a failing CPU test, and the GPU tests compare the CUDA path with these
    same files.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from fbls_b200 import api, synth  # noqa: E402

EVIDENCE_PERIODS = [1.3, 1.30481313, 0.9, 2.6, 1.95]
FLOAT = r"-?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?"


def _block(lines, start_pattern, end_pattern, first=0):
    """(first line index, last line index) of the block that starts at the
    first line matching start_pattern at or after `first` and ends at the
    next line matching end_pattern."""
    a = next(i for i in range(first, len(lines)) if re.search(start_pattern, lines[i]))
    b = next(i for i in range(a, len(lines)) if re.search(end_pattern, lines[i]))
    return a, b


def _ratio(expr: str) -> float:
    """A literal `x` or `x / y` of the reference's test sources."""
    parts = [float(p) for p in expr.split("/")]
    return parts[0] / parts[1] if len(parts) == 2 else parts[0]


def reference_kats(ref: Path) -> dict:
    out = {}
    # erfc table
    path = "src/search/math.rs"
    lines = (ref / path).read_text().splitlines()
    a, b = _block(lines, r"fn erfc_reference_values", r"^\s*\];")
    cases = [[float(x), float(y)] for line in lines[a:b + 1]
             for x, y in re.findall(rf"\(\s*({FLOAT})\s*,\s*({FLOAT})\s*\)", line)]
    tol = re.search(rf"<\s*({FLOAT})", "\n".join(lines[b:b + 8]))
    assert len(cases) == 16 and tol, (len(cases), tol)
    out["erfc"] = {"source": f"{path}:{a + 1}-{b + 1}", "cases": cases, "rel_tol": float(tol.group(1))}
    # period grid property
    path = "src/search/grid.rs"
    lines = (ref / path).read_text().splitlines()
    a, b = _block(lines, r"fn grid_bounds_and_drift", r"^\s*\}\s*$")
    text = "\n".join(lines[a:b + 1])
    args = [float(x) for x in re.search(r"period_grid\(([^)]*)\)", text).group(1).split(",")]
    slack = float(re.search(rf"\(1\.0 \+ ({FLOAT})\)", text).group(1))
    assert len(args) == 5
    out["period_grid"] = {"source": f"{path}:{a + 1}-{b + 1}", "args": args, "drift_slack": slack}
    # segment edges and detrending windows
    path = "src/prep/curve.rs"
    lines = (ref / path).read_text().splitlines()
    a, b = _block(lines, r"fn edges_follow_gap_separated_segments", r"^\s*\}\s*$")
    text = "\n".join(lines[a:b + 1])
    t = [float(x) for x in re.search(r"let t = \[([^\]]*)\]", text).group(1).split(",")]
    call = re.search(rf"segment_edges\(&t,\s*({FLOAT})\),\s*vec!\[([^\]]*)\]", text)
    out["segment_edges"] = {"source": f"{path}:{a + 1}-{b + 1}", "time": t, "gap": float(call.group(1)),
                            "want": [float(x) for x in call.group(2).split(",")]}
    a, b = _block(lines, r"fn windows_group_equal_clamped_values", r"^\s*\}\s*$")
    text = "\n".join(lines[a:b + 1])
    d = [_ratio(x) for x in re.search(r"let d = \[([^\]]*)\]", text).group(1).split(",")]
    wargs = [float(x) for x in re.search(r"detrending_windows\(&d,\s*([^)]*)\)", text).group(1).split(",")]
    first = re.search(rf"w\[0\], \(({FLOAT}), vec!\[([^\]]*)\]\)", text)
    rest = [(int(i), float(v)) for i, v in re.findall(rf"w\[(\d+)\]\.0, ({FLOAT})\)", text)]
    out["detrending_windows"] = {"source": f"{path}:{a + 1}-{b + 1}", "durations": d, "args": wargs,
                                 "first": [float(first.group(1)), [int(x) for x in first.group(2).split(",")]],
                                 "window_days": rest}
    return out


def single_event_curve(days=6.0, cadence_s=600.0, seed=3):
    """A curve with one transit-like dip of 4e-3 at 0.37 of its span."""
    rng = np.random.default_rng(seed)
    t = synth.T0 + np.arange(int(days * 86400 / cadence_s)) * cadence_s / 86400.0
    flux = rng.normal(0.0, 1e-3, t.shape[0])
    mid = synth.T0 + 0.37 * days
    flux[np.abs(t - mid) <= 0.06] -= 4e-3
    return t, flux, np.full_like(t, 1e-3)


def detrend_series(seed=1, n=3000):
    """Two segments, a sine trend, noise and 20 outliers."""
    rng = np.random.default_rng(seed)
    t = np.sort(np.concatenate([rng.uniform(0.0, 5.0, n // 2), rng.uniform(5.7, 11.0, n - n // 2)]))
    f = 0.004 * np.sin(1.3 * t) + rng.normal(0.0, 1e-3, n)
    f[rng.integers(0, n, 20)] += 0.03
    return t, f


def rescore_inputs(st, table, seed=8):
    """Search rows, random rows, rows with an observation on a window edge
    and degenerate rows (zero, negative, NaN and infinite values)."""
    rng = np.random.default_rng(seed)
    ta = st.time + st.origin
    rand = np.column_stack([np.exp(rng.uniform(np.log(0.3), np.log(6.0), 600)),
                            rng.uniform(ta[0] - 2.0, ta[-1] + 2.0, 600), rng.uniform(0.01, 0.3, 600)])
    edge = []
    for j in rng.integers(0, ta.shape[0], 150):
        period, duration = rng.uniform(0.4, 3.0), rng.uniform(0.02, 0.2)
        edge.append([period, ta[j] - duration / 2.0 - period * rng.integers(-3, 4), duration])
        edge.append([period, ta[j] + duration / 2.0, duration])
    odd = [[0.0, ta[10], 0.1], [-2.0, ta[10], 0.1], [3.0, np.nan, 0.1], [3.0, ta[10], np.nan],
           [1.0, ta[10], 1.5], [2.0, ta[100], 0.0], [0.004, ta[10], 0.001], [5.0, ta[0] - 1e4, 0.2],
           [np.inf, ta[10], 0.2]]
    rows = np.vstack([table[:, :3], rand, np.array(edge), np.array(odd)])
    excluded = (rng.uniform(size=st.n) < 0.2).astype(np.uint8)
    return rows, excluded


def oracle_fixtures():
    arrays, meta = {}, {}
    c, cfg = synth.small_curve(), synth.small_config()
    meta["config"] = dataclasses.asdict(cfg)
    arrays.update(input_time=c.time, input_flux=c.flux, input_flux_err=c.flux_err)
    st = oracle.family_state(c.time, c.flux, c.flux_err, cfg.durations_days())
    arrays.update(state_time=st.time, state_v=st.v, state_w=st.w, state_durations=st.durations, state_rho=st.rho)
    meta["state"] = {"baseline_norm": st.baseline_norm, "origin": st.origin, "residual_energy": st.residual_energy}

    grid, bands = api.band_plan(st, cfg)
    meta["grid_len"] = int(len(grid))
    meta["bands"] = []
    for b, band in enumerate(bands):
        bank = api.bank_for(band, cfg)
        nbs = [band["nb"] // 2, band["nb"]]
        meta["bands"].append({"nb": int(band["nb"]), "nbs": nbs, "shape_gate": bank.shape_gate})
        arrays[f"b{b}_periods"] = band["periods"]
        arrays[f"b{b}_durations"] = band["durations"]
        arrays[f"b{b}_rho"] = band["rho"]
        for nb in nbs:
            for mode in (0, 1):
                rec, score, depth, flags, _ = oracle.scan_bank(st, band["periods"], nb, band["durations"], band["rho"],
                                                               ingress=cfg.ingress_fractions, layers=cfg.shape_layers,
                                                               shape_gate=bank.shape_gate, mode=mode)
                key = f"b{b}_nb{nb}_m{mode}"
                arrays[key + "_rec"], arrays[key + "_score"] = rec, score
                arrays[key + "_depth"], arrays[key + "_flags"] = depth, flags.astype(np.uint32) & 3

    rows, ogrid, stats = oracle.signal_search(st, cfg)
    assert len(ogrid) == len(grid)
    arrays["signal_rows"] = rows
    keys = ("periods", "prescan_survivors", "phase_bins", "templates_scanned")
    meta["signal_stats"] = [{k: int(s[k]) for k in keys} for s in stats]

    meta["evidence"] = []
    for period in EVIDENCE_PERIODS:
        ev = oracle.compare_search(st, period, cfg)
        meta["evidence"].append({"period": period, "rows": [{k: (int(v) if isinstance(v, (int, np.integer)) else float(v))
                                                             for k, v in r.items()} for r in ev]})

    rrows, excluded = rescore_inputs(st, rows)
    arrays["rescore_rows"], arrays["rescore_excluded"] = rrows, excluded
    none = np.zeros(st.n, np.uint8)
    arrays["rescore_sums_none"] = oracle.rescore_rows(st.time, st.v, st.w, none, rrows, st.origin)
    arrays["rescore_sums_excluded"] = oracle.rescore_rows(st.time, st.v, st.w, excluded, rrows, st.origin)
    ta = st.time + st.origin
    arrays["count_none"] = oracle.count_rows(ta, none, rrows)
    arrays["count_excluded"] = oracle.count_rows(ta, excluded, rrows)

    t, flux, err = single_event_curve()
    arrays.update(event_time=t, event_flux=flux, event_flux_err=err)
    est = oracle.family_state(t, flux, err, cfg.durations_days())
    erows, estats = oracle.single_event_search(est, cfg)
    arrays["event_rows"] = erows
    meta["event_stats"] = json.loads(json.dumps(estats))

    t, f = detrend_series()
    arrays.update(detrend_time=t, detrend_flux=f)
    meta["detrend"] = {"window": 0.5, "gap": 0.5, "iterations": 10}
    arrays["detrend_out"] = oracle.biweight_flatten(t, f, 0.5, gap=0.5, iterations=10)
    return arrays, meta


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="the reference's source tree (read as text)")
    args = ap.parse_args()
    ref = Path(args.reference)
    if ref.exists():
        kats = reference_kats(ref)
        (HERE / "reference_kats.json").write_text(json.dumps(kats, indent=1) + "\n")
    else:
        print(f"{ref} not found: reference_kats.json left as it is")
    arrays, meta = oracle_fixtures()
    (HERE / "oracle_small.json").write_text(json.dumps(meta, indent=1) + "\n")
    np.savez_compressed(HERE / "oracle_small.npz", **arrays)
    print("wrote", sorted(p.name for p in HERE.iterdir() if p.suffix in (".json", ".npz")))


if __name__ == "__main__":
    main()
