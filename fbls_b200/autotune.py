"""Autotuner of the fold's launch shape, measured on the GPU.

The fold's period group (periods per CTA, sharing each staged observation
chunk) trades shared memory for histograms against CTAs per launch; the
built-in rule takes the largest group whose histograms fit while every SM
still gets a CTA; caps above 32 give a period fewer lanes than a warp (down
to 8). The CTA size sets how many lanes split a staged chunk per
period, hence the segment each lane walks, and the lockstep threshold picks
between lanes stepping together (conflict-free reads, idle steps) and each
walking its own window. This sweep measures, per nb class floor(log2(nb)),
the fold's device time (CUDA events on the context's stream, the library's
kernel-timing counters) of one scan_bank pass over every period of an
octave band of the 13-sector synthetic star (the launches and period groups
of a search) at every allowed group cap, then at every CTA size
and lockstep threshold, the periods per launch and the fused against the
separate tile scan on a whole signal_search, and, on a batch of seeded
survey stars searched together, a CTA per fold unit against the persistent
work-stealing fold grid and the coarse maps' fold shape (group cap and CTA
size, then lockstep threshold); it writes
the fastest as a table:

    python -m fbls_b200.autotune --out fbls_b200/data/tuning.json

`Gpu` loads the table (fbls_set_tuning) when the device name matches. The
results of the search do not depend on it, only the launch shapes do.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time
from pathlib import Path

import numpy as np

from . import _native as N

TABLE = Path(__file__).resolve().parent / "data" / "tuning.json"
GROUPS = (1, 2, 4, 8, 16, 32, 64, 128)
LAUNCHES = (4096, 8192, 16384, 32768)
THREADS = (1024, 512, 256, 128)
PAIR_THREADS = (512, 256)
LOCKSTEP = (0, 3, 7, 15, 4096)  # 0: the built-in 11; 4096: never in lockstep
MAP_LOCKSTEP = (0, 3, 5, 7, 4096)
# (group cap, CTA size) of the coarse maps' walking folds; (0, 0) the built-in
MAP_SHAPES = ((0, 0), (16, 0), (32, 0), (64, 0), (128, 0), (32, 512), (64, 512))


def device_name(device: int = 0) -> str:
    import torch
    return torch.cuda.get_device_name(device)


def apply(table: dict) -> None:
    """Sets the process-wide tuning from a table (fbls_set_tuning)."""
    t = N.Tuning()
    for cls, g in table.get("fold_group_max", {}).items():
        t.fold_group_max[int(cls)] = int(g)
    for cls, th in table.get("fold_threads", {}).items():
        t.fold_threads[int(cls)] = int(th)
    for cls, lm in table.get("lockstep_min", {}).items():
        t.lockstep_min[int(cls)] = int(lm)
    for cls, pv in table.get("fold_pair", {}).items():
        t.fold_pair[int(cls)] = int(pv)
    t.launch_periods = int(table.get("launch_periods", 0))
    t.fold_steal = int(table.get("fold_steal", 0))
    t.fused_scan = int(table.get("fused_scan", 0))
    t.map_lockstep_min = int(table.get("map_lockstep_min", 0))
    t.map_threads = int(table.get("map_threads", 0))
    t.map_group_max = int(table.get("map_group_max", 0))
    t.batch_no_fill = int(table.get("batch_no_fill", 0))
    rc = N.load().fbls_set_tuning(C.byref(t))
    if rc:
        raise ValueError(f"tuning table rejected (status {rc})")


def current() -> dict:
    t = N.Tuning()
    N.load().fbls_get_tuning(C.byref(t))
    return {"fold_group_max": {str(c): int(g) for c, g in enumerate(t.fold_group_max) if g},
            "fold_threads": {str(c): int(v) for c, v in enumerate(t.fold_threads) if v},
            "lockstep_min": {str(c): int(v) for c, v in enumerate(t.lockstep_min) if v},
            "fold_pair": {str(c): int(v) for c, v in enumerate(t.fold_pair) if v},
            "launch_periods": int(t.launch_periods), "fold_steal": int(t.fold_steal),
            "fused_scan": int(t.fused_scan), "map_lockstep_min": int(t.map_lockstep_min),
            "map_threads": int(t.map_threads), "map_group_max": int(t.map_group_max),
            "batch_no_fill": int(t.batch_no_fill)}


def reset() -> None:
    apply({})


def load_for(device_name_: str, path: Path = TABLE) -> bool:
    """Applies the committed table when it was measured on this device model."""
    if not path.exists():
        return False
    table = json.loads(path.read_text())
    if table.get("device") != device_name_:
        return False
    apply(table)
    return True


def _median(xs) -> float:
    """The median of repeated timings (one slow step of a shared host does
    not move it)."""
    return float(np.median(np.asarray(xs, dtype=np.float64)))


def _fold_ms(gpu, dev, periods, bank, nb, reps: int) -> float:
    gpu.scan_bank(dev, periods, bank, nb)  # warm
    gpu.counters(reset=True)
    for _ in range(reps):
        gpu.scan_bank(dev, periods, bank, nb)
    return gpu.counters(reset=True)["fold_ms"] / reps


def sweep(reps: int = 3, log=print, survey_stars: int = 256) -> dict:
    from . import api, synth
    c, cfg = synth.multi_sector(), synth.multi_sector_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    grid, bands = api.band_plan(st, cfg)
    out = {"device": device_name(0),
           "workload": "13-sector synthetic star (247,104 observations), every period of an octave band at its "
                       "coarse and full nb; fold device time per pass (ms) by period-group cap, 0 = the rule",
           "fold_ms": {}, "fold_group_max": {}, "command": "python -m fbls_b200.autotune"}
    with api.Gpu(0, tuned=False) as gpu:
        dev = gpu.upload(st)
        gpu.set_kernel_timing(True)
        cases = {}
        for band in bands:
            for nb in (band["nb"] // 2, band["nb"]):
                cases.setdefault(int(np.floor(np.log2(nb))), (nb, band))
        out["fold_threads"], out["lockstep_min"], out["fold_pair"], out["shape_ms"] = {}, {}, {}, {}
        for cls, (nb, band) in sorted(cases.items()):
            bank = api.bank_for(band, cfg)
            # the whole band, so the launches have the period groups of a search
            periods = band["periods"]
            reset()
            times = {0: _fold_ms(gpu, dev, periods, bank, nb, reps)}  # the built-in rule
            for g in GROUPS:
                apply({"fold_group_max": {str(cls): g}})
                times[g] = _fold_ms(gpu, dev, periods, bank, nb, reps)
            reset()
            best = min(times, key=times.get)
            out["fold_ms"][str(cls)] = {"nb": int(nb), **{str(k): round(v, 4) for k, v in times.items()}}
            if best != 0 and times[best] < 0.98 * times[0]:
                out["fold_group_max"][str(cls)] = int(best)
            log(f"nb {nb} (class {cls}): " + ", ".join(f"G<={k or 'rule'}: {v:.3f} ms" for k, v in times.items())
                + f" -> {best or 'rule'}")
            # CTA size and lockstep threshold at the chosen group cap.
            caps = {str(cls): out["fold_group_max"][str(cls)]} if str(cls) in out["fold_group_max"] else {}
            shapes = {}
            for pair, ths in ((0, THREADS), (1, PAIR_THREADS)):
                for th in ths:
                    for lm in LOCKSTEP:
                        apply({"fold_group_max": caps, "fold_threads": {str(cls): th},
                               "lockstep_min": {str(cls): lm}, "fold_pair": {str(cls): pair}})
                        shapes[(pair, th, lm)] = _fold_ms(gpu, dev, periods, bank, nb, reps)
            reset()
            base = shapes[(0, 1024, 0)]
            bp, bth, blm = min(shapes, key=shapes.get)
            out["shape_ms"][str(cls)] = {f"{'pair ' if p else ''}{th}/{lm or 'rule'}": round(v, 4)
                                         for (p, th, lm), v in shapes.items()}
            if shapes[(bp, bth, blm)] < 0.98 * base:
                if bth != 1024:
                    out["fold_threads"][str(cls)] = int(bth)
                if blm:
                    out["lockstep_min"][str(cls)] = int(blm)
                if bp:
                    out["fold_pair"][str(cls)] = 1
            log(f"nb {nb} (class {cls}): form/threads/lockstep " +
                ", ".join(f"{'pair ' if p else ''}{th}/{lm or 'rule'}: {v:.3f}" for (p, th, lm), v in shapes.items())
                + f" -> {'pair ' if bp else ''}{bth}/{blm or 'rule'}")
        tuned = {"fold_group_max": out["fold_group_max"], "fold_threads": out["fold_threads"],
                 "lockstep_min": out["lockstep_min"], "fold_pair": out["fold_pair"]}
        launches = {}
        for lp in LAUNCHES:
            apply({**tuned, "launch_periods": lp})
            gpu.signal_search(st, cfg, dev=dev)
            ms = []
            for _ in range(reps):
                gpu.timer_start()
                gpu.signal_search(st, cfg, dev=dev)
                ms.append(gpu.timer_stop())
            launches[lp] = _median(ms)
            log(f"launch {lp}: {launches[lp]:.2f} ms per signal_search")
        best = min(launches, key=launches.get)
        out["signal_search_ms"] = {str(k): round(v, 3) for k, v in launches.items()}
        out["launch_periods"] = int(best) if launches[best] < 0.99 * launches[16384] else 0
        # The tile scan fused into the fold's CTAs against the separate scan
        # and merge kernels over prefix rows in device memory.
        sep = {}
        for flag in (0, 1):
            apply({**tuned, "launch_periods": out["launch_periods"], "fused_scan": flag})
            gpu.signal_search(st, cfg, dev=dev)
            ms = []
            for _ in range(reps):
                gpu.timer_start()
                gpu.signal_search(st, cfg, dev=dev)
                ms.append(gpu.timer_stop())
            sep[flag] = _median(ms)
            log(f"fused_scan {flag}: {sep[flag]:.2f} ms per signal_search")
        out["fused_scan_ms"] = {str(k): round(v, 3) for k, v in sep.items()}
        out["fused_scan"] = 1 if sep[1] < 0.99 * sep[0] else 0
        tuned["fused_scan"] = out["fused_scan"]

        # The per-class choices together, on the whole search: kept only
        # where they beat the built-in shapes end to end.
        def search_ms(table):
            apply(table)
            gpu.signal_search(st, cfg, dev=dev)
            ms = []
            for _ in range(reps):
                gpu.timer_start()
                gpu.signal_search(st, cfg, dev=dev)
                ms.append(gpu.timer_stop())
            return _median(ms)

        rest = {"launch_periods": out["launch_periods"], "fused_scan": out["fused_scan"]}
        variants = {"built-in shapes": {}, "tuned groups": {"fold_group_max": out["fold_group_max"]},
                    "tuned groups and lockstep": {"fold_group_max": out["fold_group_max"],
                                                  "lockstep_min": out["lockstep_min"]},
                    "tuned groups, lockstep and CTA sizes": {k: tuned[k] for k in
                                                             ("fold_group_max", "fold_threads", "lockstep_min")},
                    "tuned groups, lockstep, CTA sizes and paired walks": {
                        k: tuned[k] for k in ("fold_group_max", "fold_threads", "lockstep_min", "fold_pair")}}
        whole = {name: search_ms({**v, **rest}) for name, v in variants.items()}
        for name, v in whole.items():
            log(f"signal_search with {name}: {v:.2f} ms")
        pick = min(whole, key=whole.get)
        out["whole_search_ms"] = {k: round(v, 3) for k, v in whole.items()}
        for k in ("fold_group_max", "fold_threads", "lockstep_min", "fold_pair"):
            out[k] = variants[pick].get(k, {})
            tuned[k] = out[k]
        dev.free()
        # The batch's fold jobs: a CTA per unit against the persistent
        # work-stealing grid, on seeded survey stars searched together.
        rng = np.random.default_rng(77)
        stars = []
        for _ in range(survey_stars):
            cs = synth.survey_star(rng)
            cc = synth.survey_config(cs)
            stars.append((api.prepared_family(cs.time, cs.flux, cs.flux_err, cc), cc.period_max))
        devs = [gpu.upload(s_) for s_, _ in stars]
        steal = {}
        for flag in (0, 1):
            apply({**tuned, "launch_periods": out["launch_periods"], "fold_steal": flag})
            gpu.search_batch([s_ for s_, _ in stars], cfg, period_max=[p for _, p in stars], devs=devs, workers=0)
            ts = []
            for _ in range(reps):
                t0 = time.perf_counter()
                gpu.search_batch([s_ for s_, _ in stars], cfg, period_max=[p for _, p in stars], devs=devs,
                                 workers=0)
                ts.append(time.perf_counter() - t0)
            steal[flag] = _median(ts)
            log(f"survey of {survey_stars} stars, fold_steal {flag}: {1e3 * steal[flag]:.1f} ms")
        out["survey_ms"] = {"stars": survey_stars, **{str(k): round(1e3 * v, 2) for k, v in steal.items()}}
        out["fold_steal"] = 1 if steal[1] < 0.99 * steal[0] else 0
        # Whole period groups in the batch's job launches (no per-pass cut
        # to fill the SMs) on the same stars.
        whole = {0: steal[out["fold_steal"]]}
        apply({**tuned, "launch_periods": out["launch_periods"], "fold_steal": out["fold_steal"],
               "batch_no_fill": 1})
        gpu.search_batch([s_ for s_, _ in stars], cfg, period_max=[p for _, p in stars], devs=devs, workers=0)
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            gpu.search_batch([s_ for s_, _ in stars], cfg, period_max=[p for _, p in stars], devs=devs, workers=0)
            ts.append(time.perf_counter() - t0)
        whole[1] = _median(ts)
        log(f"survey of {survey_stars} stars, batch_no_fill 1: {1e3 * whole[1]:.1f} ms")
        out["survey_whole_groups_ms"] = {str(k): round(1e3 * v, 2) for k, v in whole.items()}
        out["batch_no_fill"] = 1 if whole[1] < 0.99 * whole[0] else 0
        # The coarse maps' folds (the proposal network's input, binned
        # families) by lockstep threshold, on the same stars.
        from . import proposal as pr
        pstars = [(s_, p) for s_, p in stars]
        saved = np.load(pr.WEIGHTS)
        bin_days = float(saved["bin_days"])
        oversample = float(saved["map_oversample"]) if "map_oversample" in saved.files else 2.0
        def time_maps(knobs):
            apply({**tuned, "launch_periods": out["launch_periods"], "fold_steal": out["fold_steal"],
                   "batch_no_fill": out["batch_no_fill"], **knobs})
            pr.features(gpu, pstars, devs, bin_days, oversample=oversample)
            ts = []
            for _ in range(reps):
                t0 = time.perf_counter()
                pr.features(gpu, pstars, devs, bin_days, oversample=oversample)
                ts.append(time.perf_counter() - t0)
            return _median(ts)

        # Shapes first (group cap x CTA size: fewer lanes per period, longer
        # segments), then the lockstep threshold at the best shape.
        shapes = {}
        for gm, th in MAP_SHAPES:
            shapes[(gm, th)] = time_maps({"map_group_max": gm, "map_threads": th})
            log(f"coarse maps of {survey_stars} stars, group cap {gm or 'rule'}, {th or 1024} threads: "
                f"{1e3 * shapes[(gm, th)]:.1f} ms")
        gm, th = min(shapes, key=shapes.get)
        if shapes[(gm, th)] >= 0.98 * shapes[(0, 0)]:
            gm, th = 0, 0
        out["map_shape_ms"] = {f"{g_ or 'rule'}x{t_ or 1024}": round(1e3 * v, 2) for (g_, t_), v in shapes.items()}
        out["map_group_max"], out["map_threads"] = int(gm), int(th)
        maps = {}
        for lm in MAP_LOCKSTEP:
            maps[lm] = time_maps({"map_group_max": gm, "map_threads": th, "map_lockstep_min": lm})
            log(f"coarse maps of {survey_stars} stars, map lockstep {lm or 'rule'}: {1e3 * maps[lm]:.1f} ms")
        best = min(maps, key=maps.get)
        out["maps_ms"] = {str(k): round(1e3 * v, 2) for k, v in maps.items()}
        out["map_lockstep_min"] = int(best) if maps[best] < 0.98 * maps[0] else 0
        for d in devs:
            d.free()
    reset()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--out", default=str(TABLE))
    ap.add_argument("--reps", type=int, default=5)
    args = ap.parse_args(argv)
    t0 = time.time()
    table = sweep(args.reps, log=lambda m: print(f"[{time.time() - t0:6.1f} s] {m}", flush=True))
    Path(args.out).write_text(json.dumps(table, indent=1) + "\n")
    print(json.dumps({k: table[k] for k in ("fold_group_max", "fold_threads", "lockstep_min", "fold_pair",
                                             "launch_periods",
                                             "fused_scan", "fold_steal", "map_lockstep_min", "map_threads",
                                             "map_group_max", "batch_no_fill")}))


if __name__ == "__main__":
    main()
