#!/usr/bin/env python
"""Benchmark of the FBLS search hot path on B200: BLS trials/s and stars/s.

A step is one signal_search (every octave band: coarse prescan over all
periods, full scan on the survivors) of one synthetic star:

  multi_sector (default): 13 sectors x 27.4 d at 120 s with a 1 d gap each
      (247,104 points), white 8e-4 + AR(1) red noise, one 400 ppm box at
      17.3 d; 20 durations 0.5-15 h, periods 0.5-20 d at period_oversample 3
      (189,216 periods under the reference's grid rule).
  single_sector: one sector (19,008 points), 12 durations, 13,065 periods.
  survey: a step is one fbls_search_batch over --stars seeded survey stars
      (1-13 sectors, 120/200/600 s cadence, 30 % with a box), the stars'
      band scans fused into job launches (--batch-workers 0) or spread over
      host worker threads with their own streams; timed by the host clock
      around the device-synchronised batch.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--workload survey]

Trials are templates as the reference counts them (P x nd x ns x nb per
scanned batch, scan.rs:352). `value` is whole-job trials/s with the star's
fields resident in HBM; `e2e` repeats the step through the C ABI with host
buffers (upload, scan, download inside the timed region). With N > 1 every
rank runs its own star (replicas, no collective on the data path); time is
the max over ranks.

--impl reference times the reference algorithm on the host cores. The
reference (Rust + cuda-oxide) cannot be built here, so its CPU restatement
(oracle/) runs instead, on a bounded sample of the same workload's periods.
"""
from __future__ import annotations

import argparse
import gc
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "stars/s & BLS trials/s on 1 B200; proposal vs exhaustive at 99% top-1 recall"
UNIT = "BLS trials/s"


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _bf16_peak():
    """Dense bf16 tensor peak (TFLOP/s): the burst figure of MEASURED_PEAKS.json,
    else this pool's earlier measurement."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        if "bf16_tflops" in d:
            return float(d["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def _network_flops(curves: int) -> int:
    """Forward FLOPs of the proposal network over `curves` coarse maps: the
    convolutions' GEMMs, 2 x CH x (ci x KW) x T per layer (bias, ReLU, pooling
    and the head are not counted)."""
    from fbls_b200 import proposal as pr
    flops, t, ci = 0, pr.T_IN, pr.MAP_CHANNELS
    for pool in pr.POOLS:
        flops += 2 * pr.CH * ci * pr.KW * t
        t //= pool
        ci = pr.CH
    return flops * curves


def _l2_copy_peak(device: str, copies: int = 32, reps: int = 10):
    """The copy rate (read + write bytes per second, GB/s) of a buffer pair
    that stays in L2, measured here: the same STREAM-style copy as the HBM
    peak at sizes of 4-24 MiB (8-48 MiB of L2), 32 copies per CUDA graph
    replay so that launch gaps do not count; the best size is kept."""
    import torch
    best, best_mib = 0.0, 0
    for mib in (4, 8, 12, 16, 24):
        a = torch.ones(mib * 1024 * 1024 // 4, dtype=torch.float32, device=device)
        b = torch.empty_like(a)
        side = torch.cuda.Stream(device)
        side.wait_stream(torch.cuda.current_stream(device))
        with torch.cuda.stream(side):
            for _ in range(3):
                b.copy_(a)
        torch.cuda.current_stream(device).wait_stream(side)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            for _ in range(copies):
                b.copy_(a)
        for _ in range(2):
            graph.replay()
        torch.cuda.synchronize(device)
        ms = float("inf")
        for _ in range(reps):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            graph.replay()
            e.record()
            e.synchronize()
            ms = min(ms, s.elapsed_time(e))
        rate = 2.0 * a.numel() * 4 * copies / (ms * 1e-3) / 1e9
        if rate > best:
            best, best_mib = rate, mib
        del graph, a, b
    return best, best_mib


def _workload(name, period_oversample=None):
    """(curve, config, description) of a single-star workload; a
    `period_oversample` other than the configuration's 3 gives the denser-grid
    variants (6.9 on single_sector: ~30k periods; 19 on multi_sector: ~1.2M)."""
    from fbls_b200 import synth
    if name == "single_sector":
        c, cfg = synth.single_sector(), synth.single_sector_config()
        desc = ("single_sector: 1 x 27.4 d sector at 120 s with a 1 d gap (19,008 points), 12 durations 0.5-12 h, "
                "periods 0.5-13.7 d at period_oversample {os:g}")
    else:
        c, cfg = synth.multi_sector(), synth.multi_sector_config()
        desc = ("multi_sector: 13 x 27.4 d sectors at 120 s with a 1 d gap each (247,104 points), white 8e-4 + AR(1) "
                "(0.95, 3e-4), 400 ppm box at 17.3 d; 20 durations 0.5-15 h, periods 0.5-20 d at "
                "period_oversample {os:g}")
    if period_oversample is not None:
        cfg.period_oversample = float(period_oversample)
    return c, cfg, desc.format(os=cfg.period_oversample)


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                smax.append(float(parts[2].split()[0]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _barrier(world: int) -> None:
    """Every rank meets here (no-op on one rank)."""
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _over_ranks(maxes, sums, world: int, device: str = "cpu"):
    """(max over ranks of each of `maxes`, sum over ranks of each of `sums`):
    step times take the slowest rank, work adds up (the whole job's
    throughput); identity on one rank. Every rank calls it, in the same order."""
    maxes, sums = [float(x) for x in maxes], [float(x) for x in sums]
    if world <= 1:
        return maxes, sums
    import torch
    import torch.distributed as dist
    t = torch.tensor(maxes + sums, dtype=torch.float64, device=device)
    mx, sm = t[:len(maxes)].clone(), t[len(maxes):].clone()
    if len(maxes):
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    if len(sums):
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return mx.tolist(), sm.tolist()


def _oracle_sample(state, cfg, every: int, threads: int):
    """The reference algorithm on every `every`-th period of each band: (trials, seconds)."""
    import oracle
    _, bands = oracle.band_plan(state, cfg)
    trials = 0
    t0 = time.perf_counter()
    for sel, d, r in bands:
        rows, st = oracle.scan_periods(state, sel[::every], d, r, cfg, threads=threads)
        trials += st["templates_scanned"]
    return trials, time.perf_counter() - t0


def _cpu_sample(curve, cfg, target_seconds: float):
    """Calibrated oracle sample taking about target_seconds on all host cores."""
    import oracle
    st = oracle.family_state(curve.time, curve.flux, curve.flux_err, cfg.durations_days())
    threads = os.cpu_count() or 1
    every = 4096
    trials, sec = _oracle_sample(st, cfg, every, threads)
    while sec < 0.25 * target_seconds and every > 1:
        every = max(1, int(every * max(sec, 1e-3) / target_seconds))
        trials, sec = _oracle_sample(st, cfg, every, threads)
    return st, every, threads, trials, sec


def _workload_config(state, cfg, desc: str, world: int) -> dict:
    """The `config` of a single-star workload's line, the same for both arms."""
    from fbls_b200 import api
    grid, bands = api.band_plan(state, cfg)
    return {"workload": desc, "stars": world, "periods": int(len(grid)), "bands": len(bands),
            "observations": state.n, "period_oversample": cfg.period_oversample,
            "l2": "flushed between steps (256 MiB write)",
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"}


def run_reference(args):
    world, rank, local = _dist()
    if rank != 0:
        return
    from fbls_b200 import api
    curve, cfg, desc = _workload(args.workload, args.period_oversample)
    state = api.prepared_family(curve.time, curve.flux, curve.flux_err, cfg)
    st, every, threads, trials, sec = _cpu_sample(curve, cfg, args.cpu_seconds)
    for _ in range(args.warmup):
        _oracle_sample(st, cfg, every, threads)
    times, tr = [], 0
    for _ in range(args.steps):
        t, s = _oracle_sample(st, cfg, every, threads)
        times.append(s)
        tr = t
    total = sum(times)
    value = tr * args.steps / total
    sample = f"every {every}th period of each band (coarse prescan + full scan of survivors), {tr} trials per step"
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": _workload_config(state, cfg, desc, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference (Rust + cuda-oxide) not buildable offline; its CPU restatement (oracle/) is timed",
    }
    print(json.dumps(out))


def run_gpu(args):
    import torch
    world, rank, local = _dist()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    from fbls_b200 import api

    curve, cfg, desc = _workload(args.workload, args.period_oversample)
    state = api.prepared_family(curve.time, curve.flux, curve.flux_err, cfg)
    gpu = api.Gpu(local)
    dev = gpu.upload(state)
    grid, bands = api.band_plan(state, cfg)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")

    def step():
        return gpu.signal_search(state, cfg, dev=dev)

    for _ in range(args.warmup):
        rows, glen, stats = step()
    torch.cuda.synchronize()
    gpu.counters(reset=True)
    gpu.set_kernel_timing(True)
    clocks = Clocks(local)
    if world > 1:
        torch.distributed.barrier()
    clocks.start()
    times = []
    trials = 0
    gc.collect()
    gc.disable()  # no collector pauses inside the timed steps
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        gpu.timer_start()
        rows, glen, stats = step()
        times.append(gpu.timer_stop())
        trials += sum(s["templates_scanned"] for s in stats)
    torch.cuda.synchronize()
    _barrier(world)
    clk = clocks.stop()
    gpu.set_kernel_timing(False)
    ctr = gpu.counters(reset=True)
    (total_ms,), (trials,) = _over_ranks([sum(times)], [trials], world, f"cuda:{local}")
    value = trials / (total_ms * 1e-3)

    # End to end through the C ABI with host buffers: fbls_search_batch with
    # the star's prepared family in (pinned) host memory, which the library
    # uploads into the context's reusable family buffer; scan; rows back.
    pinned = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (state.time, state.v, state.w)]

    def e2e_step():
        sub = api.FamilyState(pinned[0].numpy(), pinned[1].numpy(), pinned[2].numpy(), state.baseline_norm,
                              state.origin, state.residual_energy, state.durations, state.rho)
        return gpu.search_batch([sub], cfg, workers=0)[0]

    for _ in range(args.warmup):  # the batch path's workspaces grow on its first call
        e2e_step()
    torch.cuda.synchronize()
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        gpu.timer_start()
        rows_e, glen_e, _ = e2e_step()
        e2e_ms.append(gpu.timer_stop())
    gc.enable()
    torch.cuda.synchronize()
    _barrier(world)
    (e2e_total,), _ = _over_ranks([sum(e2e_ms)], [], world, f"cuda:{local}")
    e2e_value = trials / (e2e_total * 1e-3)
    h2d = 3 * 8 * state.n
    d2h = sum((s["periods"] + s["prescan_survivors"]) * (9 * 8 + 8 + 8 + 4) for s in stats) + 40 * len(rows_e)

    peak, peak_kind = _peaks()
    from fbls_b200 import autotune
    fused = bool(autotune.current().get("fused_scan", 0))
    kernel = ("k_fold_scan (fold + prefix + tile scan + merge, fused)" if fused else "k_fold_walk (fold + prefix)")
    fold_launches = max(ctr["fold_launches"], 1)
    fold_ms_per = ctr["fold_ms"] / fold_launches
    fold_bytes_per = ctr["fold_bytes"] / fold_launches
    achieved = fold_bytes_per / (fold_ms_per * 1e-3) / 1e9 if fold_ms_per > 0 else 0.0
    # DRAM bytes per fold launch: one committed ncu capture of a smaller
    # launch of this kernel (measured once, not in this run) scaled to this
    # run's mean launch by what grows with it: the prefix rows written and
    # the periods folded.
    traffic = None
    prof = ROOT / "profiles" / "fold_traffic.json"
    if prof.exists() and not fused:
        try:
            rates = json.loads(prof.read_text())
            rows_per_launch = (ctr["fold_bytes"] - 24.0 * ctr["fold_updates"]) / fold_launches
            periods_per_launch = ctr["fold_updates"] / state.n / fold_launches
            traffic = int(rates["write_per_row_byte"] * rows_per_launch + rates["read_per_period"] * periods_per_launch)
        except (OSError, ValueError, KeyError):
            traffic = None

    if rank != 0:
        return
    l2_peak, l2_mib = _l2_copy_peak(f"cuda:{local}")
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": _workload_config(state, cfg, desc, world),
        "stars_per_s": world * args.steps / (total_ms * 1e-3),
        "step_ms": [round(t, 2) for t in times],
        "trials_per_step": trials / args.steps / world,
        "box_trials_per_s": value / len(cfg.ingress_fractions),
        "rows_per_step": int(len(rows)),
        "gpu_launches": int(ctr["launches"]),
        "kernel_ms": ({"fold_scan_merge": ctr["fold_ms"] / args.steps} if fused else
                      {"fold_prefix": ctr["fold_ms"] / args.steps, "scan_tiles+merge": ctr["scan_ms"] / args.steps}),
        "roofline": {"kernel": kernel, "bound": "hbm", "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "algorithmic_bytes_per_launch": fold_bytes_per, "launch_ms": fold_ms_per,
                     "l2": {"peak": l2_peak, "frac": achieved / l2_peak if l2_peak > 0 else None,
                            "peak_kind": f"measured here: copy of a {l2_mib} MiB buffer pair that stays in L2"},
                     "traffic_source": "one ncu capture of an nb-1536 launch scaled to this run's mean launch "
                                       "(profiles/fold_traffic.json)",
                     "limiter": {"pipe": "shared memory and issue", "wavefronts_frac_of_peak": 0.639,
                                 "wavefronts_per_update": 0.61, "issue_active_frac": 0.697,
                                 "dram_frac_of_peak": 0.021,
                                 "source": "ncu --set full of one nb-1536 launch of this workload "
                                           "(profiles/k_fold_walk_multi_sector.md)"},
                     "note": "algorithmic bytes count the observation stream once per period (24 n B); it is "
                             "served from L2 and shared memory, and the kernel is bound by the shared-memory "
                             "pipe (64 % of its wavefront peak) and instruction issue (70 %) in an ncu capture; "
                             "2 % of DRAM peak"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(d2h),
                "ms_per_step": e2e_total / args.steps, "step_ms": [round(t, 2) for t in e2e_ms],
                "rows_equal_resident": bool(np.array_equal(rows_e, rows))},
        "clocks": clk,
    }
    if world == 1 and not args.no_cpu:
        st, every, threads, tr, sec = _cpu_sample(curve, cfg, args.cpu_seconds)
        out["cpu_baseline"] = {"value": tr / sec, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"every {every}th period of each band, {tr} trials, {sec:.1f} s"}
    dev.free()
    if world == 1 and args.extras_stars > 0:
        out.update(_metric_second_half(gpu, args.extras_stars))
    print(json.dumps(out))
    gpu.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def _metric_second_half(gpu, count: int) -> dict:
    """The metric's other parts on `count` seeded survey stars (held out from
    the proposal network's training seeds): the batched exhaustive search's
    stars/s (resident families, and end to end with host families), and the
    proposal-pruned search against it (stars/s, speed-up, top-1 recall: the
    pruned search's best row is the exhaustive best row). Host clock around
    each device-synchronised batch; one warm-up, two timed steps each."""
    import torch
    from fbls_b200 import proposal as pr
    stars, cfg = _survey(count, 1000)
    pstars = [(s, p) for _, s, p in stars]
    states, pmax = [s for s, _ in pstars], [p for _, p in pstars]
    devs = [gpu.upload(s) for s in states]
    net = pr.load_net(0)

    def timed(fn, steps=2):
        fn()
        out, ts = None, []
        for _ in range(steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = fn()
            ts.append(time.perf_counter() - t0)
        return out, sum(ts) / len(ts), ts

    full, t_ex, ts_ex = timed(lambda: gpu.search_batch(states, cfg, period_max=pmax, devs=devs, workers=0))
    _, t_e2e, _ = timed(lambda: gpu.search_batch(states, cfg, period_max=pmax, workers=0), steps=1)
    def recall(pruned):
        hits = labelled = 0
        for (fr, _, _), (pr_rows, _, _) in zip(full, pruned):
            if fr.shape[0] == 0:
                continue
            labelled += 1
            best = fr[int(np.argmax(fr[:, 3]))]
            hits += int(pr_rows.shape[0] > 0 and np.array_equal(pr_rows[int(np.argmax(pr_rows[:, 3]))], best))
        return hits, labelled

    # At 99 % top-1 recall: the fewest bands whose held-out band recall
    # reaches the operating point's (proposal.OPERATING_RECALL); and at
    # cfg4's 32 bands.
    k99 = pr.bands_for_recall(pr.OPERATING_RECALL)
    rec_table = np.load(pr.WEIGHTS)["recall"]
    (pruned, _), t_pr, ts_pr = timed(lambda: pr.search_proposed(gpu, net, pstars, devs, cfg, k=k99, workers=0))
    hits, labelled = recall(pruned)
    (pruned32, _), t_32, ts_32 = timed(lambda: pr.search_proposed(gpu, net, pstars, devs, cfg, k=pr.TOP_BANDS,
                                                                  workers=0))
    hits32, _ = recall(pruned32)
    trials = sum(t for _, _, t in full)
    for d in devs:
        d.free()
    desc = (f"{count} seeded survey stars (1-13 sectors ~ Geometric(0.4), cadence 120/200/600 s, white + AR(1) "
            "noise, 30 % with a box), 20 durations 0.5-15 h, periods 0.5-min(20, baseline/2) d")
    return {
        "survey": {"stars": count, "workload": desc, "stars_per_s": count / t_ex, "trials_per_s": trials / t_ex,
                   "step_ms": [round(1e3 * t, 1) for t in ts_ex],
                   "e2e_stars_per_s": count / t_e2e, "e2e_h2d_bytes": 24 * sum(s.n for s in states),
                   "timing": "host clock around the device-synchronised fbls_search_batch (stars fused)"},
        "proposal": {"stars": count, "exhaustive_stars_per_s": count / t_ex, "proposal_stars_per_s": count / t_pr,
                     "speedup": t_ex / t_pr, "top1_recall": hits / max(labelled, 1),
                     "stars_with_detection": labelled, "bands_searched": k99, "bands": pr.BANDS,
                     "heldout_band_recall": float(rec_table[k99 - 1]),
                     "bands_rule": f"the fewest bands whose held-out band recall (the training run's labelled "
                                   f"held-out stars) reaches {pr.OPERATING_RECALL}",
                     "step_ms": [round(1e3 * t, 1) for t in ts_pr],
                     "top32": {"bands_searched": pr.TOP_BANDS, "proposal_stars_per_s": count / t_32,
                               "speedup": t_ex / t_32, "top1_recall": hits32 / max(labelled, 1),
                               "heldout_band_recall": float(rec_table[pr.TOP_BANDS - 1])},
                     "timing": "host clock around coarse maps + network + pruned fbls_search_batch"},
    }


def _survey(count: int, seed: int):
    """`count` seeded survey stars (1-13 sectors, 120/200/600 s cadence, 30 %
    with an injected box), prepared: [(FamilyState, period_max)], base config."""
    from fbls_b200 import api, synth
    rng = np.random.default_rng(seed)
    stars = []
    for _ in range(count):
        c = synth.survey_star(rng)
        cfg = synth.survey_config(c)
        stars.append((c, api.prepared_family(c.time, c.flux, c.flux_err, cfg), cfg.period_max))
    return stars, synth.survey_config(stars[0][0])


def run_survey(args):
    """A step is one fbls_search_batch over a survey of args.stars stars."""
    import torch
    world, rank, local = _dist()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    from fbls_b200 import api

    stars, cfg = _survey(args.stars, 1000 + rank)
    states = [s for _, s, _ in stars]
    pmax = [p for _, _, p in stars]
    n_obs = sum(s.n for s in states)
    gpu = api.Gpu(local)
    devs = [gpu.upload(s) for s in states]
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")

    def step(resident=True):
        return gpu.search_batch(states, cfg, period_max=pmax, devs=devs if resident else None,
                                workers=args.batch_workers)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    gpu.counters(reset=True)
    clocks = Clocks(local)
    if world > 1:
        torch.distributed.barrier()
    clocks.start()
    gc.collect()
    gc.disable()
    times, trials = [], 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = step()
        times.append((time.perf_counter() - t0) * 1e3)
        trials += sum(t for _, _, t in out)
    torch.cuda.synchronize()
    _barrier(world)
    clk = clocks.stop()
    ctr = gpu.counters(reset=True)
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out_e = step(resident=False)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    gc.enable()
    torch.cuda.synchronize()
    _barrier(world)
    (total_ms, e2e_total), (trials,) = _over_ranks([sum(times), sum(e2e_ms)], [trials], world, f"cuda:{local}")
    if rank != 0:
        return
    value = trials / (total_ms * 1e-3)
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"survey: {args.stars} seeded stars per GPU (1-13 sectors ~ Geometric(0.4), "
                               "cadence 120/200/600 s, white + AR(1) 0.9 noise, 30 % with a box), 20 durations "
                               "0.5-15 h, periods 0.5-min(20, baseline/2) d",
                   "stars": args.stars * world, "observations": n_obs, "batch_workers": args.batch_workers,
                   "l2": "flushed between steps (256 MiB write)",
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
        "stars_per_s": args.stars * world * args.steps / (total_ms * 1e-3),
        "step_ms": [round(t, 2) for t in times],
        "gpu_launches": int(ctr["launches"]),
        "e2e": {"value": trials / (e2e_total * 1e-3), "unit": UNIT,
                "h2d_bytes_per_step": 24 * n_obs,
                "d2h_bytes_per_step": sum(92 * g + 40 * len(r) for r, g, _ in out_e),
                "ms_per_step": e2e_total / args.steps,
                "stars_per_s": args.stars * world * args.steps / (e2e_total * 1e-3)},
        "clocks": clk,
    }
    if world == 1 and not args.no_cpu:
        st, every, threads, tr, sec = _cpu_sample(stars[0][0], cfg, args.cpu_seconds)
        out["cpu_baseline"] = {"value": tr / sec, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"first survey star, every {every}th period of each band, {tr} trials, "
                                         f"{sec:.1f} s"}
    print(json.dumps(out))
    for d in devs:
        d.free()
    gpu.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def _kernel_table(path, steps):
    """One run of each step under torch.profiler (CUDA activity only):
    the step's host-clock time and the device time of every kernel and copy,
    written as text tables."""
    import torch
    from torch.profiler import ProfilerActivity, profile
    out = []
    for name, fn in steps.items():
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
        out.append(f"## {name} ({1e3 * wall:.1f} ms host clock, under the profiler)\n\n" +
                   prof.key_averages().table(sort_by="cuda_time_total", row_limit=16, max_name_column_width=48))
    Path(path).write_text("\n\n".join(out) + "\n")


def run_proposal(args):
    """Proposal-pruned search against the exhaustive search on the survey
    workload: both timed on the same resident stars (host clock around the
    device-synchronised batches), the top-1 recall of the pruned search (its
    best row is the exhaustive best row), and the stars/s ratio."""
    import torch
    from fbls_b200 import api
    from fbls_b200 import proposal as pr
    torch.cuda.set_device(0)
    if args.bands is None:
        args.bands = pr.bands_for_recall(pr.OPERATING_RECALL)
    stars, cfg = _survey(args.stars, 1000)
    pstars = [(s, p) for _, s, p in stars]
    gpu = api.Gpu(0)
    devs = [gpu.upload(s) for s, _ in pstars]
    net = pr.load_net(0)
    states, pmax = [s for s, _ in pstars], [p for _, p in pstars]

    def exhaustive():
        return gpu.search_batch(states, cfg, period_max=pmax, devs=devs, workers=args.batch_workers)

    def proposed():
        return pr.search_proposed(gpu, net, pstars, devs, cfg, k=args.bands, workers=args.batch_workers)

    for _ in range(args.warmup):
        exhaustive()
        proposed()
    gc.collect()
    gc.disable()
    t_ex, t_pr = [], []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        full = exhaustive()
        t_ex.append(time.perf_counter() - t0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pruned, logits = proposed()
        t_pr.append(time.perf_counter() - t0)
        parts = dict(pr.search_proposed.last_ms)
    gc.enable()
    if args.kernel_table:
        # the proposal step whole, then its coarse maps and its pruned search
        # (the last step's bands) apart
        ranges = [pr.ranges_for(l, args.bands) for l in logits]
        _kernel_table(args.kernel_table, {
            "exhaustive batch": exhaustive, "proposal step": proposed,
            "coarse maps": lambda: pr.features(gpu, pstars, devs, net.bin_days, device=True,
                                               oversample=net.map_oversample),
            "pruned search": lambda: gpu.search_batch(states, cfg, period_max=pmax, devs=devs,
                                                      workers=args.batch_workers, ranges=ranges)})
    hits = labelled = 0
    for (fr, _, _), (pr_rows, _, _) in zip(full, pruned):
        if fr.shape[0] == 0:
            continue
        labelled += 1
        best = fr[int(np.argmax(fr[:, 3]))]
        if pr_rows.shape[0] and np.array_equal(pr_rows[int(np.argmax(pr_rows[:, 3]))], best):
            hits += 1
    tex, tpr = sum(t_ex) / len(t_ex), sum(t_pr) / len(t_pr)
    rec = np.load(pr.WEIGHTS)
    out = {
        "metric": METRIC, "value": args.stars / tpr, "unit": "stars/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * tpr, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 search, bf16 network", "data": "synthetic",
        "config": {"workload": f"proposal: {args.stars} seeded survey stars (as --workload survey), the "
                               f"exhaustive search of the {args.bands} best of {pr.BANDS} log-period bands",
                   "batch_workers": args.batch_workers, "bands_searched": args.bands},
        "exhaustive_stars_per_s": args.stars / tex,
        "proposal_stars_per_s": args.stars / tpr,
        "speedup": tex / tpr,
        "top1_recall": hits / max(labelled, 1), "stars_with_detection": labelled,
        "network_heldout_recall_at_k": float(rec["recall"][args.bands - 1]),
        "step_ms": {"exhaustive": [round(1e3 * t, 1) for t in t_ex], "proposal": [round(1e3 * t, 1) for t in t_pr]},
        "proposal_ms_last_step": {k: round(v, 1) for k, v in parts.items()},
    }
    tpeak, tkind = _bf16_peak()
    net_s = parts.get("network", 0.0) * 1e-3
    if net_s > 0:
        achieved = _network_flops(args.stars) / net_s / 1e12
        out["network_roofline"] = {
            "kernel": "k_gemm_bf16 (the network's convolutions, forward)", "bound": "tensor",
            "achieved": achieved, "peak": tpeak, "peak_kind": tkind, "unit": "TFLOP/s", "frac": achieved / tpeak,
            "flops_per_curve": _network_flops(1),
            "note": "host clock around the band scores of the last step (feature upload, forward, logits download)"}
    print(json.dumps(out))
    for d in devs:
        d.free()
    gpu.close()


def _full_chunk(seed: int, start: int, count: int):
    """Stars [start, start + count) of the survey-scale batch (one seeded
    stream per star): prepared families and what was injected."""
    from fbls_b200 import api, synth
    out = []
    for i in range(start, start + count):
        c = synth.survey_star_full(np.random.default_rng([seed, i]))
        cfg = synth.survey_config(c)
        st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
        out.append((st, cfg.period_max, c.label, c.period))
    return out


def run_full(args):
    """Survey-scale full form: --stars seeded stars (8 % boxes, 2 %
    eclipsing-binary-like pairs); a step is the proposal-pruned search of all
    of them followed by the evidence comparison (null, box, box plus
    secondary) of each star's best candidate, in batches. Also timed once:
    the exhaustive batched search, the reference for top-1 recall. Host clock
    around device-synchronised calls."""
    import concurrent.futures as cf
    import multiprocessing as mp
    import torch
    chunk = 250
    with cf.ProcessPoolExecutor(max_workers=min(16, os.cpu_count() or 1), mp_context=mp.get_context("spawn")) as ex:
        parts = list(ex.map(_full_chunk, [2000] * ((args.stars + chunk - 1) // chunk),
                            range(0, args.stars, chunk), [min(chunk, args.stars - s) for s in range(0, args.stars, chunk)]))
    stars = [x for p in parts for x in p]
    from fbls_b200 import api, synth
    from fbls_b200 import proposal as pr
    torch.cuda.set_device(0)
    cfg = synth.survey_config(synth.survey_star(np.random.default_rng(0)))
    gpu = api.Gpu(0)
    states, pmax = [s for s, _, _, _ in stars], [p for _, p, _, _ in stars]
    devs = [gpu.upload(s) for s in states]
    net = pr.load_net(0)
    pstars = list(zip(states, pmax))
    k = args.bands if args.bands is not None else pr.bands_for_recall(pr.OPERATING_RECALL)

    def full_form():
        t0 = time.perf_counter()
        pruned, _ = pr.search_proposed(gpu, net, pstars, devs, cfg, k=k, workers=0)
        t1 = time.perf_counter()
        idx, cands, cdevs = [], [], []
        for i, (rows, _, _) in enumerate(pruned):
            if rows.shape[0]:
                idx.append(i)
                cands.append((states[i], float(rows[int(np.argmax(rows[:, 3])), 0])))
                cdevs.append(devs[i])
        ev = []
        for s in range(0, len(cands), 1024):
            ev += gpu.compare_batch(cands[s:s + 1024], cfg, devs=cdevs[s:s + 1024])
        t2 = time.perf_counter()
        return pruned, idx, ev, (t1 - t0, t2 - t1)

    # warm-up on a slice, then the timed full form
    sub = slice(0, min(256, len(states)))
    pr.search_proposed(gpu, net, pstars[sub], devs[sub], cfg, k=k, workers=0)
    gpu.compare_batch([(states[0], 1.0)], cfg, devs=[devs[0]])
    gpu.set_kernel_timing(True)
    gpu.counters(reset=True)
    clocks = Clocks(0)
    clocks.start()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pruned, idx, ev, (t_search, t_ev) = full_form()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    ctr = gpu.counters(reset=True)
    gpu.set_kernel_timing(False)
    parts_ms = dict(pr.search_proposed.last_ms)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    full = gpu.search_batch(states, cfg, period_max=pmax, devs=devs, workers=0)
    t_ex = time.perf_counter() - t0
    hits = labelled = 0
    pairs = pair_binary = 0
    evmap = dict(zip(idx, ev))
    for i, ((fr, _, _), (prr, _, _)) in enumerate(zip(full, pruned)):
        if fr.shape[0]:
            labelled += 1
            best = fr[int(np.argmax(fr[:, 3]))]
            hits += int(prr.shape[0] > 0 and np.array_equal(prr[int(np.argmax(prr[:, 3]))], best))
        if "pair" in stars[i][2] and i in evmap and evmap[i]:
            pairs += 1
            row = next((r for r in evmap[i] if r["selection_flags"] & 1), evmap[i][0])
            pair_binary += int(row["log_bf_binary_noise"] > row["log_bf_planet_noise"])
    peak, peak_kind = _peaks()
    tpeak, tkind = _bf16_peak()
    fold_launches = max(ctr["fold_launches"], 1)
    fold_ms = ctr["fold_ms"] / fold_launches
    hbm = ctr["fold_bytes"] / fold_launches / (fold_ms * 1e-3) / 1e9 if fold_ms > 0 else 0.0
    net_s = parts_ms.get("network", 0.0) * 1e-3
    tflops = _network_flops(len(states)) / net_s / 1e12 if net_s > 0 else 0.0
    n_obs = sum(s.n for s in states)
    out = {
        "metric": METRIC, "value": len(states) / wall, "unit": "stars/s", "n_gpus": 1, "steps": 1, "warmup": 1,
        "ms_per_step": 1e3 * wall, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 search and evidence, bf16 network", "data": "synthetic",
        "config": {"workload": f"full: {len(states)} seeded survey stars (1-13 sectors ~ Geometric(0.4), cadence "
                               "120/200/600 s, white + AR(1) noise; 8 % boxes, 2 % eclipsing-binary-like pairs "
                               f"with unequal depths 1-20 %); proposal ({k} of 1024 bands) -> pruned search -> "
                               "evidence of each star's best candidate",
                   "stars": len(states), "observations": n_obs, "bands_searched": k,
                   "boxes": sum("box" in x[2] for x in stars), "pairs": sum("pair" in x[2] for x in stars)},
        "seconds": {"proposal_and_pruned_search": t_search, "evidence": t_ev, **{k: v / 1e3 for k, v in parts_ms.items()}},
        "evidence_candidates": len(ev), "evidence_candidates_per_s": len(ev) / t_ev if t_ev > 0 else None,
        "exhaustive_stars_per_s": len(states) / t_ex, "speedup_vs_exhaustive_search": t_ex / wall,
        "top1_recall": hits / max(labelled, 1), "stars_with_detection": labelled,
        "pairs_with_evidence": pairs, "pairs_binary_preferred": pair_binary,
        "roofline": {"hbm": {"kernel": "fold + prefix", "achieved": hbm, "peak": peak, "peak_kind": peak_kind,
                             "unit": "GB/s", "frac": hbm / peak},
                     "tensor": {"kernel": "proposal network forward", "achieved": tflops, "peak": tpeak,
                                "peak_kind": tkind, "unit": "TFLOP/s", "frac": tflops / tpeak}},
        "gpu_launches": int(ctr["launches"]),
        "clocks": clk,
    }
    print(json.dumps(out))
    for d in devs:
        d.free()
    gpu.close()


def _rescore_bytes(time_rel, origin, rows, n_all):
    """Algorithmic bytes of one rescoring block: every observation the
    windowed kernels visit (t, v, w and the exclusion byte for the family;
    t and the byte for the merged times), two binary searches per transit
    window, and the rows in and results out."""
    period, epoch, duration = rows[:, 0], rows[:, 1], rows[:, 2]
    total = 0.0
    for t, c, per_visit in ((time_rel, epoch - origin, 25.0), (time_rel + origin, epoch, 9.0)):
        klo = np.floor((t[0] - c) / period) - 1.0
        khi = np.ceil((t[-1] - c) / period) + 1.0
        for r in range(rows.shape[0]):
            ks = c[r] + np.arange(klo[r], khi[r] + 1.0) * period[r]
            lo = np.searchsorted(t, ks - duration[r] / 2.0 - 1e-6, side="left")
            hi = np.searchsorted(t, ks + duration[r] / 2.0 + 1e-6, side="right")
            visits = int(np.maximum(hi - np.maximum(lo, np.concatenate([[0], np.maximum.accumulate(hi)[:-1]])), 0).sum())
            total += per_visit * visits + len(ks) * 2 * math.ceil(math.log2(t.shape[0] + 1)) * 8.0
    return total + rows.shape[0] * (2 * 24.0 + 24.0 + 8.0)


def run_rescore(args):
    """Peak-selection rescoring: a step is one refresh
    block of select_peaks on the 13-sector star, 8192 rows rescored, i.e.
    fbls_rescore_rows over the family outside the excluded set plus
    fbls_count_rows over the merged times, through the C ABI with host
    arrays. value: rows per second of kernel time (CUDA events on the
    context's stream); e2e: rows per second of the whole calls."""
    import torch
    import oracle
    from fbls_b200 import api, synth
    torch.cuda.set_device(0)
    c, cfg = synth.multi_sector(), synth.multi_sector_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    rng = np.random.default_rng(17)
    R = args.rows
    ta = st.time + st.origin
    period = np.exp(rng.uniform(math.log(0.5), math.log(20.0), R))
    rows = np.column_stack([period, ta[0] + rng.uniform(0.0, 1.0, R) * period, rng.choice(st.durations, R)])
    ex = (rng.uniform(size=st.n) < 0.05).astype(np.uint8)
    gpu = api.Gpu(0)
    dev = gpu.upload(st)

    def step():
        return gpu.rescore_rows(dev, ex, rows), gpu.count_rows(ta, ex, rows)

    for _ in range(args.warmup):
        step()
    gpu.set_kernel_timing(True)
    gpu.counters(reset=True)
    clocks = Clocks(0)
    clocks.start()
    times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sums, counts = step()
        times.append((time.perf_counter() - t0) * 1e3)
    clk = clocks.stop()
    ctr = gpu.counters(reset=True)
    kernel_ms = ctr["rescore_ms"] / args.steps
    wall_ms = sum(times) / args.steps
    algo = _rescore_bytes(st.time, st.origin, rows, ta.shape[0])
    peak, peak_kind = _peaks()
    out = {
        "metric": "rescored rows/s (peak selection, rescore_rows + count_rows)", "value": R / (kernel_ms * 1e-3),
        "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": kernel_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"rescore: {R} rows (period log-U[0.5, 20] d, the family's durations) of the "
                               "13-sector star (247,104 observations), 5 % excluded",
                   "rows": R, "observations": int(st.n),
                   "l2": "inputs (2.2 MB) stay in L2; the kernels visit only transit windows"},
        "step_ms": [round(t, 3) for t in times],
        "gpu_launches": int(ctr["rescore_launches"]),
        "e2e": {"value": R / (wall_ms * 1e-3), "unit": "rows/s", "ms_per_step": wall_ms,
                "h2d_bytes_per_step": 2 * R * 24 + 2 * st.n + 8 * st.n,
                "d2h_bytes_per_step": R * 24 + R * 8},
        "roofline": {"kernel": "k_rescore_rows + k_count_rows", "bound": "hbm", "achieved": algo / (kernel_ms * 1e-3) / 1e9,
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": algo / (kernel_ms * 1e-3) / 1e9 / peak, "traffic": None,
                     "algorithmic_bytes_per_step": algo,
                     "note": "bytes the windowed walk must touch; the kernels are latency-bound (binary searches, "
                             "one CTA per row), not bandwidth-bound"},
        "clocks": clk,
    }
    if not args.no_cpu:
        sample = 16
        t0 = time.perf_counter()
        oracle.rescore_rows(st.time, st.v, st.w, ex, rows[:sample], st.origin)
        oracle.count_rows(ta, ex, rows[:sample])
        sec = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": sample / sec, "unit": "rows/s", "cores": 1, "kind": "port",
                               "sample": f"the first {sample} rows through the oracle's full scan (the reference "
                                         f"kernels' loops, single thread), {sec:.2f} s"}
        assert np.array_equal(sums[:sample], oracle.rescore_rows(st.time, st.v, st.w, ex, rows[:sample], st.origin))
    print(json.dumps(out))
    dev.free()
    gpu.close()


def run_single_event(args):
    """Single-event scan: a step is one
    single_event_search of the 13-sector star (one trial period of 357 d, nb
    68,544, 20 durations x 3 shapes), through the C ABI with the family
    resident. value: templates per second of kernel time (fold + scan_all,
    CUDA events around the launches on the context's stream); e2e: of the
    whole call."""
    import torch
    import oracle
    from fbls_b200 import api, synth
    torch.cuda.set_device(0)
    c, cfg = synth.multi_sector(), synth.multi_sector_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    gpu = api.Gpu(0)
    dev = gpu.upload(st)
    for _ in range(args.warmup):
        rows, stats = gpu.single_event_search(st, cfg, dev=dev)
    gpu.set_kernel_timing(True)
    gpu.counters(reset=True)
    clocks = Clocks(0)
    clocks.start()
    times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rows, stats = gpu.single_event_search(st, cfg, dev=dev)
        times.append((time.perf_counter() - t0) * 1e3)
    clk = clocks.stop()
    ctr = gpu.counters(reset=True)
    tm = stats["templates_scanned"]
    ms = (ctr["fold_ms"] + ctr["scan_ms"]) / args.steps
    wall = sum(times) / len(times)
    out = {
        "metric": "single-event templates/s", "value": tm / (ms * 1e-3), "unit": "templates/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "single_event: the 13-sector star (247,104 observations), trial period "
                               "baseline + 2 x 15 h, 20 durations 0.5-15 h, 3 shapes x 4 layers",
                   "templates": tm, "survivors": stats["threshold_survivors"]},
        "step_ms": [round(t, 3) for t in times],
        "kernel_ms": {"fold": ctr["fold_ms"] / args.steps, "scan_all": ctr["scan_ms"] / args.steps},
        "gpu_launches": int(ctr["launches"]) // args.steps,
        "e2e": {"value": tm / (wall * 1e-3), "unit": "templates/s", "ms_per_step": wall,
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 40 * int(rows.shape[0])},
        "clocks": clk,
    }
    if not args.no_cpu:
        ost = oracle.family_state(c.time, c.flux, c.flux_err, cfg.durations_days())
        t0 = time.perf_counter()
        want, wst = oracle.single_event_search(ost, cfg)
        sec = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": wst["templates_scanned"] / sec, "unit": "templates/s", "cores": 1,
                               "kind": "port", "sample": f"the whole search on the oracle (fold, prefix, every "
                                                         f"template), single thread, {sec:.2f} s"}
        out["parity"] = bool(np.array_equal(rows, want))
    print(json.dumps(out))
    dev.free()
    gpu.close()


def _evidence_candidates(gpu, st, cfg, count: int):
    """The `count` strongest distinct periods (0.1 % apart) of the star's
    signal_search rows at the configuration's threshold (the candidates the
    pipeline's evidence step would see)."""
    rows, _, _ = gpu.signal_search(st, cfg)
    periods = []
    for i in np.argsort(-rows[:, 3]):
        p = float(rows[i, 0])
        if all(abs(p - q) > 1e-3 * q for q in periods):
            periods.append(p)
        if len(periods) == count:
            break
    return periods


def run_evidence(args):
    """Evidence (model comparison): a step is one fbls_compare_batch of
    --candidates trial periods of the 13-sector star (its strongest distinct
    signal_search periods; the family resident). value: candidates per second
    of device time (CUDA events around the batch on the context's stream);
    e2e: of the whole call with the rows back on the host."""
    import torch
    import oracle
    from fbls_b200 import api, synth
    torch.cuda.set_device(0)
    c, cfg = synth.multi_sector(), synth.multi_sector_config()
    # The 400 ppm star has few periods over the default threshold (7.1): the
    # candidates and the comparison use 5.0, so that every candidate passes
    # the screen and runs the full joint pass.
    cfg.threshold = 5.0
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    gpu = api.Gpu(0)
    dev = gpu.upload(st)
    periods = _evidence_candidates(gpu, st, cfg, args.candidates)
    cands = [(st, p) for p in periods]
    devs = [dev] * len(cands)
    for _ in range(args.warmup):
        got = gpu.compare_batch(cands, cfg, devs=devs)
    gpu.counters(reset=True)
    clocks = Clocks(0)
    clocks.start()
    walls, dev_ms = [], []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gpu.timer_start()
        got = gpu.compare_batch(cands, cfg, devs=devs)
        dev_ms.append(gpu.timer_stop())
        walls.append((time.perf_counter() - t0) * 1e3)
    clk = clocks.stop()
    ctr = gpu.counters(reset=True)
    ms = sum(dev_ms) / len(dev_ms)
    wall = sum(walls) / len(walls)
    nrows = sum(len(g) for g in got)
    out = {
        "metric": "evidence candidates/s", "value": len(cands) / (ms * 1e-3), "unit": "candidates/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"evidence: {len(cands)} candidates of the 13-sector star (247,104 observations, "
                               f"20 durations 0.5-15 h, periods {min(periods):.3f}-{max(periods):.3f} d; the "
                               "strongest distinct periods of its search at threshold 5), planet / binary / noise "
                               "comparison per candidate at threshold 5",
                   "candidates": len(cands), "rows": nrows},
        "step_ms": [round(t, 3) for t in dev_ms],
        "gpu_launches": int(ctr["launches"]) // args.steps,
        "e2e": {"value": len(cands) / (wall * 1e-3), "unit": "candidates/s", "ms_per_step": wall,
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 2 * 13 * 8 * len(cands)},
        "clocks": clk,
    }
    if not args.no_cpu:
        ost = oracle.family_state(c.time, c.flux, c.flux_err, cfg.durations_days())
        sample = periods[:4]
        t0 = time.perf_counter()
        want = [oracle.compare_search(ost, p, cfg) for p in sample]
        sec = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": len(sample) / sec, "unit": "candidates/s", "cores": 1, "kind": "port",
                               "sample": f"the first {len(sample)} candidates on the oracle, single thread, "
                                         f"{sec:.2f} s"}
        ok = True
        for g, w in zip(got[:len(sample)], want):
            ok = ok and len(g) == len(w) and all(
                a["selection_flags"] == b["selection_flags"] and a["epoch"] == b["epoch"] and
                abs(a["log_bf_planet_noise"] - b["log_bf_planet_noise"]) <= 1e-9 * max(1.0, abs(b["log_bf_planet_noise"]))
                for a, b in zip(g, w))
        out["parity"] = bool(ok)
    print(json.dumps(out))
    dev.free()
    gpu.close()


def run_detrend(args):
    """Biweight detrending: a step is one
    fbls_biweight_flatten of the 13-sector curve (247,104 observations at
    120 s) with a 0.75 d window, c 5, 10 iterations, gap 0.5 d. value:
    observations per second of kernel time; e2e: of the whole call (window
    bounds on the host, upload, download)."""
    import torch
    import oracle
    from fbls_b200 import api, synth
    torch.cuda.set_device(0)
    c = synth.multi_sector()
    t = c.time - c.time[0]
    gpu = api.Gpu(0)
    for _ in range(args.warmup):
        out = gpu.biweight_flatten(t, c.flux, 0.75)
    gpu.set_kernel_timing(True)
    gpu.counters(reset=True)
    clocks = Clocks(0)
    clocks.start()
    times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = gpu.biweight_flatten(t, c.flux, 0.75)
        times.append((time.perf_counter() - t0) * 1e3)
    clk = clocks.stop()
    ctr = gpu.counters(reset=True)
    ms = ctr["detrend_ms"] / args.steps
    wall = sum(times) / len(times)
    n = t.shape[0]
    res = {
        "metric": "detrended observations/s (biweight, 0.75 d window)", "value": n / (ms * 1e-3),
        "unit": "observations/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "detrend: the 13-sector curve (247,104 observations at 120 s, 1 d gaps), biweight "
                               "window 0.75 d (about 540 observations), c 5, 10 iterations, gap 0.5 d"},
        "step_ms": [round(x, 2) for x in times], "gpu_launches": int(ctr["launches"]) // args.steps,
        "e2e": {"value": n / (wall * 1e-3), "unit": "observations/s", "ms_per_step": wall,
                "h2d_bytes_per_step": 16 * n, "d2h_bytes_per_step": 8 * n},
        "clocks": clk,
    }
    if not args.no_cpu:
        k = 2000
        t0 = time.perf_counter()
        want = oracle.biweight_flatten(t[:k], c.flux[:k], 0.75)
        sec = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": k / sec, "unit": "observations/s", "cores": 1, "kind": "port",
                               "sample": f"the first {k} observations through the oracle's form of the reference "
                                         f"kernel (single thread), {sec:.2f} s"}
        res["parity_sample"] = bool(np.array_equal(gpu.biweight_flatten(t[:k], c.flux[:k], 0.75), want))
    print(json.dumps(res))
    gpu.close()


def run_precision_report(args):
    """The precision forms against the FP64 reference on every period of every
    band at the coarse and the full nb. Modes of the scan: 0, the reference's
    mixed ranking (f32 pre-rank from compensated (hi, lo) f32 prefix pairs,
    f64 rescans and winner); 1, f64 ranking throughout (the FP64 oracle's
    arithmetic); 2, the f32 form (f32 ranking and winner from the (hi, lo)
    pairs only, no f64 prefix rows written or read). Per mode against mode 1:
    the share of periods with the same winning template (bin = phase, width,
    shape, duration) and the relative errors of the reported power (score^2),
    SNR (score) and depth, with the device time of the pass. And the bin
    index: for every observation at every 8th period of each band, the fold's
    f64 bin against an f32 product, a double-single product, and the
    double-single product with its exact f64 fallback near integers."""
    import torch
    from fbls_b200 import api
    curve, cfg, desc = _workload(args.workload, args.period_oversample)
    state = api.prepared_family(curve.time, curve.flux, curve.flux_err, cfg)
    grid, bands = api.band_plan(state, cfg)
    out = {"report": "precision", "workload": desc, "reference": "mode 1 (f64 ranking, the FP64 oracle's arithmetic)",
           "passes": [], "bins": []}
    key = [2, 3, 7, 8]  # phase, width, ingress (shape), rho (duration)
    with api.Gpu(0) as gpu:
        dev = gpu.upload(state)
        for band in bands:
            bank = api.bank_for(band, cfg)
            for nb in (band["nb"] // 2, band["nb"]):
                res, ms = {}, {}
                for mode in (1, 0, 2):
                    gpu.scan_bank(dev, band["periods"], bank, nb, precision_mode=mode)  # warm
                    torch.cuda.synchronize()
                    gpu.timer_start()
                    res[mode] = gpu.scan_bank(dev, band["periods"], bank, nb, precision_mode=mode)
                    ms[mode] = gpu.timer_stop()
                ref = res[1]
                ok = np.isfinite(ref[1]) & (ref[1] > 0)
                top = ok & (ref[1] >= bank.threshold)
                rec = {"nb": int(nb), "periods": int(len(band["periods"])), "periods_over_threshold": int(top.sum()),
                       "ms": {f"mode{m}": round(ms[m], 3) for m in ms}}
                for mode in (0, 2):
                    got = res[mode]
                    same = (got[0][:, key] == ref[0][:, key]).all(axis=1)
                    both = ok & same
                    rs = np.abs(got[1][both] - ref[1][both]) / ref[1][both]
                    rp = np.abs(got[1][both] ** 2 - ref[1][both] ** 2) / ref[1][both] ** 2
                    rd = np.abs(got[2][both] - ref[2][both]) / np.maximum(np.abs(ref[2][both]), 1e-300)
                    tb = top & same
                    rec[f"mode{mode}"] = {
                        "same_template": float(same[ok].mean()) if ok.any() else 1.0,
                        "same_template_over_threshold": float(same[top].mean()) if top.any() else 1.0,
                        "max_rel_snr": float(rs.max(initial=0.0)), "max_rel_power": float(rp.max(initial=0.0)),
                        "max_rel_depth": float(rd.max(initial=0.0)),
                        "p99_rel_snr": float(np.percentile(rs, 99)) if rs.size else 0.0,
                        "max_rel_snr_over_threshold": float(
                            (np.abs(got[1][tb] - ref[1][tb]) / ref[1][tb]).max(initial=0.0))}
                out["passes"].append(rec)
            scales = band["nb"] / np.asarray(band["periods"][::8], dtype=np.float64)
            b = gpu.precision_bins(dev, scales, band["nb"])
            b["nb"] = int(band["nb"])
            out["bins"].append(b)
        dev.free()
    p = out["passes"]
    w = [x["periods"] for x in p]
    for mode in (0, 2):
        out[f"mode{mode}"] = {
            "same_template": float(np.average([x[f"mode{mode}"]["same_template"] for x in p], weights=w)),
            "max_rel_snr": max(x[f"mode{mode}"]["max_rel_snr"] for x in p),
            "max_rel_power": max(x[f"mode{mode}"]["max_rel_power"] for x in p),
            "max_rel_depth": max(x[f"mode{mode}"]["max_rel_depth"] for x in p),
            "max_rel_snr_over_threshold": max(x[f"mode{mode}"]["max_rel_snr_over_threshold"] for x in p),
            "ms": sum(x["ms"][f"mode{mode}"] for x in p)}
    out["mode1_ms"] = sum(x["ms"]["mode1"] for x in p)
    tot = {k: sum(b[k] for b in out["bins"]) for k in out["bins"][0] if k != "nb"}
    out["bins_total"] = tot
    print(json.dumps(out))


def run_profile_case(args):
    """One bounded launch set for profiler captures. fold: one scan_bank pass
    of the 13-sector star's octave band [8, 16) d at its coarse grid (1536
    bins), first 4096 periods: one k_fold, one k_scan_tiles and one k_merge
    launch, ~0.6 GB on device. maps: the coarse maps of args.stars seeded
    survey stars in one fbls_coarse_features call: one k_bin_fields_jobs, one
    k_fold_walk_jobs and one k_map_features launch."""
    if args.profile_case == "maps":
        from fbls_b200 import api
        from fbls_b200 import proposal as pr
        stars, _ = _survey(args.stars, 1000)
        pstars = [(s, p) for _, s, p in stars]
        saved = np.load(pr.WEIGHTS)
        with api.Gpu(0) as gpu:
            devs = [gpu.upload(s) for s, _ in pstars]
            gpu.counters(reset=True)
            t0 = time.perf_counter()
            pr.features(gpu, pstars, devs, float(saved["bin_days"]), oversample=float(saved["map_oversample"]))
            ms = 1e3 * (time.perf_counter() - t0)
            ctr = gpu.counters()
            for d in devs:
                d.free()
        print(json.dumps({"case": "maps", "stars": len(pstars), "observations": sum(s.n for s, _ in pstars),
                          "ms": ms, "fold_updates": ctr["fold_updates"], "launches": ctr["launches"]}))
        return
    from fbls_b200 import api, synth
    curve, cfg = synth.multi_sector(), synth.multi_sector_config()
    state = api.prepared_family(curve.time, curve.flux, curve.flux_err, cfg)
    grid, bands = api.band_plan(state, cfg)
    band = bands[4]
    nb = band["nb"] // 2
    periods = band["periods"][:4096]
    with api.Gpu(0) as gpu:
        dev = gpu.upload(state)
        gpu.set_kernel_timing(True)
        rec, score, depth, flags, stats = gpu.scan_bank(dev, periods, api.bank_for(band, cfg), nb)
        ctr = gpu.counters()
        dev.free()
    print(json.dumps({"case": "fold", "nb": nb, "periods": len(periods), "observations": state.n,
                      "fold_ms": ctr["fold_ms"], "fold_updates": ctr["fold_updates"],
                      "fold_algorithmic_bytes": ctr["fold_bytes"], "scan_ms": ctr["scan_ms"],
                      "templates": stats["templates_scanned"]}))


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--profile-case", choices=["fold", "maps"], default=None,
                    help="run one bounded launch set for profiler captures instead of the benchmark")
    ap.add_argument("--precision-report", action="store_true",
                    help="compare the mixed f32/f64 ranking with f64 ranking on every period (one JSON line)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fbls_b200", choices=["fbls_b200", "reference"])
    ap.add_argument("--workload", default="multi_sector",
                    choices=["multi_sector", "single_sector", "survey", "proposal", "rescore", "single_event",
                             "detrend", "evidence", "full"])
    ap.add_argument("--candidates", type=int, default=32, help="evidence workload: candidates per batch")
    ap.add_argument("--rows", type=int, default=8192, help="rescore workload: rows per step")
    ap.add_argument("--stars", type=int, default=None,
                    help="survey / proposal workloads: stars per GPU (default 512); full: stars (default 10000)")
    ap.add_argument("--batch-workers", type=int, default=0,
                    help="survey / proposal workloads: search_batch host worker threads (0: stars fused into "
                         "job launches)")
    ap.add_argument("--bands", type=int, default=None,
                    help="proposal and full workloads: log-period bands (of 1024) searched per star (default: the "
                         "fewest whose held-out recall reaches the operating point's)")
    ap.add_argument("--period-oversample", type=float, default=None,
                    help="single-star workloads: period grid density (default 3; 19 gives multi_sector's ~1.2M "
                         "periods, 6.9 single_sector's ~30k)")
    ap.add_argument("--extras-stars", type=int, default=128,
                    help="default workload, 1 GPU: survey stars for the metric's survey and proposal keys (0: none)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--kernel-table", default=None,
                    help="proposal workload: after the timed steps, write the device time per kernel of one "
                         "exhaustive and one proposal step (torch.profiler, CUPTI) to this file")
    args = ap.parse_args()
    if args.stars is None:
        args.stars = 10000 if args.workload == "full" else 512
    if args.precision_report:
        run_precision_report(args)
    elif args.profile_case:
        run_profile_case(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "survey":
        run_survey(args)
    elif args.workload == "proposal":
        run_proposal(args)
    elif args.workload == "rescore":
        run_rescore(args)
    elif args.workload == "single_event":
        run_single_event(args)
    elif args.workload == "detrend":
        run_detrend(args)
    elif args.workload == "evidence":
        run_evidence(args)
    elif args.workload == "full":
        run_full(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
