"""Greedy peak selection with event-overlap rescoring (src/select/peaks.rs).

A row of the signal-search table is accepted when at least `min_events`
transit epochs hold three or more observations, fewer than half of its
in-transit observations are shared with accepted ephemerides, its amplitude
statistic without the observations of accepted ephemerides reaches the
threshold scaled by the square root of its unshared fraction (floored at half
the threshold), and the statistic without its strongest single event keeps at
least half of the threshold. After each acceptance the strongest remaining
rows are rescored, lazily, in blocks of 8192 (peaks.rs:308-487).

The rescoring sums run on the GPU (`Gpu.rescore_rows`, `Gpu.count_rows`, the
library's kernels for kernels.rs:936-1042); the rest is host logic restated
from the reference with the same f64 operations in the same order, so the
accepted peaks are the reference's.
"""
from __future__ import annotations

import heapq
import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from .api import FamilyState

NEG_INF = -math.inf


@dataclass
class Peak:
    """An accepted ephemeris (peaks.rs:18-45; evidence fields filled later)."""
    period_days: float
    epoch_bjd: float
    duration_hours: float
    snr: float
    snr_folded: float
    snr_without_strongest_event: float
    depth: float
    depth_ppm: float
    events: int
    family: int
    pass_: int
    row: int
    planet_log_odds: Optional[float] = None
    log_bf_planet_noise: Optional[float] = None
    log_bf_binary_noise: Optional[float] = None
    binary_secondary_ratio: Optional[float] = None
    binary_secondary_phase: Optional[float] = None
    binary_odd_even_ratio: Optional[float] = None
    binary_period_days: Optional[float] = None
    ingress_fraction: Optional[float] = None
    evidence_epoch_bjd: Optional[float] = None
    evidence_duration_hours: Optional[float] = None
    model_preferred: bool = False
    binary_diagnostics_complete: bool = False


@dataclass
class SingleEvent:
    """A single-event template kept by select_events (peaks.rs:47-55)."""
    epoch_bjd: float
    duration_hours: float
    snr: float
    depth: float
    depth_ppm: float
    points: int


@dataclass
class Selection:
    accepted: List[Peak]
    masks: List[np.ndarray]
    excluded: np.ndarray


def _fmax(a: float, b: float) -> float:
    """f64::max: the other operand when one is NaN."""
    if a != a:
        return b
    if b != b:
        return a
    return a if a > b else b


def round_half_away(x):
    """f64::round (halves away from zero), exactly, elementwise; the sign of
    a zero result is the input's, as there (-0.4 rounds to -0.0)."""
    x = np.asarray(x, dtype=np.float64)
    r = np.trunc(x)
    frac = x - r  # exact
    return np.copysign(r + np.where(np.abs(frac) >= 0.5, np.sign(x), 0.0), x)


def rem_euclid(x, m: float):
    """f64::rem_euclid for a positive or negative divisor, elementwise."""
    r = np.fmod(x, m)
    return np.where(r < 0.0, r + abs(m), r)


def transit_mask(time, period: float, epoch: float, duration: float, margin: float) -> np.ndarray:
    """curve.rs:572-585: |phase| <= (1 + margin) duration / 2."""
    t = np.asarray(time, dtype=np.float64)
    phase = rem_euclid((t - epoch) + period / 2.0, period) - period / 2.0
    return np.abs(phase) <= (1.0 + margin) * duration / 2.0


def overlap(a: np.ndarray, b: np.ndarray) -> float:
    """Fraction of a's observations also in b (peaks.rs:56-62)."""
    total = int(np.count_nonzero(a))
    if total == 0:
        return 0.0
    return float(np.count_nonzero(a & b)) / float(total)


def event_count(time, period: float, epoch: float, duration: float, minimum_points: int) -> int:
    """Distinct transit epochs with at least `minimum_points` in-transit
    observations (peaks.rs:65-82)."""
    t = np.asarray(time, dtype=np.float64)
    inside = transit_mask(t, period, epoch, duration, 0.0)
    cycles = round_half_away((t[inside] - epoch) / period).astype(np.int64)
    if cycles.size == 0:
        return 0
    _, counts = np.unique(cycles, return_counts=True)
    return int(np.count_nonzero(counts >= minimum_points))


def nearest_rho(state: FamilyState, duration: float) -> float:
    """rho of the family duration nearest `duration`, first on ties (peaks.rs:84-92)."""
    d = state.durations
    best = 0
    for i in range(1, len(d)):
        if abs(d[i] - duration) < abs(d[best] - duration):
            best = i
    return float(state.rho[best])


def positions(state: FamilyState, time_all: np.ndarray) -> np.ndarray:
    """Index of every family observation in the merged times (peaks.rs:95-103)."""
    idx = np.searchsorted(time_all, np.asarray(state.time) + state.origin, side="left")
    return np.minimum(idx, len(time_all) - 1)


def without_strongest_event(state: FamilyState, pos: np.ndarray, row, excluded: np.ndarray) -> Tuple[float, int]:
    """Box statistic after removing the strongest single event, and the
    number of events with data (peaks.rs:254-298)."""
    period, epoch, duration = float(row[0]), float(row[1]), float(row[2])
    t = np.asarray(state.time)
    keep = ~excluded[pos]
    ta = t + state.origin
    phase = rem_euclid((ta - epoch) + period / 2.0, period) - period / 2.0
    inside = keep & (np.abs(phase) <= duration / 2.0)
    members = np.flatnonzero(inside)
    if members.size == 0:
        return NEG_INF, 0
    cycles = round_half_away((ta[members] - epoch) / period).astype(np.int64)
    v, w = state.v, state.w
    sums = {}
    for i, cyc in zip(members.tolist(), cycles.tolist()):  # observation order, as the reference
        e = sums.setdefault(cyc, [0.0, 0.0, 0.0])
        e[0] += v[i]
        e[1] += w[i]  # p == w (curve.rs:440-447)
        e[2] += w[i]
    rho = nearest_rho(state, duration)
    c = state.baseline_norm
    strongest, best = 0, NEG_INF
    for cyc in sorted(sums):
        a, hp, ww = sums[cyc]
        value = a / rho / math.sqrt(_fmax(ww - hp * hp / c, 1e-300))
        if value > best:
            strongest, best = cyc, value
    a = hp = norm = 0.0
    for i, cyc in zip(members.tolist(), cycles.tolist()):
        if cyc != strongest:
            a += v[i]
            hp += w[i]
            norm += w[i]
    q = norm - hp * hp / c
    value = a / rho / math.sqrt(_fmax(q, 1e-300)) if (q > 0.0 and a > 0.0) else NEG_INF
    return value, len(sums)


class Rescorer:
    """Batched rescoring on the GPU (peaks.rs:113-252): box sums per row over
    the family observations outside the excluded set, in-transit counts over
    the merged time vector."""

    def __init__(self, gpu, states: Sequence[FamilyState], time_all: np.ndarray):
        self.gpu = gpu
        self.devs = [gpu.upload(s) for s in states]
        self.time_all = np.ascontiguousarray(time_all, dtype=np.float64)

    def close(self) -> None:
        for d in self.devs:
            d.free()
        self.devs = []

    def evaluate(self, indices: Sequence[int], table: np.ndarray, family: np.ndarray, states: Sequence[FamilyState],
                 pos: Sequence[np.ndarray], excluded: np.ndarray, threshold: float) -> List[Tuple[float, float]]:
        """(score, required threshold) of every row in `indices`."""
        idx = np.asarray(indices, dtype=np.int64)
        rows = np.ascontiguousarray(table[idx, :3])
        counts = self.gpu.count_rows(self.time_all, excluded.astype(np.uint8), rows)
        required = []
        for slot in range(len(idx)):
            total = float(max(int(counts[slot, 0]), 1))
            unshared = float(counts[slot, 1]) / total
            required.append(_fmax(threshold * math.sqrt(unshared), 0.5 * threshold))
        scores = [NEG_INF] * len(idx)
        fam = family[idx]
        for k, dev in enumerate(self.devs):
            slots = np.flatnonzero(fam == k)
            if slots.size == 0:
                continue
            sums = self.gpu.rescore_rows(dev, excluded[pos[k]].astype(np.uint8), rows[slots])
            c = states[k].baseline_norm
            for m, sl in enumerate(slots.tolist()):
                a, hp, norm = float(sums[m, 0]), float(sums[m, 1]), float(sums[m, 2])
                q = norm - hp * hp / c
                if q > 0.0 and a > 0.0:
                    scores[sl] = (a / nearest_rho(states[k], float(rows[sl, 2]))) / math.sqrt(_fmax(q, 1e-300))
        return [(scores[s], required[s]) for s in range(len(idx))]


def select_peaks(gpu, table: np.ndarray, family, states: Sequence[FamilyState], time_all: np.ndarray,
                 threshold: float, limit: int, min_events: int, taken: Sequence[np.ndarray],
                 excluded_in: np.ndarray, pass_: int, rescorer: Optional[Rescorer] = None) -> Selection:
    """peaks.rs:308-487. `table`: rows (period, epoch, duration, score, depth)
    of every family; `family`: the family of each row; `time_all`: the merged
    ascending times; `taken`: masks of ephemerides accepted earlier;
    `excluded_in`: observations excluded so far."""
    margin = 0.5
    max_iterations = 20000
    block = 8192
    table = np.asarray(table, dtype=np.float64).reshape(-1, 5)
    family = np.asarray(family, dtype=np.int64)
    time_all = np.ascontiguousarray(time_all, dtype=np.float64)
    accepted: List[Peak] = []
    masks = [np.asarray(m, dtype=bool) for m in taken]
    excluded = np.array(excluded_in, dtype=bool, copy=True)
    if table.shape[0] == 0:
        return Selection(accepted, masks, excluded)
    pos = [positions(s, time_all) for s in states]
    own = rescorer is None
    if own:
        rescorer = Rescorer(gpu, states, time_all)
    try:
        score = table[:, 3]
        remaining = np.where(np.isfinite(score) & (score >= threshold), score, NEG_INF).tolist()
        fresh = [not bool(excluded.any())] * table.shape[0]
        # Max-heap by score, ties to the lower row index (Entry's order).
        heap = [(-remaining[i], i) for i in range(table.shape[0]) if math.isfinite(remaining[i])]
        heapq.heapify(heap)

        def refresh() -> None:
            stale, kept = [], []
            while heap:
                nv, i = heapq.heappop(heap)
                if -nv != remaining[i]:
                    continue
                if fresh[i]:
                    kept.append((nv, i))
                else:
                    stale.append(i)
                    if len(stale) == block:
                        break
            for e in kept:
                heapq.heappush(heap, e)
            if not stale:
                return
            values = rescorer.evaluate(stale, table, family, states, pos, excluded, threshold)
            for (rescored, required), i in zip(values, stale):
                remaining[i] = rescored if rescored >= required else NEG_INF
                fresh[i] = True
                if math.isfinite(remaining[i]):
                    heapq.heappush(heap, (-remaining[i], i))

        iterations = 0
        while len(accepted) < limit and iterations < max_iterations:
            iterations += 1
            while heap and -heap[0][0] != remaining[heap[0][1]]:
                heapq.heappop(heap)
            if not heap:
                break
            i = heap[0][1]
            if not fresh[i]:
                refresh()
                continue
            heapq.heappop(heap)
            isolated = remaining[i]
            remaining[i] = NEG_INF
            row = table[i]
            mask = transit_mask(time_all, row[0], row[1], row[2], 0.0)
            if any(overlap(mask, other) >= 0.5 for other in masks):
                continue
            events = event_count(time_all, row[0], row[1], row[2], 3)
            if events < min_events:
                continue
            k = int(family[i])
            leftover, _ = without_strongest_event(states[k], pos[k], row, excluded)
            if min_events > 1 and leftover < 0.5 * threshold:
                continue
            wide = transit_mask(time_all, row[0], row[1], row[2], margin)
            excluded |= wide
            masks.append(wide)
            accepted.append(Peak(
                period_days=float(row[0]), epoch_bjd=float(row[1]), duration_hours=24.0 * float(row[2]),
                snr=isolated, snr_folded=float(row[3]), snr_without_strongest_event=leftover, depth=float(row[4]),
                depth_ppm=1e6 * float(row[4]), events=events, family=k, pass_=pass_, row=i))
            for j in range(len(fresh)):
                fresh[j] = False
            refresh()
    finally:
        if own:
            rescorer.close()
    return Selection(accepted, masks, excluded)


def select_events(table: np.ndarray, time, threshold: float, limit: int,
                  taken: Sequence[np.ndarray]) -> List[SingleEvent]:
    """Greedy suppression of single-event templates overlapping accepted
    ephemerides (peaks.rs:488-545)."""
    table = np.asarray(table, dtype=np.float64).reshape(-1, 5)
    t = np.asarray(time, dtype=np.float64)
    output: List[SingleEvent] = []
    masks = [np.asarray(m, dtype=bool) for m in taken]
    if table.shape[0] == 0:
        return output
    score = table[:, 3]
    remaining = np.where(np.isfinite(score) & (score >= threshold), score, NEG_INF)
    iterations = 0
    while len(output) < limit and iterations < 5000:
        iterations += 1
        top = remaining.max()
        i = int(np.flatnonzero(remaining == top)[-1])  # Iterator::max_by keeps the last of equal maxima
        if not math.isfinite(remaining[i]):
            break
        row = table[i]
        inside = np.abs(t - row[1]) <= row[2] / 2.0
        near = np.abs(table[:, 1] - row[1]) <= (table[:, 2] + row[2]) / 2.0
        remaining[near] = NEG_INF
        points = int(np.count_nonzero(inside))
        if points < 3 or any(overlap(inside, other) >= 0.5 for other in masks):
            continue
        masks.append(np.abs(t - row[1]) <= 0.75 * row[2])
        output.append(SingleEvent(epoch_bjd=float(row[1]), duration_hours=24.0 * float(row[2]), snr=float(row[3]),
                                  depth=float(row[4]), depth_ppm=1e6 * float(row[4]), points=points))
    return output
