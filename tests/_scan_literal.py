"""A literal NumPy restatement of the reference's scan path, written apart
from oracle/ (no shared code) so that the two readings of the reference check
each other. Test infrastructure only.

Follows src/search/kernels.rs operation for operation, vectorised across the
128 lanes of a tile (each NumPy float32 / float64 elementwise operation rounds
once, as the device's operations do):

  phase_cell            kernels.rs:314-327   (bin = floor(t * scale) mod nb)
  prefix_block          kernels.rs:237-309   (warp scans of 32, warp totals,
                                              carries; doubled copy; hi, lo)
  interval / interval32 kernels.rs:51-78
  shape_sums(_f32)      kernels.rs:80-146
  block_winner          kernels.rs:148-206   (max value, min key, min lane)
  rank_fast / rank_exact kernels.rs:389-455
  scan_tiles            kernels.rs:610-845   (f32 pass, tile shape gate,
                                              invalid key nb1 + j, near-tie /
                                              unsafe / sensitive retry,
                                              f64 rescan, f64 winner)
  merge_tiles           kernels.rs:1115-1155
  factors               scan.rs:157-171

scan_bank_literal also counts, per tile, which branch each pass took, so a
test can show that every branch was exercised.
"""
from __future__ import annotations

import math
from collections import Counter

import numpy as np

TILE = 128
F_V, F_W, F_N = 0, 1, 2
KEY_MAX = np.uint64(0xFFFFFFFFFFFFFFFF)
F32 = np.float32
NEG_INF = -math.inf


def _bins(time, scale: float, nb: int) -> np.ndarray:
    """phase_cell: floor of the one rounded f64 product, then mod nb (the
    reference's corrected-reciprocal quotient gives the exact remainder)."""
    cell = np.floor(np.asarray(time, dtype=np.float64) * scale).astype(np.int64)
    return cell % nb


def fold(time, v, w, scale: float, nb: int) -> np.ndarray:
    """Histogram [nb][3] (v, w, count), each bin's terms added in
    observation order (np.add.at is sequential)."""
    b = _bins(time, scale, nb)
    h = np.zeros((nb, 3))
    np.add.at(h[:, F_V], b, np.asarray(v, dtype=np.float64))
    np.add.at(h[:, F_W], b, np.asarray(w, dtype=np.float64))
    np.add.at(h[:, F_N], b, 1.0)
    return h


def _warp_scan(x: np.ndarray) -> np.ndarray:
    """Inclusive scan of 32 values by shuffle-up steps 1, 2, 4, 8, 16."""
    v = x.copy()
    lane = np.arange(32)
    off = 1
    while off < 32:
        other = np.concatenate([np.zeros(off), v[:-off]])
        v = np.where(lane >= off, v + other, v)
        off *= 2
    return v


def prefix_block(hist: np.ndarray, nb: int):
    """Doubled exclusive prefix rows [3][2nb + 1] in f64 and their (hi, lo)
    f32 pairs, with the reference's association: per 256-bin segment, warp
    scans of 32, each warp's offset = carry + the earlier warps' totals added
    in order, the carry grows by the sum of the segment's warp totals."""
    stride = 2 * nb + 1
    cum = np.zeros((3, stride))
    for field in range(3):
        carry = 0.0
        for seg in range(0, nb, 256):
            vals = np.zeros(256)
            take = min(256, nb - seg)
            vals[:take] = hist[seg:seg + take, field]
            local = np.concatenate([_warp_scan(vals[32 * w:32 * w + 32]) for w in range(8)])
            totals = [local[32 * w + 31] for w in range(8)]
            for lane in range(take):
                w = lane // 32
                offset = carry
                for k in range(w):
                    offset = offset + totals[k]
                cum[field, seg + lane + 1] = local[lane] + offset
            total = 0.0
            for k in range(8):
                total = total + totals[k]
            carry = carry + total
        cum[field, nb + 1:] = cum[field, 1:nb + 1] + carry
    hi = cum.astype(F32)
    lo = (cum - hi.astype(np.float64)).astype(F32)
    return cum, hi, lo


def factors_of(ingress, layers: int) -> np.ndarray:
    return np.array([1.0 - 2.0 * ing * ((l / (layers - 1)) if layers > 1 else 0.0)
                     for ing in ingress for l in range(layers)])


class _Lane:
    def __init__(self):
        self.best = np.full(TILE, NEG_INF)
        self.key = np.full(TILE, KEY_MAX, dtype=np.uint64)
        self.di = np.zeros(TILE, dtype=np.int64)
        self.bad = np.zeros(TILE, dtype=bool)
        self.sensitive = np.zeros(TILE, dtype=bool)
        self.unsafe = np.zeros(TILE, dtype=bool)


def _rank_fast(s: _Lane, a32, hp32, norm32, rho: float, baseline: float, valid, key, di: int, ctr: Counter):
    cn = F32(baseline) * norm32
    qq = F32(rho * rho) * (cn - hp32 * hp32)
    merit = a32 * a32 / qq
    safe = (cn > F32(0.0)) & (qq >= F32(0.001) * cn) & (merit >= F32(1e-30)) & (merit <= F32(1e30))
    s.unsafe |= valid & ~safe
    if (valid & ~safe).any():
        ctr["unsafe_lanes"] += int((valid & ~safe).sum())
    best = s.best.astype(F32)
    guard = F32(1e-5)
    near = (best > F32(0.0)) & (np.abs(merit - best) <= guard * np.fmax(merit, best))
    far_better = merit > best * (F32(1.0) + F32(4.0) * guard)
    ok = valid & safe
    s.sensitive = np.where(ok & far_better, False, s.sensitive | (ok & near))
    better = ok & ((merit > best) | ((merit == best) & (key < s.key)))
    s.best = np.where(better, merit.astype(np.float64), s.best)
    s.key = np.where(better, key, s.key)
    s.di = np.where(better, di, s.di)
    return np.where(ok, merit, F32(-np.inf))


def _rank_exact(s: _Lane, a, hp, norm, rho: float, baseline: float, valid, key, di: int):
    d = hp * hp / baseline
    q = norm - d
    s.bad |= valid & (q <= 0.0)
    candidate = (a / rho) / np.sqrt(np.fmax(q, 1e-300))
    merit = np.where(valid & (q > 0.0) & (candidate < np.inf), candidate, NEG_INF)
    better = (merit > s.best) | ((merit == s.best) & (key < s.key))
    s.best = np.where(better, merit, s.best)
    s.key = np.where(better, key, s.key)
    s.di = np.where(better, di, s.di)
    return merit


def _interval(cum, field, start, width):
    return cum[field, start + width] - cum[field, start]


def _interval32(hi, lo, field, start, width):
    return (hi[field, start + width] - hi[field, start]) + (lo[field, start + width] - lo[field, start])


def _shape_sums(cum, jj, k, outer, ing, factors, si, layers):
    if ing == 0.0:
        return outer
    l = float(layers)
    a = outer[0] / l
    hp = outer[1] / l
    norm = outer[2] / (l * l)
    for layer in range(1, layers):
        width = max(1, int(math.floor(k * factors[si * layers + layer] + 0.5)))
        start = jj + (k - width) // 2
        dw = _interval(cum, F_W, start, width)
        a = a + _interval(cum, F_V, start, width) / l
        hp = hp + dw / l
        norm = norm + dw * ((2.0 * layer + 1.0) / (l * l))
    return a, hp, norm


def _shape_sums_f32(hi, lo, jj, k, outer, ing, factors, si, layers):
    if ing == 0.0:
        return outer
    l = F32(layers)
    a = outer[0] / l
    hp = outer[1] / l
    norm = outer[2] / (l * l)
    for layer in range(1, layers):
        width = max(1, int(math.floor(k * factors[si * layers + layer] + 0.5)))
        start = jj + (k - width) // 2
        dw = _interval32(hi, lo, F_W, start, width)
        a = a + _interval32(hi, lo, F_V, start, width) / l
        hp = hp + dw / l
        norm = norm + dw * ((F32(2.0) * F32(layer) + F32(1.0)) / (l * l))
    return a, hp, norm


def _block_winner(value, key):
    """Largest value, then smallest key, then lowest lane."""
    best = 0
    for lane in range(1, TILE):
        v, k = value[lane], key[lane]
        if v > value[best] or (v == value[best] and k < key[best]):
            best = lane
    return value[best], key[best], best


def scan_tile(cum, hi, lo, scale, tile, nb, durations, rho, ingress, factors, layers, baseline, gate, n,
              ctr: Counter):
    """One tile of scan_tiles: (parts[9], key, flags)."""
    nd, ns = len(durations), len(ingress)
    j = tile * TILE + np.arange(TILE)
    jj = np.minimum(j, nb - 1)
    nb1 = np.uint64(nb + 1)
    state = _Lane()
    fast, retry = True, False
    winner_key, winner_di, winner_value, bad_any = KEY_MAX, 0, NEG_INF, False
    with np.errstate(all="ignore"):
        for pass_ in range(2):
            if pass_ == 1:
                if not retry:
                    break
                fast = False
                state = _Lane()
                ctr["rescans"] += 1
            gate_value = gate * gate / baseline if fast else gate
            for di in range(nd):
                raw_k = max(1, int(math.floor(durations[di] * scale + 0.5)))
                k = min(raw_k, nb // 2)
                r = rho[di]
                key = np.uint64(k) * nb1 + jj.astype(np.uint64)
                if fast:
                    count = _interval32(hi, lo, F_N, jj, k)
                    w = _interval32(hi, lo, F_W, jj, k)
                    outer32 = (_interval32(hi, lo, F_V, jj, k), w, w)
                    usable = (j < nb) & (raw_k < nb // 2) & (count >= F32(3.0)) & (
                        count.astype(np.float64) <= n - 3.0)
                    valid = usable & (outer32[0] > F32(0.0))
                    merit = _rank_fast(state, *outer32, r, baseline, valid, key, di, ctr).astype(np.float64)
                else:
                    count = _interval(cum, F_N, jj, k)
                    w = _interval(cum, F_W, jj, k)
                    outer = (_interval(cum, F_V, jj, k), w, w)
                    usable = (j < nb) & (raw_k < nb // 2) & (count >= 3.0) & (count <= n - 3.0)
                    valid = usable & (outer[0] > 0.0)
                    merit = _rank_exact(state, *outer, r, baseline, valid, key, di)
                if (valid & (merit >= gate_value)).any():
                    ctr["gate_open" if fast else "gate_open_f64"] += 1
                    for si in range(1, ns):
                        ing = ingress[si]
                        key2 = (np.uint64(si) * nb1 + np.uint64(k)) * nb1 + jj.astype(np.uint64)
                        if fast:
                            a, hp, norm = _shape_sums_f32(hi, lo, jj, k, outer32, ing, factors, si, layers)
                            _rank_fast(state, a, hp, norm, r, baseline, usable & (a > F32(0.0)), key2, di, ctr)
                        else:
                            w = _interval(cum, F_W, jj, k)
                            outer = (_interval(cum, F_V, jj, k), w, w)
                            a, hp, norm = _shape_sums(cum, jj, k, outer, ing, factors, si, layers)
                            _rank_exact(state, a, hp, norm, r, baseline, usable & (a > 0.0), key2, di)
                else:
                    ctr["gate_closed" if fast else "gate_closed_f64"] += 1
            if fast:
                none = state.best <= 0.0
                if none.any():
                    ctr["invalid_key_lanes"] += int(none.sum())
                state.key = np.where(none, nb1 + jj.astype(np.uint64), state.key)
            value, key, chosen = _block_winner(state.best, state.key)
            guard = 1e-5 if fast else 1e-10
            near_top = (state.best > 0.0) & (state.best >= value * (1.0 - guard))
            near_count = int(near_top.sum())
            near_sensitive = bool((near_top & state.sensitive).any())
            unsafe_any = bool(state.unsafe.any())
            winner_key, winner_value, winner_di = key, value, int(state.di[chosen])
            retry = fast and (unsafe_any or near_count > 1 or near_sensitive)
            if fast:
                if unsafe_any:
                    ctr["retry_unsafe"] += 1
                if near_count > 1:
                    ctr["retry_near_tie"] += 1
                if near_sensitive:
                    ctr["retry_sensitive"] += 1
            bad_any = bad_any or bool(state.bad.any())
    wk = int(winner_key)
    phase = wk % (nb + 1)
    width = (wk // (nb + 1)) % (nb + 1)
    si = min(wk // ((nb + 1) * (nb + 1)), ns - 1)
    ing = ingress[si]
    r = rho[winner_di]
    w = _interval(cum, F_W, phase, width)
    outer = (_interval(cum, F_V, phase, width), w, w)
    a0, hp, norm = _shape_sums(cum, phase, width, outer, ing, factors, si, layers)
    a = a0 / r
    d = hp * hp / baseline
    q = max(norm - d, 1e-300)
    val = a / math.sqrt(q) if winner_value > NEG_INF else NEG_INF
    depth = a / q * r
    flags = (1 if retry else 0) | (2 if bad_any else 0)
    return np.array([phase, width, a, norm, d, ing, r, val, depth]), wk, flags


def scan_bank_literal(time, v, w, baseline: float, periods, nb: int, durations, rho, ingress=(0.0, 0.2, 0.45),
                      layers: int = 4, gate: float = 0.6 * 7.1):
    """Every period's winner at nb bins: records [P, 9] (period, scale,
    phase, width, a, norm, d, ingress, rho), score, depth, flags (OR of the
    tiles'), and the branch counts."""
    ctr = Counter()
    factors = factors_of(ingress, layers)
    n = float(len(time))
    tiles = (nb + TILE - 1) // TILE
    P = len(periods)
    rec = np.zeros((P, 9))
    score = np.zeros(P)
    depth = np.zeros(P)
    flags = np.zeros(P, dtype=np.uint32)
    for f, period in enumerate(periods):
        scale = nb / period
        cum, hi, lo = prefix_block(fold(time, v, w, scale, nb), nb)
        # merge_tiles: the best tile by (score, lowest key)
        best, bkey, chosen, parts = NEG_INF, int(KEY_MAX), 0, []
        for t in range(tiles):
            part, key, fl = scan_tile(cum, hi, lo, scale, t, nb, durations, rho, ingress, factors, layers,
                                      baseline, gate, n, ctr)
            parts.append(part)
            flags[f] |= fl
            if part[7] > best or (part[7] == best and key < bkey):
                best, bkey, chosen = part[7], key, t
        rec[f, 0] = period
        rec[f, 1] = scale
        rec[f, 2:] = parts[chosen][:7]
        score[f] = best
        depth[f] = parts[chosen][8]
        ctr["tiles"] += tiles
    return rec, score, depth, flags, ctr
