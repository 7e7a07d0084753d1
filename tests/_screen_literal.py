"""A literal NumPy restatement of the evidence screen (src/search/evidence.rs)
written apart from oracle/, to pin the oracle's reading of it. Test
infrastructure only. Vectorised over the 64 lanes of a tile; every f64
operation in the reference's order.

  host set-up         evidence.rs:699-747  (durations below P / 4, sorted;
                                            nb; duration log masses; shape
                                            priors and layer table)
  fold_two            evidence.rs:75-92    (bin = floor(t scale) mod 2 nb)
  prefix_fields       evidence.rs:96-144   (Hillis-Steele over 256 bins per
                                            segment, plus the carry)
  circular_sum        evidence.rs:37-45
  layered_sum         evidence.rs:48-65
  comparison_screen   evidence.rs:151-273
  screen maximum, pilot tile (last maximum of the planet bound) and pilot
  key                 evidence.rs:834-844

positive_amplitude_evidence and log_add are taken from the oracle's scalar
functions (pinned separately against mpmath); everything else is written
here.
"""
from __future__ import annotations

import math

import numpy as np

import oracle

EV_TILE = 64


def setup(state, period: float, cfg):
    ds = sorted(((d, r) for d, r in zip(state.durations, state.rho) if d < period / 4.0), key=lambda x: x[0])
    if not ds:
        return None
    durations = [d for d, _ in ds]
    rho = [r for _, r in ds]
    ns, layers = len(cfg.ingress_fractions), cfg.shape_layers
    n = state.time.shape[0]
    nb = max(8, 4 * int(math.ceil(cfg.phase_oversample * period / durations[0] / 4.0)))
    scale = nb / period
    dlm = [-0.5 * ((n - 1.0) * math.log(r * r) + state.residual_energy / (r * r)) for r in rho]
    dmax = max(dlm)
    dlm = [x - dmax for x in dlm]
    logits = [(-4.0 * i, 2.0 * i) for i in cfg.ingress_fractions]

    def lse(v):
        high = max(v)
        return high if high == -math.inf else high + math.log(sum(math.exp(x - high) for x in v))

    lp0, lb0 = lse([l[0] for l in logits]), lse([l[1] for l in logits])
    priors = [x for l in logits for x in (l[0] - lp0, l[1] - lb0)]
    shapes = []
    for ing in cfg.ingress_fractions:
        previous = 0.0
        for layer in range(layers):
            fraction = 1.0 - 2.0 * ing * layer / (max(layers, 2) - 1)
            inc = 1.0 / layers
            shapes.append((fraction, inc, inc * (2.0 * previous + inc)))
            previous += inc
    return dict(durations=durations, rho=rho, nb=nb, nb2=2 * nb, scale=scale, dlm=dlm, priors=priors,
                shapes=shapes, ns=ns, layers=layers, n=n)


def prefix_fields(state, s):
    nb2 = s["nb2"]
    cell = np.floor(state.time * s["scale"]).astype(np.int64) % nb2
    folded = np.zeros((3, nb2))
    np.add.at(folded[0], cell, state.v)
    np.add.at(folded[1], cell, state.w)
    np.add.at(folded[2], cell, 1.0)
    cum = np.zeros((3, nb2 + 1))
    lane = np.arange(256)
    for f in range(3):
        carry = 0.0
        for seg in range(0, nb2, 256):
            x = np.zeros(256)
            take = min(256, nb2 - seg)
            x[:take] = folded[f, seg:seg + take]
            stride = 1
            while stride < 256:
                add = np.concatenate([np.zeros(stride), x[:-stride]])
                x = np.where(lane >= stride, x + add, x)
                stride *= 2
            cum[f, seg + 1:seg + take + 1] = x[:take] + carry
            carry = carry + x[255]
    return cum


def _circ(row, start, width, nb2):
    j = start % nb2
    end = j + width
    return row[np.minimum(end, nb2)] - row[j] + row[np.maximum(end - nb2, 0)]


def _layered(row, start, width, s, si, squared):
    value = 0.0
    for layer in range(s["layers"]):
        fraction, inc, sq = s["shapes"][si * s["layers"] + layer]
        inner = max(1, int(math.floor(width * fraction + 0.5)))
        value = value + (sq if squared else inc) * _circ(row, start + (width - inner) // 2, inner, s["nb2"])
    return value


def screen(state, s, cum, params):
    """Per tile (max score, planet bound, binary bound, key); a tile without a
    usable template keeps zeros."""
    nb, nb2, n, c = s["nb"], s["nb2"], float(s["n"]), state.baseline_norm
    tiles = (nb + EV_TILE - 1) // EV_TILE
    out = np.zeros((tiles, 4))
    for tile in range(tiles):
        j = tile * EV_TILE + np.arange(EV_TILE)
        jj = np.minimum(j, nb - 1)
        best = np.full(EV_TILE, -math.inf)
        bound = np.full(EV_TILE, -math.inf)
        best_a, best_q = np.zeros(EV_TILE), np.ones(EV_TILE)
        best_null, best_ps, best_bs = np.zeros(EV_TILE), np.zeros(EV_TILE), np.zeros(EV_TILE)
        best_key = np.zeros(EV_TILE, dtype=np.int64)
        for di, (d, r) in enumerate(zip(s["durations"], s["rho"])):
            raw_k = max(1, int(math.floor(d * s["scale"] + 0.5)))
            k = min(raw_k, nb2 // 8 - 1)
            count = _circ(cum[2], jj, k, nb2) + _circ(cum[2], jj + nb, k, nb2)
            usable = (j < nb) & (raw_k < nb2 // 8) & (count >= 3.0) & (count <= n - 3.0)
            for si in range(s["ns"]):
                a = _layered(cum[0], jj, k, s, si, False) + _layered(cum[0], jj + nb, k, s, si, False)
                pe = _layered(cum[1], jj, k, s, si, False)
                po = _layered(cum[1], jj + nb, k, s, si, False)
                ne = _layered(cum[1], jj, k, s, si, True)
                no = _layered(cum[1], jj + nb, k, s, si, True)
                qe, qo, qeo = ne - pe * pe / c, no - po * po / c, -pe * po / c
                q = qe + qo + 2.0 * qeo
                with np.errstate(all="ignore"):
                    score = a / np.sqrt(np.fmax(q * (r * r), 1e-300))
                valid = usable & (a > 0.0) & (q > 0.0)
                merit = 0.5 * score * score + s["dlm"][di] + s["priors"][si * 2]
                up = valid & (merit > bound)
                best_a = np.where(up, a / (r * r), best_a)
                best_q = np.where(up, q / (r * r), best_q)
                best_null = np.where(up, s["dlm"][di], best_null)
                best_ps = np.where(up, s["priors"][si * 2], best_ps)
                best_bs = np.where(up, s["priors"][si * 2 + 1], best_bs)
                best_key = np.where(up, (si * len(s["durations"]) + di) * nb + jj, best_key)
                bound = np.where(up, merit, bound)
                best = np.where(valid & (score > best), score, best)
        maximum = -math.inf
        bound_maximum, chosen = -math.inf, EV_TILE
        for l in range(EV_TILE):
            if best[l] > maximum:
                maximum = best[l]
            if bound[l] > bound_maximum:
                bound_maximum, chosen = bound[l], l
        if chosen == EV_TILE:
            continue
        L = chosen
        pae = oracle.positive_amplitude_evidence
        lower_p = pae(best_a[L], best_q[L], params[0]) + math.log(0.75) + best_null[L] + best_ps[L]
        lower_b = (oracle.log_add(pae(best_a[L], best_q[L], params[1]), pae(best_a[L], best_q[L], params[2]))
                   + math.log(0.025) + best_null[L] + best_bs[L])
        out[tile] = (maximum, lower_p, lower_b, float(best_key[L]))
    return out


def pilot(state, period: float, cfg):
    """(screen maximum, pilot key) as compare_search picks them, or None when
    no duration is below a quarter period."""
    s = setup(state, period, cfg)
    if s is None:
        return None
    cum = prefix_fields(state, s)
    sc = screen(state, s, cum, oracle.evidence_parameters(cfg))
    maximum = max(sc[:, 0].max(), -math.inf)
    winner = 0
    for t in range(1, sc.shape[0]):
        if sc[t, 1] >= sc[winner, 1]:
            winner = t
    return maximum, sc[winner, 3], s
