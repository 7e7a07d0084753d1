"""Proposal network of the learned form: a 1D CNN that reads a star's coarse
periodogram (best box score per period and duration, from fbls_coarse_map)
and scores log-period bands, so that only the best bands get the exhaustive
scan.

Input: 4 durations x 8192 log-spaced periods over [0.5, 20] d. Six
convolution layers (kernel 7, 64 channels, GELU; max-pool 2 after each of the
first three), then a 1x1 head: 1024 band logits, one per position; the top 32
bands are searched. Every layer runs on this library's kernels (fbls_nn_*):
convolutions as bf16 tensor-core GEMMs with f32 accumulation, trained by
softmax cross-entropy and AdamW. torch is used for device buffers only.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N

PMIN, PMAX = 0.5, 20.0
T_IN = 8192
BANDS = 1024
CH = 64
KW = 7
POOLS = (2, 2, 2, 1, 1, 1)
HEAD_G = 1
MAP_CHANNELS = 4
ACTIVATION = "gelu"
TOP_BANDS = 32       # bands searched per star (cfg4's top-32)
# The held-out band recall the operating point asks for: above the metric's
# 99 % top-1 recall, because the held-out stars share the training stars'
# distribution (1-4 sectors, every star injected) and survey batches reach
# beyond it (up to 13 sectors, binary pairs): at 0.995 (3 bands) a 10,000-star
# survey batch measured 0.983.
OPERATING_RECALL = 0.999
WEIGHT_DECAY = 1e-4  # AdamW, on the convolution and head weights (not the biases)


_MAP_PERIODS = np.geomspace(PMIN, PMAX, T_IN)
_MAP_PERIODS.setflags(write=False)


def map_periods() -> np.ndarray:
    """The network's T_IN log-spaced map periods over [PMIN, PMAX] (read-only)."""
    return _MAP_PERIODS


def band_of(period: float) -> int:
    b = int(math.floor(BANDS * math.log(period / PMIN) / math.log(PMAX / PMIN)))
    return min(max(b, 0), BANDS - 1)


def band_range(b: int) -> Tuple[float, float]:
    r = math.log(PMAX / PMIN) / BANDS
    return PMIN * math.exp(r * b), PMIN * math.exp(r * (b + 1))


def map_bank(state) -> Tuple[np.ndarray, np.ndarray]:
    """Four of the family's durations (shortest, two inner, longest) and their rho."""
    d = np.asarray(state.durations, dtype=np.float64)
    order = np.argsort(d, kind="stable")
    idx = order[np.unique(np.round(np.linspace(0, len(d) - 1, MAP_CHANNELS)).astype(int))]
    while len(idx) < MAP_CHANNELS:
        idx = np.append(idx, idx[-1])
    return d[idx], np.asarray(state.rho, dtype=np.float64)[idx]


def map_range(state, period_max: float) -> Tuple[int, int]:
    """[i0, i1): the map periods a star's search covers (contiguous)."""
    lo = max(PMIN, 4.0 * float(np.min(state.durations)) * (1.0 + 1e-9))
    hi = min(period_max, float(state.time[-1]))
    i0 = int(np.searchsorted(_MAP_PERIODS, lo, side="left"))
    i1 = int(np.searchsorted(_MAP_PERIODS, hi, side="right"))
    return i0, max(i0, i1)


def map_plan(state, period_max: float):
    """The map periods a star's search covers (mask over map_periods()) and
    the map's durations and rho."""
    i0, i1 = map_range(state, period_max)
    keep = np.zeros(T_IN, dtype=bool)
    keep[i0:i1] = True
    d, r = map_bank(state)
    return keep, d, r


def map_features(m: np.ndarray, keep: np.ndarray) -> np.ndarray:
    """(4, T_IN) features: log1p of the coarse map, standardised per duration
    over the covered periods, 0 elsewhere. A numpy restatement of what
    fbls_coarse_features computes on the device (the tests' reference)."""
    x = np.zeros((MAP_CHANNELS, T_IN), dtype=np.float32)
    if keep.sum() < 8:
        return x
    f = np.log1p(np.maximum(m, 0.0)).T
    mu = f.mean(axis=1, keepdims=True)
    sd = f.std(axis=1, keepdims=True) + 1e-3
    x[:, keep] = (f - mu) / sd
    return x


def star_map(gpu, dev, state, period_max: float, bin_days: float = 0.0) -> np.ndarray:
    """(4, T_IN) features of one star (observations summed over bins of
    bin_days first when it is positive)."""
    return features(gpu, [(state, period_max)], [dev], bin_days=bin_days)[:, 0, :]


class Net:
    """Parameters (one flat f32 buffer), Adam state and per-batch workspaces."""

    def __init__(self, device: int = 0, seed: int = 0):
        import torch
        self.torch = torch
        self.dev = torch.device(f"cuda:{device}")
        self.lib = N.load()
        shapes = []
        ci = MAP_CHANNELS
        for _ in POOLS:
            shapes += [("W", (CH, ci * KW)), ("b", (CH,))]
            ci = CH
        shapes += [("wh", (CH,)), ("bh", (1,))]
        self.shapes = shapes
        n = sum(int(np.prod(s)) for _, s in shapes)
        g = torch.Generator().manual_seed(seed)
        flat = torch.zeros(n, dtype=torch.float32)
        o = 0
        for kind, s in shapes:
            k = int(np.prod(s))
            if kind == "W":
                flat[o:o + k] = torch.randn(k, generator=g) * math.sqrt(2.0 / s[1])
            elif kind == "wh":
                flat[o:o + k] = torch.randn(k, generator=g) * math.sqrt(1.0 / s[0])
            o += k
        self.w = flat.to(self.dev)
        self.grad = torch.zeros_like(self.w)
        self.m = torch.zeros_like(self.w)
        self.v = torch.zeros_like(self.w)
        self.t = 0
        self.views = []
        o = 0
        for kind, s in shapes:
            k = int(np.prod(s))
            self.views.append((self.w[o:o + k].view(*s), self.grad[o:o + k].view(*s)))
            o += k
        self._ws: Dict[int, dict] = {}
        self._graphs: Dict[int, tuple] = {}  # captured inference graphs by batch size
        self.ones = torch.ones(4096, dtype=torch.float32, device=self.dev)

    # -- workspace -------------------------------------------------------
    def _workspace(self, B: int) -> dict:
        if B in self._ws:
            return self._ws[B]
        torch = self.torch
        ws = {"X": [], "Xc": [], "Y": [], "Z": [], "idx": []}
        T = T_IN
        ci = MAP_CHANNELS
        for P in POOLS:
            ws["Xc"].append(torch.empty(ci * KW, B * T, device=self.dev))
            ws["Y"].append(torch.empty(CH, B * T, device=self.dev))
            ws["Z"].append(torch.empty(CH, B * (T // P), device=self.dev))
            ws["idx"].append(torch.empty(CH * B * (T // P), dtype=torch.uint8, device=self.dev))
            T //= P
            ci = CH
        ws["T_out"] = T
        ws["logits"] = torch.empty(B, BANDS, device=self.dev)
        ws["loss"] = torch.empty(B, device=self.dev)
        ws["dlogits"] = torch.empty(B, BANDS, device=self.dev)
        ws["labels"] = torch.empty(B, dtype=torch.int32, device=self.dev)
        self._ws[B] = ws
        return ws

    @staticmethod
    def _p(t) -> int:
        return t.data_ptr()

    def _check(self, rc: int, what: str):
        if rc != 0:
            raise RuntimeError(f"{what} failed with status {rc}")

    def _stream(self):
        """torch's current stream: the library's kernels run on it, so a
        forward pass can be captured into a CUDA graph."""
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    def _gemm(self, A, B, Cm, M, Nn, K, sa, sb, sc, alpha=1.0, beta=0.0, batch=1, bs=(0, 0, 0)):
        self._check(self.lib.fbls_nn_gemm(self._p(A), self._p(B), self._p(Cm), M, Nn, K, sa[0], sa[1], bs[0],
                                          sb[0], sb[1], bs[1], sc[0], sc[1], bs[2], batch, alpha, beta,
                                          self._stream()), "gemm")

    # -- forward / backward ------------------------------------------------
    def forward(self, x, labels=None):
        """x: device tensor (4, B, T_IN) f32 (channel-major). Returns logits (B, 32)
        and, with labels (B,) int32, the mean loss (a device scalar)."""
        B = x.shape[1]
        ws = self._workspace(B)
        lib = self.lib
        X = x.contiguous()
        T = T_IN
        ci = MAP_CHANNELS
        ws["X"] = [X]
        for l, P in enumerate(POOLS):
            W, _ = self.views[2 * l]
            b, _ = self.views[2 * l + 1]
            Xc, Y, Z, idx = ws["Xc"][l], ws["Y"][l], ws["Z"][l], ws["idx"][l]
            self._check(lib.fbls_nn_im2col(self._p(X), self._p(Xc), B, ci, T, KW, KW // 2, self._stream()), "im2col")
            n = B * T
            # Y (CH x n) = W (CH x ci*KW) . Xc (ci*KW x n)
            self._gemm(W, Xc, Y, CH, n, ci * KW, (ci * KW, 1), (n, 1), (n, 1))
            self._check(lib.fbls_nn_bias_gelu_pool(self._p(Y), self._p(b), self._p(Z), self._p(idx), B, CH, T, P,
                                                   self._stream()), "activation and pool")
            X = Z
            ws["X"].append(Z)
            T //= P
            ci = CH
        wh, _ = self.views[-2]
        bh, _ = self.views[-1]
        lab = None
        if labels is not None:
            ws["labels"].copy_(labels)
            lab = ws["labels"]
        self._check(lib.fbls_nn_head(self._p(X), self._p(wh), self._p(bh), self._p(lab) if lab is not None else None,
                                     self._p(ws["logits"]), self._p(ws["loss"]), self._p(ws["dlogits"]), B, CH, T,
                                     HEAD_G, self._stream()), "head")
        loss = ws["loss"].mean() if labels is not None else None
        return ws["logits"], loss

    def backward(self, B: int):
        """Gradients of the mean loss of the last forward (with labels) into self.grad."""
        ws = self._workspace(B)
        lib = self.lib
        torch = self.torch
        self.grad.zero_()
        T = ws["T_out"]
        wh, dwh = self.views[-2]
        bh, dbh = self.views[-1]
        Zl = ws["X"][-1]
        dZ = torch.empty_like(Zl)
        self._check(lib.fbls_nn_head_bwd(self._p(Zl), self._p(wh), self._p(ws["dlogits"]), self._p(dZ), self._p(dwh),
                                         self._p(dbh), B, CH, T, HEAD_G, self._stream()), "head backward")
        Ts = [T_IN]
        for P in POOLS:
            Ts.append(Ts[-1] // P)
        for l in reversed(range(len(POOLS))):
            P = POOLS[l]
            Tl = Ts[l]
            ci = MAP_CHANNELS if l == 0 else CH
            W, dW = self.views[2 * l]
            b, db = self.views[2 * l + 1]
            dY = torch.empty(CH, B * Tl, device=self.dev)
            self._check(lib.fbls_nn_bias_gelu_pool_bwd(self._p(dZ), self._p(ws["Y"][l]), self._p(ws["idx"][l]),
                                                       self._p(b), self._p(dY), self._p(db), B, CH, Tl, P,
                                                       self._stream()), "activation and pool backward")
            n = B * Tl
            Xc = ws["Xc"][l]
            kdim = ci * KW
            # dW (CH x kdim) = dY (CH x n) . Xc^T (n x kdim), split over S chunks of n.
            S = max(1, min(64, n // 8192))
            while n % S:
                S -= 1
            part = torch.empty(S, CH * kdim, device=self.dev)
            self._gemm(dY, Xc, part, CH, kdim, n // S, (n, 1), (1, n), (kdim, 1), batch=S,
                       bs=(n // S, n // S, CH * kdim))
            # dW += ones(1 x S) . part (S x CH*kdim)
            self._gemm(self.ones, part, dW, 1, CH * kdim, S, (0, 1), (CH * kdim, 1), (0, 1), beta=1.0)
            if l == 0:
                break
            # dXc (kdim x n) = W^T (kdim x CH) . dY (CH x n); dZ_prev = col2im(dXc)
            dXc = torch.empty(kdim, n, device=self.dev)
            self._gemm(W, dY, dXc, kdim, n, CH, (1, kdim), (n, 1), (n, 1))
            dZ = torch.empty(ci, B * Tl, device=self.dev)
            self._check(lib.fbls_nn_col2im(self._p(dXc), self._p(dZ), B, ci, Tl, KW, KW // 2, self._stream()),
                        "col2im")

    def adam(self, lr: float = 1e-3, weight_decay: float = WEIGHT_DECAY):
        """One AdamW step: weights decay, biases do not (one launch per
        parameter tensor)."""
        self.t += 1
        o = 0
        for kind, shape in self.shapes:
            k = int(np.prod(shape))
            wd = weight_decay if kind in ("W", "wh") else 0.0
            off = 4 * o
            self._check(self.lib.fbls_nn_adamw(self._p(self.w) + off, self._p(self.grad) + off, self._p(self.m) + off,
                                               self._p(self.v) + off, k, lr, 0.9, 0.999, 1e-8, wd, self.t,
                                               self._stream()), "adamw")
            o += k

    def state_dict(self) -> np.ndarray:
        return self.w.detach().cpu().numpy().copy()

    def load(self, flat: np.ndarray):
        self.w.copy_(self.torch.from_numpy(np.asarray(flat, dtype=np.float32)))


# ---- data, training, proposal ------------------------------------------------

def _survey_chunk(seed: int, start: int, count: int, max_sectors: int, inject_fraction: float):
    from . import api, synth
    out = []
    for i in range(start, start + count):
        attempt = 0
        while True:
            c = synth.survey_star(np.random.default_rng([seed, i, attempt]), inject_fraction=inject_fraction)
            attempt += 1
            if c.time[-1] - c.time[0] <= 27.4 * max_sectors + 1.0:
                break
        cfg = synth.survey_config(c)
        out.append((api.prepared_family(c.time, c.flux, c.flux_err, cfg), cfg.period_max))
    return out


def survey_stars(count: int, seed: int, max_sectors: int = 13, inject_fraction: float = 1.0):
    """Seeded survey stars (the survey generator of synth, one seeded stream
    per star, redrawn above max_sectors), prepared: [(FamilyState,
    period_max)] and the base SearchConfig. Large sets are generated on a
    pool of spawned processes."""
    from . import synth
    chunk = 500
    starts = list(range(0, count, chunk))
    sizes = [min(chunk, count - s) for s in starts]
    if count <= 2 * chunk:
        out = _survey_chunk(seed, 0, count, max_sectors, inject_fraction)
    else:
        import concurrent.futures as cf
        import multiprocessing as mp
        import os
        with cf.ProcessPoolExecutor(max_workers=min(32, os.cpu_count() or 1),
                                    mp_context=mp.get_context("spawn")) as ex:
            parts = ex.map(_survey_chunk, [seed] * len(starts), starts, sizes, [max_sectors] * len(starts),
                           [inject_fraction] * len(starts))
            out = [x for p in parts for x in p]
    return out, synth.survey_config(synth.survey_star(np.random.default_rng(0)))


def top_band(rows: np.ndarray) -> int:
    """Band of the exhaustive search's best row (-1 when it found none)."""
    if rows.shape[0] == 0:
        return -1
    return band_of(float(rows[int(np.argmax(rows[:, 3])), 0]))


def features(gpu, stars, devs, bin_days: float = 0.0, device: bool = False, oversample: float = 2.0):
    """(4, count, T_IN) float32, channel-major: every star's coarse map
    (phase cells of dmin / oversample over time bins of bin_days) and its
    features in one fbls_coarse_features call (map_features on the device);
    a numpy array, or with device=True a torch tensor left on the GPU for
    the network."""
    periods, ds, rs, offsets = [], [], [], []
    banks = {}
    for st, pmax in stars:
        i0, i1 = map_range(st, pmax)
        key = (st.durations.tobytes(), st.rho.tobytes())
        if key not in banks:
            banks[key] = map_bank(st)
        d, r = banks[key]
        periods.append(_MAP_PERIODS[i0:i1])
        ds.append(d)
        rs.append(r)
        offsets.append(i0)
    return gpu.coarse_features(devs, periods, ds, rs, offsets, T_IN, oversample, bin_days, device=device)


def train(net: Net, x: np.ndarray, y: np.ndarray, epochs: int = 30, batch: int = 128, lr: float = 2e-3,
          seed: int = 0, log=None):
    """AdamW (cosine learning rate) on the softmax cross-entropy of the band
    labels y (>= 0)."""
    torch = net.torch
    keep = np.nonzero(y >= 0)[0]
    xs = torch.from_numpy(x[:, keep, :]).to(net.dev)
    ys = torch.from_numpy(y[keep].astype(np.int32)).to(net.dev)
    rng = np.random.default_rng(seed)
    n = keep.shape[0]
    for ep in range(epochs):
        order = torch.from_numpy(rng.permutation(n)).to(net.dev)
        total = 0.0
        for s in range(0, n - batch + 1, batch):
            idx = order[s:s + batch]
            _, loss = net.forward(xs[:, idx, :], ys[idx])
            net.backward(batch)
            net.adam(lr * (0.5 * (1 + math.cos(math.pi * ep / epochs))))
            total += loss.item()
        if log:
            log(f"epoch {ep} loss {total / max(1, n // batch):.4f}")


def _inference_graph(net: Net, batch: int):
    """The forward pass of `batch` maps captured once into a CUDA graph (a
    static input buffer and logits), replayed for every batch: 12 kernel
    launches become one graph launch."""
    torch = net.torch
    if batch in net._graphs:
        return net._graphs[batch]
    xin = torch.zeros(MAP_CHANNELS, batch, T_IN, device=net.dev)
    side = torch.cuda.Stream(net.dev)
    side.wait_stream(torch.cuda.current_stream(net.dev))
    with torch.cuda.stream(side):
        net.forward(xin)  # workspace allocated before the capture
    torch.cuda.current_stream(net.dev).wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        logits, _ = net.forward(xin)
    net._graphs[batch] = (graph, xin, logits)
    return net._graphs[batch]


def scores(net: Net, x, batch: int = 256, graph: bool = True) -> np.ndarray:
    """Band logits (count, BANDS): the forward pass in batches, replayed from
    a captured CUDA graph (graph=False launches the kernels one by one). x is
    a numpy array or a torch tensor on the network's GPU (features(...,
    device=True)), which is read there without a copy through the host."""
    torch = net.torch
    out = []
    if graph:
        g, xin, logits = _inference_graph(net, batch)
    on_device = isinstance(x, torch.Tensor)
    for s in range(0, x.shape[1], batch):
        if on_device:
            xb = x[:, s:s + batch, :]
        else:
            xb = torch.from_numpy(np.ascontiguousarray(x[:, s:s + batch, :])).to(net.dev)
        n = xb.shape[1]
        if graph:
            xin[:, :n].copy_(xb)
            if n < batch:
                xin[:, n:].zero_()
            g.replay()
            out.append(logits[:n].detach().cpu().numpy().copy())
        else:
            lg, _ = net.forward(xb)
            out.append(lg[:n].detach().cpu().numpy().copy())
    return np.concatenate(out, axis=0)


def recall_at(logits: np.ndarray, y: np.ndarray) -> np.ndarray:
    """recall[k-1] = fraction of labelled stars whose band is in the top k."""
    keep = y >= 0
    order = np.argsort(-logits[keep], axis=1)
    hit = order == y[keep][:, None]
    return np.cumsum(hit, axis=1).sum(axis=0) / max(1, keep.sum()) if keep.any() else np.ones(BANDS)


def ranges_for(logits_row: np.ndarray, k: int) -> List[Tuple[float, float]]:
    """Period ranges of the k best bands, merged where adjacent."""
    best = sorted(np.argsort(-logits_row)[:k].tolist())
    out: List[Tuple[float, float]] = []
    for b in best:
        lo, hi = band_range(b)
        if out and abs(out[-1][1] - lo) < 1e-12 * hi:
            out[-1] = (out[-1][0], hi)
        else:
            out.append((lo, hi))
    if out:  # the outermost bands reach the grid ends
        if best[0] == 0:
            out[0] = (0.0, out[0][1])
        if best[-1] == BANDS - 1:
            out[-1] = (out[-1][0], float("inf"))
    return out


WEIGHTS = __import__("pathlib").Path(__file__).resolve().parent / "data" / "proposal_weights.npz"


def load_net(device: int = 0, path=None) -> Net:
    """The network with the committed weights (trained by main() below)."""
    net = Net(device)
    saved = np.load(path or WEIGHTS)
    net.load(saved["weights"])
    net.bin_days = float(saved["bin_days"]) if "bin_days" in saved.files else 0.0
    net.map_oversample = float(saved["map_oversample"]) if "map_oversample" in saved.files else 2.0
    return net


def bands_for_recall(target: float = 0.99, path=None) -> int:
    """The fewest bands whose held-out band recall (the committed weights'
    recall table: the exhaustive search's best band among the network's k
    best) reaches `target`: the k at which the proposal path runs at that
    recall."""
    rec = np.load(path or WEIGHTS)["recall"]
    hit = np.nonzero(rec >= target)[0]
    return int(hit[0]) + 1 if hit.size else BANDS


def search_proposed(gpu, net: Net, stars, devs, cfg, k: int = TOP_BANDS, workers: int = 0):
    """The proposal-pruned search of many stars: coarse maps and their
    features in one call, band scores, then the exhaustive search of each
    star's k best bands only (its rows are the full search's rows in those
    bands), by search_batch with `workers` (0: the stars' band scans fused into
    job launches). Returns the batch results and logits."""
    import time
    t0 = time.perf_counter()
    x = features(gpu, stars, devs, getattr(net, "bin_days", 0.0), device=True,
                 oversample=getattr(net, "map_oversample", 2.0))
    t1 = time.perf_counter()
    logits = scores(net, x)
    ranges = [ranges_for(l, k) for l in logits]
    t2 = time.perf_counter()
    res = gpu.search_batch([s for s, _ in stars], cfg, period_max=[p for _, p in stars], devs=devs,
                           workers=workers, ranges=ranges)
    t3 = time.perf_counter()
    search_proposed.last_ms = {"maps": 1e3 * (t1 - t0), "network": 1e3 * (t2 - t1), "search": 1e3 * (t3 - t2)}
    return res, logits


def main(argv=None):
    """Trains the proposal network on exhaustive-search labels of seeded survey
    stars and writes its weights and held-out recall:

        python -m fbls_b200.proposal --train 50000 --test 5000 --out weights.npz
    """
    import argparse
    import json
    import time
    from . import api
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--train", type=int, default=50000)
    ap.add_argument("--test", type=int, default=5000)
    ap.add_argument("--max-sectors", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--workers", type=int, default=0, help="search_batch workers of the labelling search")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--bin-minutes", type=float, default=10.0, help="time bins of the coarse map (0: none)")
    ap.add_argument("--map-oversample", type=float, default=2.0,
                    help="phase cells per shortest map duration of the coarse map")
    ap.add_argument("--labels", default=None,
                    help="band labels of these seeded stars from an earlier run (its .npz); else the exhaustive "
                         "search makes them")
    ap.add_argument("--out", required=True)
    args = ap.parse_args(argv)
    t0 = time.time()
    log = lambda m: print(f"[{time.time() - t0:7.1f} s] {m}", flush=True)
    stars, cfg = survey_stars(args.train + args.test, args.seed, args.max_sectors)
    log(f"prepared {len(stars)} stars")
    with api.Gpu(0) as gpu:
        devs = [gpu.upload(s) for s, _ in stars]
        if args.labels:
            prev = np.load(args.labels)
            if (int(prev["seed"]), int(prev["max_sectors"]), int(prev["labels"].shape[0])) != (
                    args.seed, args.max_sectors, len(stars)):
                raise SystemExit("--labels: made for other stars (seed, sectors or count differ)")
            y = prev["labels"]
        else:
            res = gpu.search_batch([s for s, _ in stars], cfg, period_max=[p for _, p in stars], devs=devs,
                                   workers=args.workers)
            y = np.array([top_band(r) for r, _, _ in res])
        log(f"exhaustive labels: {int((y >= 0).sum())} of {len(y)} stars with a detection")
        bin_days = args.bin_minutes / 1440.0
        x = features(gpu, stars, devs, bin_days, oversample=args.map_oversample)
        log("coarse maps done")
        net = Net(0, seed=args.seed)
        ntr = args.train
        train(net, x[:, :ntr], y[:ntr], epochs=args.epochs, log=log)
        lt = scores(net, x[:, ntr:])
        rec = recall_at(lt, y[ntr:])
        log("held-out recall@k " + " ".join(f"{k}:{rec[k - 1]:.4f}" for k in (1, 2, 4, 8, 16, 32, 64)))
        np.savez(args.out, weights=net.state_dict(), recall=rec, train=ntr, test=args.test, seed=args.seed,
                 max_sectors=args.max_sectors, epochs=args.epochs, bin_days=bin_days,
                 map_oversample=args.map_oversample, labels=y.astype(np.int16))
        print(json.dumps({"recall": rec.tolist(), "labelled_test": int((y[ntr:] >= 0).sum())}))
        for d in devs:
            d.free()


if __name__ == "__main__":
    main()
