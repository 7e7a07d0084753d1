"""The proposal network in numpy f64 -- TEST INFRASTRUCTURE ONLY: the oracle
of fbls_b200.proposal.Net's forward pass, loss and gradients, which tests
compare with the device kernels (bf16 GEMM operands, f32 accumulation).

Parameters are one flat vector laid out as the Net lays them out: for each
convolution layer W (CH, ci*KW), where W[o, c*KW + k] weighs input channel c
at tap k, then its bias b (CH,); then the head's wh (CH,) and bh (1,).

Input x is channel-major (C, B, T). A layer computes
y[o, b, t] = b[o] + sum_{c,k} W[o, c*KW + k] * x[c, b, t + k - KW//2]
(zero outside [0, T)), then the activation (ReLU, or GELU y Phi(y) with the
normal CDF Phi), then the maximum over P consecutive t. The
head computes h[b, t] = sum_c wh[c] * z[c, b, t] + bh and the band logits
logits[b, g] = mean(h[b, g*G : (g+1)*G]) with G = T_out / bands. The loss is
the batch mean of the softmax cross-entropy of the band labels.

operands="f64" is the network's mathematics. operands="bf16" is the device's
numeric contract on top of it: every operand of the convolutions' GEMMs
(forward W and the im2col columns; backward the output gradient with the
columns, and W with the output gradient) is rounded to f32 and then to bf16,
to nearest with ties to even as the device's staging does; products and sums
stay in f64. Rounded activations move ReLU and max-pool decisions, so the
device's gradients follow this mode far more closely than the f64 one.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np
from scipy.special import erf


def _gelu(y):
    return 0.5 * y * (1.0 + erf(y / np.sqrt(2.0)))


def _gelu_grad(y):
    return 0.5 * (1.0 + erf(y / np.sqrt(2.0))) + y * np.exp(-0.5 * y * y) / np.sqrt(2.0 * np.pi)


def shapes(in_channels: int, channels: int, kw: int, pools: Sequence[int]) -> List[Tuple[str, Tuple[int, ...]]]:
    out = []
    ci = in_channels
    for _ in pools:
        out += [("W", (channels, ci * kw)), ("b", (channels,))]
        ci = channels
    return out + [("wh", (channels,)), ("bh", (1,))]


def _split(w: np.ndarray, layout):
    views, o = [], 0
    for _, s in layout:
        k = int(np.prod(s))
        views.append(w[o:o + k].reshape(s))
        o += k
    assert o == w.shape[0], (o, w.shape)
    return views


def bf16_round(a) -> np.ndarray:
    """f64 values rounded to f32, then to bf16 (nearest, ties to even), as f64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    out = r.view(np.float32).astype(np.float64)
    nan = np.isnan(f)
    out[nan] = np.nan
    return out.reshape(np.shape(a))


def _im2col(x: np.ndarray, kw: int) -> np.ndarray:
    """(C, B, T) -> (C*kw, B*T): row c*kw + k holds x[c, b, t + k - kw//2]."""
    C, B, T = x.shape
    pad = kw // 2
    xp = np.zeros((C, B, T + 2 * pad))
    xp[:, :, pad:pad + T] = x
    cols = np.empty((C, kw, B, T))
    for k in range(kw):
        cols[:, k] = xp[:, :, k:k + T]
    return cols.reshape(C * kw, B * T)


def _col2im(dcols: np.ndarray, C: int, B: int, T: int, kw: int) -> np.ndarray:
    pad = kw // 2
    d = dcols.reshape(C, kw, B, T)
    dxp = np.zeros((C, B, T + 2 * pad))
    for k in range(kw):
        dxp[:, :, k:k + T] += d[:, k]
    return dxp[:, :, pad:pad + T]


class ProposalNet:
    """Forward and backward of the network for one batch, in f64."""

    def __init__(self, in_channels: int, channels: int, kw: int, pools: Sequence[int], bands: int,
                 operands: str = "f64", activation: str = "relu"):
        if operands not in ("f64", "bf16"):
            raise ValueError("operands must be 'f64' or 'bf16'")
        if activation not in ("relu", "gelu"):
            raise ValueError("activation must be 'relu' or 'gelu'")
        self.activation = activation
        self.in_channels, self.channels, self.kw = in_channels, channels, kw
        self.pools, self.bands = tuple(pools), bands
        self._op = bf16_round if operands == "bf16" else (lambda a: a)
        self.layout = shapes(in_channels, channels, kw, pools)
        self.size = sum(int(np.prod(s)) for _, s in self.layout)

    def forward(self, w, x, labels=None):
        """(logits (B, bands), mean loss or None); keeps what backward needs."""
        w = np.asarray(w, dtype=np.float64)
        x = np.asarray(x, dtype=np.float64)
        p = _split(w, self.layout)
        C, B, T = x.shape
        cache = []
        h = x
        for l, P in enumerate(self.pools):
            W, b = p[2 * l], p[2 * l + 1]
            ci, Tl = h.shape[0], h.shape[2]
            cols = _im2col(h, self.kw)
            y = (self._op(W) @ self._op(cols)).reshape(self.channels, B, Tl) + b[:, None, None]
            r = np.maximum(y, 0.0) if self.activation == "relu" else _gelu(y)
            win = r.reshape(self.channels, B, Tl // P, P)
            arg = np.argmax(win, axis=3)  # first maximum of each window
            z = np.take_along_axis(win, arg[..., None], axis=3)[..., 0]
            cache.append((h, cols, y, arg, P))
            h = z
        wh, bh = p[-2], p[-1]
        T_out = h.shape[2]
        G = T_out // self.bands
        head = np.einsum("c,cbt->bt", wh, h) + bh[0]
        logits = head.reshape(B, self.bands, G).mean(axis=2)
        self._state = (p, cache, h, G, logits, labels)
        if labels is None:
            return logits, None
        lab = np.asarray(labels, dtype=np.int64)
        m = logits.max(axis=1, keepdims=True)
        lse = m[:, 0] + np.log(np.exp(logits - m).sum(axis=1))
        loss = float(np.mean(lse - logits[np.arange(B), lab]))
        return logits, loss

    def backward(self) -> np.ndarray:
        """Gradient of the last forward's mean loss, in the flat layout."""
        p, cache, z_last, G, logits, labels = self._state
        assert labels is not None, "backward needs a forward with labels"
        lab = np.asarray(labels, dtype=np.int64)
        B = logits.shape[0]
        m = logits.max(axis=1, keepdims=True)
        sm = np.exp(logits - m)
        sm /= sm.sum(axis=1, keepdims=True)
        dlogits = sm
        dlogits[np.arange(B), lab] -= 1.0
        dlogits /= B
        dhead = np.repeat(dlogits, G, axis=1) / G  # (B, T_out)
        wh = p[-2]
        grads = [None] * len(p)
        grads[-2] = np.einsum("bt,cbt->c", dhead, z_last)
        grads[-1] = np.array([dhead.sum()])
        dz = wh[:, None, None] * dhead[None]
        for l in reversed(range(len(self.pools))):
            h, cols, y, arg, P = cache[l]
            W = p[2 * l]
            ci, _, Tl = h.shape
            dr = np.zeros((self.channels, B, Tl // P, P))
            np.put_along_axis(dr, arg[..., None], dz[..., None], axis=3)
            dy = dr.reshape(self.channels, B, Tl) * ((y > 0.0) if self.activation == "relu" else _gelu_grad(y))
            grads[2 * l + 1] = dy.sum(axis=(1, 2))
            dy2 = dy.reshape(self.channels, B * Tl)
            grads[2 * l] = self._op(dy2) @ self._op(cols).T
            if l > 0:
                dz = _col2im(self._op(W).T @ self._op(dy2), ci, B, Tl, self.kw)
        return np.concatenate([g.reshape(-1) for g in grads])
