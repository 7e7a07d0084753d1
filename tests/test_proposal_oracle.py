"""The proposal network's oracle (oracle/proposal_net.py, numpy f64) on the
CPU: its logits, loss and gradients against PyTorch autograd in f64 (an
independent implementation of the same network), a finite-difference check of
single weights, its parameter layout against the library's constants and the
committed weights, and its bf16-operand mode (the rounding against torch's
bf16 conversion; the mode near the f64 one)."""
import math

import numpy as np
import pytest

from oracle.proposal_net import ProposalNet, shapes
from fbls_b200 import proposal as pr

B = 5


def _net(operands="f64"):
    return ProposalNet(pr.MAP_CHANNELS, pr.CH, pr.KW, pr.POOLS, pr.BANDS, operands=operands, activation=pr.ACTIVATION)


def _weights(net, seed):
    """He-style initial weights as the library's Net draws them, with
    nonzero biases so that every term of the gradient is exercised."""
    rng = np.random.default_rng(seed)
    parts = []
    for kind, s in net.layout:
        k = int(np.prod(s))
        if kind == "W":
            parts.append(rng.normal(size=k) * math.sqrt(2.0 / s[1]))
        elif kind == "wh":
            parts.append(rng.normal(size=k) * math.sqrt(1.0 / s[0]))
        else:
            parts.append(rng.normal(size=k) * 0.05)
    return np.concatenate(parts)


def _inputs(seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(pr.MAP_CHANNELS, B, pr.T_IN))
    labels = rng.integers(0, pr.BANDS, B)
    return x, labels


def _torch(net, w, x, labels):
    """The same network with torch.nn.functional in f64 on the CPU."""
    import torch
    import torch.nn.functional as F
    wt = torch.tensor(w, dtype=torch.float64, requires_grad=True)
    views, o = [], 0
    for _, s in net.layout:
        k = int(np.prod(s))
        views.append(wt[o:o + k].view(*s))
        o += k
    h = torch.tensor(x, dtype=torch.float64).permute(1, 0, 2)
    ci = pr.MAP_CHANNELS
    for l, P in enumerate(pr.POOLS):
        W = views[2 * l].view(pr.CH, ci, pr.KW)
        y = F.conv1d(h, W, views[2 * l + 1], padding=pr.KW // 2)
        h = F.max_pool1d(F.gelu(y) if pr.ACTIVATION == "gelu" else F.relu(y), P)
        ci = pr.CH
    head = torch.einsum("bct,c->bt", h, views[-2]) + views[-1]
    logits = head.view(head.shape[0], pr.BANDS, -1).mean(dim=2)
    loss = F.cross_entropy(logits, torch.tensor(labels, dtype=torch.long))
    loss.backward()
    return logits.detach().numpy(), float(loss.item()), wt.grad.numpy()


def test_layout_matches_the_library_and_the_committed_weights():
    net = _net()
    assert net.layout == shapes(pr.MAP_CHANNELS, pr.CH, pr.KW, pr.POOLS)
    saved = np.load(pr.WEIGHTS)
    assert saved["weights"].shape == (net.size,)
    t_out = pr.T_IN
    for P in pr.POOLS:
        t_out //= P
    assert t_out // pr.BANDS == pr.HEAD_G


@pytest.mark.parametrize("seed", [1, 2])
def test_forward_and_gradients_match_torch_autograd(seed):
    net = _net()
    w = _weights(net, seed)
    x, labels = _inputs(seed + 10)
    logits, loss = net.forward(w, x, labels)
    grad = net.backward()
    tl, tloss, tgrad = _torch(net, w, x, labels)
    assert np.allclose(logits, tl, rtol=1e-12, atol=1e-12)
    assert abs(loss - tloss) <= 1e-12 * abs(tloss)
    assert np.allclose(grad, tgrad, rtol=1e-9, atol=1e-13)
    assert np.linalg.norm(grad) > 0


def test_gradient_by_finite_differences():
    net = _net()
    w = _weights(net, 3)
    x, labels = _inputs(13)
    net.forward(w, x, labels)
    grad = net.backward()
    offsets = np.cumsum([0] + [int(np.prod(s)) for _, s in net.layout])
    # one weight of every parameter block: the first and last conv layers, biases and the head
    picks = [int(offsets[k] + (offsets[k + 1] - offsets[k]) // 3) for k in range(len(net.layout))]
    for i in picks:
        h = 1e-6 * max(1.0, abs(w[i]))
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (net.forward(wp, x, labels)[1] - net.forward(wm, x, labels)[1]) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-5 * max(1e-3, abs(grad[i])), (i, fd, grad[i])


def test_committed_weights_give_finite_logits():
    net = _net()
    w = np.load(pr.WEIGHTS)["weights"].astype(np.float64)
    x, _ = _inputs(21)
    logits, loss = net.forward(w, x)
    assert loss is None and logits.shape == (B, pr.BANDS) and np.isfinite(logits).all()


def test_bf16_rounding_is_torch_round_to_nearest_even():
    import torch
    from oracle.proposal_net import bf16_round
    rng = np.random.default_rng(4)
    v = rng.normal(size=50000) * 10.0 ** rng.integers(-35, 35, 50000)
    v = np.concatenate([v, [0.0, -0.0, 1.0, 1.00390625, 1.01171875, 65504.0, 3.4e38, 1e-40, -1e-45, np.inf, -np.inf]])
    want = torch.from_numpy(v.astype(np.float32)).bfloat16().float().double().numpy()
    assert np.array_equal(bf16_round(v), want)
    assert np.isnan(bf16_round(np.array([np.nan]))[0])


def test_bf16_operand_mode_stays_near_the_f64_mode():
    w = _weights(_net(), 5)
    x, labels = _inputs(15)
    exact, rounded = _net(), _net("bf16")
    l64, loss64 = exact.forward(w, x, labels)
    g64 = exact.backward()
    l16, loss16 = rounded.forward(w, x, labels)
    g16 = rounded.backward()
    assert 0 < np.abs(l16 - l64).max() <= 0.03 * np.abs(l64).max()
    assert abs(loss16 - loss64) <= 0.02 * abs(loss64)
    assert g16 @ g64 / (np.linalg.norm(g16) * np.linalg.norm(g64)) > 0.95
    with pytest.raises(ValueError):
        ProposalNet(pr.MAP_CHANNELS, pr.CH, pr.KW, pr.POOLS, pr.BANDS, operands="f16")
    with pytest.raises(ValueError):
        ProposalNet(pr.MAP_CHANNELS, pr.CH, pr.KW, pr.POOLS, pr.BANDS, activation="tanh")
