"""Proposal path: the coarse periodogram (fbls_coarse_map) is, per period and
duration, the score of the best box template over all phases, the same value
the f64 scan reports for a one-duration box-only bank at the same nb."""
import math

import numpy as np
import pytest

from fbls_b200 import api, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("workload", ["small", "single_sector"])
def test_coarse_map_matches_the_f64_box_scan(gpu, workload):
    if workload == "small":
        c, cfg = synth.small_curve(), synth.small_config()
        periods = np.geomspace(0.6, 1.15, 257)
    else:
        c, cfg = synth.single_sector(), synth.single_sector_config()
        periods = np.geomspace(2.0, 3.9, 1000)
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    dev = gpu.upload(st)
    pick = [0, len(st.durations) // 3, len(st.durations) - 1]
    durations, rho = st.durations[pick], st.rho[pick]
    oversample = 2.0
    got = gpu.coarse_map(dev, periods, durations, rho, oversample)
    nb = max(8, math.ceil(oversample * periods[-1] / durations.min()))
    for d in range(len(pick)):
        bank = api.Bank(durations=[durations[d]], rho=[rho[d]], ingress=(0.0,), layers=1, shape_gate=0.0)
        rec, score, depth, flags, stats = gpu.scan_bank(dev, periods, bank, nb, precision_mode=1)
        want = np.where(np.isfinite(score) & (score > 0), score, 0.0).astype(np.float32)
        assert np.array_equal(got[:, d], want), (d, np.nonzero(got[:, d] != want)[0][:5])
    assert (got > 0).any()
    dev.free()


# ---- proposal network kernels against a PyTorch fp32 reference -------------

def _torch_net(net, x, labels):
    """The same network in PyTorch fp32 (reference only)."""
    import torch
    import torch.nn.functional as F
    from fbls_b200 import proposal as pr
    w = net.w.detach().clone().requires_grad_(True)
    o = 0
    params = []
    for kind, s in net.shapes:
        k = int(np.prod(s))
        params.append(w[o:o + k].view(*s))
        o += k
    h = x.permute(1, 0, 2)  # (B, C, T)
    ci = pr.MAP_CHANNELS
    for l, P in enumerate(pr.POOLS):
        W = params[2 * l].view(pr.CH, ci, pr.KW)
        y = F.conv1d(h, W, params[2 * l + 1], padding=pr.KW // 2)
        h = F.max_pool1d(F.gelu(y) if pr.ACTIVATION == "gelu" else F.relu(y), P)
        ci = pr.CH
    hh = torch.einsum("bct,c->bt", h, params[-2]) + params[-1]
    logits = hh.view(hh.shape[0], -1, pr.HEAD_G).mean(dim=2)
    loss = F.cross_entropy(logits, labels.long())
    loss.backward()
    return logits.detach(), loss.detach(), w.grad.detach()


def test_nn_gemm_matches_torch(gpu):
    import torch
    from fbls_b200 import proposal as pr
    net = pr.Net(0)
    g = torch.Generator().manual_seed(1)
    A = torch.randn(70, 130, generator=g).cuda()
    B = torch.randn(130, 90, generator=g).cuda()
    Cm = torch.zeros(70, 90).cuda()
    net._gemm(A, B, Cm, 70, 90, 130, (130, 1), (90, 1), (90, 1))
    ref = A.bfloat16().float() @ B.bfloat16().float()
    assert torch.allclose(Cm, ref, rtol=1e-4, atol=1e-3)
    # transposed operands through strides, batched, with beta
    Ct = torch.ones(2, 90, 70).cuda()
    At = torch.stack([A.t().contiguous(), 2 * A.t().contiguous()])  # (2, 130, 70): A(m,k) = At[k][m]
    net._gemm(At, B, Ct, 70, 90, 130, (1, 70), (90, 1), (1, 70), beta=1.0, batch=2, bs=(130 * 70, 0, 90 * 70))
    assert torch.allclose(Ct[0], ref.t() + 1, rtol=1e-4, atol=1e-3)
    assert torch.allclose(Ct[1], 2 * ref.t() + 1, rtol=1e-4, atol=2e-3)


def test_proposal_net_forward_and_gradients_match_torch(gpu):
    import torch
    from fbls_b200 import proposal as pr
    net = pr.Net(0, seed=3)
    B = 6
    g = torch.Generator().manual_seed(2)
    x = torch.randn(pr.MAP_CHANNELS, B, pr.T_IN, generator=g).cuda()
    labels = torch.randint(0, pr.BANDS, (B,), generator=g, dtype=torch.int32).cuda()
    logits, loss = net.forward(x, labels)
    net.backward(B)
    rl, rloss, rgrad = _torch_net(net, x, labels)
    scale = rl.abs().max().item()
    assert (logits - rl).abs().max().item() <= 0.03 * scale + 1e-3
    assert abs(loss.item() - rloss.item()) <= 0.02 * abs(rloss.item()) + 1e-3
    gv, rv = net.grad, rgrad
    cos = torch.nn.functional.cosine_similarity(gv, rv, dim=0).item()
    assert cos > 0.99, cos
    assert (gv - rv).norm().item() <= 0.1 * rv.norm().item()


def test_proposal_net_training_reduces_loss(gpu):
    import torch
    from fbls_b200 import proposal as pr
    net = pr.Net(0, seed=4)
    B = 16
    g = torch.Generator().manual_seed(5)
    labels = torch.randint(0, pr.BANDS, (B,), generator=g, dtype=torch.int32)
    x = torch.randn(pr.MAP_CHANNELS, B, pr.T_IN, generator=g) * 0.1
    for b in range(B):  # a bump at the label's band in every channel
        lo = int(labels[b]) * (pr.T_IN // pr.BANDS)
        x[:, b, lo:lo + pr.T_IN // pr.BANDS] += 2.0
    x, labels = x.cuda(), labels.cuda()
    first = None
    for _ in range(60):
        _, loss = net.forward(x, labels)
        first = loss.item() if first is None else first
        net.backward(B)
        net.adam(3e-3)
    _, loss = net.forward(x, labels)
    assert loss.item() < 0.3 * first


def test_ranged_search_rows_are_the_full_search_rows_in_range(gpu):
    from fbls_b200 import proposal as pr
    c, cfg = synth.single_sector(), synth.single_sector_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    full, glen, _ = gpu.signal_search(st, cfg)
    assert full.shape[0] > 0
    ranges = pr.ranges_for(np.arange(pr.BANDS, dtype=float)[::-1] * 0 + np.eye(pr.BANDS)[[3, 12, 13, 20]].sum(0), 4)
    part, glen2, _ = gpu.signal_search(st, cfg, ranges=ranges)
    inside = np.zeros(full.shape[0], dtype=bool)
    for lo, hi in ranges:
        inside |= (full[:, 0] >= lo) & (full[:, 0] < hi)
    assert glen2 == glen
    assert np.array_equal(part, full[inside])
    # the same through the batch runner
    res = gpu.search_batch([st], cfg, period_max=[cfg.period_max], ranges=[ranges], workers=1)
    assert np.array_equal(res[0][0], full[inside])


@pytest.mark.parametrize("bin_days", [0.0, 600.0 / 86400.0])
def test_coarse_map_batch_matches_single_maps(gpu, bin_days):
    """workers 3: one map per worker thread; workers 0: every star's folds and
    box maps in shared job launches. Both equal one coarse_map per star."""
    from fbls_b200 import proposal as pr
    stars, cfg = pr.survey_stars(5, seed=3, max_sectors=2)
    devs = [gpu.upload(s) for s, _ in stars]
    p = pr.map_periods()
    plans = [pr.map_plan(st, pmax) for st, pmax in stars]
    want = [gpu.coarse_map(dev, p[keep], d, r, 2.0, bin_days=bin_days) for dev, (keep, d, r) in zip(devs, plans)]
    for workers in (3, 0):
        got = gpu.coarse_map_batch(devs, [p[keep] for keep, _, _ in plans], [d for _, d, _ in plans],
                                   [r for _, _, r in plans], 2.0, workers, bin_days)
        assert all(np.array_equal(g, w) for g, w in zip(got, want))
    for d in devs:
        d.free()


@pytest.mark.parametrize("bin_days", [0.0, 1200.0 / 86400.0])
def test_map_fold_shapes_do_not_change_the_maps(gpu, bin_days):
    """The coarse maps' folds at every lockstep threshold, CTA size and group
    cap the tuning table allows (caps above 32 give a period fewer lanes than
    a warp, and a cap drops the rule that every SM gets a CTA) give the same
    network input bit for bit."""
    from fbls_b200 import autotune
    from fbls_b200 import proposal as pr
    stars, cfg = pr.survey_stars(6, seed=9, max_sectors=3)
    devs = [gpu.upload(s) for s, _ in stars]
    saved = autotune.current()
    try:
        autotune.apply({**saved, "map_lockstep_min": 0, "map_threads": 0, "map_group_max": 0})
        want = pr.features(gpu, stars, devs, bin_days=bin_days, oversample=1.0)
        for lm, th, gm in ((3, 0, 0), (5, 0, 0), (4096, 0, 0), (0, 0, 32), (0, 0, 128), (3, 512, 64),
                           (0, 128, 16), (4096, 256, 32)):
            autotune.apply({**saved, "map_lockstep_min": lm, "map_threads": th, "map_group_max": gm})
            got = pr.features(gpu, stars, devs, bin_days=bin_days, oversample=1.0)
            assert np.array_equal(got, want), (lm, th, gm)
    finally:
        autotune.apply(saved)
    for d in devs:
        d.free()


@pytest.mark.parametrize("bin_days", [0.0, 600.0 / 86400.0])
def test_features_are_the_standardised_maps(gpu, bin_days):
    """fbls_coarse_features: the batch's network input equals, star for star,
    the features of one star, and map_features (numpy, f32) of its coarse map
    to f32 rounding."""
    from fbls_b200 import proposal as pr
    stars, cfg = pr.survey_stars(6, seed=5, max_sectors=3)
    devs = [gpu.upload(s) for s, _ in stars]
    x = pr.features(gpu, stars, devs, bin_days=bin_days)
    assert x.shape == (pr.MAP_CHANNELS, len(stars), pr.T_IN)
    # the same features copied device to device into a torch tensor
    xd = pr.features(gpu, stars, devs, bin_days=bin_days, device=True)
    assert xd.is_cuda and np.array_equal(xd.cpu().numpy(), x)
    p = pr.map_periods()
    for i, ((st, pmax), dev) in enumerate(zip(stars, devs)):
        assert np.array_equal(x[:, i, :], pr.star_map(gpu, dev, st, pmax, bin_days))
        keep, d, r = pr.map_plan(st, pmax)
        ref = pr.map_features(gpu.coarse_map(dev, p[keep], d, r, 2.0, bin_days=bin_days), keep)
        assert np.allclose(x[:, i, :], ref, rtol=1e-4, atol=1e-4)
        assert np.all(x[:, i, ~keep] == 0)
    for d in devs:
        d.free()


def test_coarse_map_batch_reports_the_failing_map(gpu):
    c, cfg = synth.small_curve(), synth.small_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    dev = gpu.upload(st)
    good = np.geomspace(0.6, 1.15, 100)
    bad = good[::-1].copy()  # not ascending
    d, r = st.durations[:2], st.rho[:2]
    want = gpu.coarse_map(dev, good, d, r, 2.0)
    for workers in (2, 0):
        with pytest.raises(api.FblsError, match="map 1: periods must be positive, finite and ascending"):
            gpu.coarse_map_batch([dev, dev, dev], [good, bad, good], [d] * 3, [r] * 3, 2.0, workers)
        got = gpu.coarse_map_batch([dev, dev], [good, good], [d] * 2, [r] * 2, 2.0, workers)
        assert all(np.array_equal(g, want) for g in got)
    dev.free()


def test_binned_coarse_map_is_the_map_of_the_binned_family(gpu):
    c, cfg = synth.small_curve(), synth.small_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    bin_days = 1500.0 / 86400.0
    t, v, w = st.time, st.v, st.w
    key = np.floor((t - t[0]) / bin_days)
    tb, vb, wb = [], [], []
    i = 0
    while i < len(t):
        j, st_t, sv, sw = i, 0.0, 0.0, 0.0
        while j < len(t) and key[j] == key[i]:
            st_t += t[j]
            sv += v[j]
            sw += w[j]
            j += 1
        tb.append(st_t / (j - i))
        vb.append(sv)
        wb.append(sw)
        i = j
    binned = api.FamilyState(np.array(tb), np.array(vb), np.array(wb), st.baseline_norm, st.origin,
                             st.residual_energy, st.durations, st.rho)
    periods = np.geomspace(0.6, 2.2, 300)
    d, r = st.durations[[0, -1]], st.rho[[0, -1]]
    dev, devb = gpu.upload(st), gpu.upload(binned)
    got = gpu.coarse_map(dev, periods, d, r, 2.0, bin_days=bin_days)
    want = gpu.coarse_map(devb, periods, d, r, 2.0)
    assert len(tb) < len(t)
    assert np.array_equal(got, want)
    dev.free()
    devb.free()


def test_graph_captured_inference_equals_launched_inference(gpu):
    # The inference graph (one capture of the 12 launches of a forward pass,
    # replayed per batch) gives the logits of the kernels launched one by one.
    import torch
    from fbls_b200 import proposal as pr
    net = pr.Net(0, seed=7)
    g = torch.Generator().manual_seed(9)
    x = torch.randn(pr.MAP_CHANNELS, 40, pr.T_IN, generator=g).numpy()
    a = pr.scores(net, x, batch=16, graph=True)
    b = pr.scores(net, x, batch=16, graph=False)
    assert a.shape == (40, pr.BANDS)
    assert np.array_equal(a, b)
    # the input as a device tensor: the same logits
    c = pr.scores(net, torch.from_numpy(x).to(net.dev), batch=16, graph=True)
    assert np.array_equal(a, c)
