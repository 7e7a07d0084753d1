"""fbls_search_batch: many stars on one device with several worker threads
must give, star for star, the rows of one signal_search per star."""
import numpy as np
import pytest

from fbls_b200 import api, synth

pytestmark = pytest.mark.gpu


def _stars(count, seed=11, max_sectors=2):
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        c = synth.survey_star(rng)
        if c.time[-1] - c.time[0] > 27.4 * max_sectors + 1:
            continue
        cfg = synth.survey_config(c)
        out.append((api.prepared_family(c.time, c.flux, c.flux_err, cfg), cfg))
    return out


@pytest.mark.parametrize("workers", [3, 0])
@pytest.mark.parametrize("uploaded", [False, True])
def test_batch_matches_per_star_search(gpu, uploaded, workers):
    """workers 3: host threads, one star each; workers 0: the stars' band
    scans fused into job launches."""
    stars = _stars(6)
    base = stars[0][1]
    pmax = [cfg.period_max for _, cfg in stars]
    want = [gpu.signal_search(st, cfg) for st, cfg in stars]
    devs = [gpu.upload(st) for st, _ in stars] if uploaded else None
    got = gpu.search_batch([st for st, _ in stars], base, period_max=pmax, devs=devs, workers=workers)
    for (rows, glen, templates), (wrows, wglen, wstats) in zip(got, want):
        assert glen == wglen
        assert templates == sum(s["templates_scanned"] for s in wstats)
        assert np.array_equal(rows, wrows)
    if devs:
        for d in devs:
            d.free()


@pytest.mark.parametrize("workers", [2, 0])
def test_batch_reports_the_failing_star(gpu, workers):
    stars = _stars(3)
    st = stars[1][0]
    short = api.FamilyState(st.time[:4], st.v[:4], st.w[:4], st.baseline_norm, st.origin, st.residual_energy,
                            st.durations, st.rho)
    states = [stars[0][0], short, stars[2][0]]
    with pytest.raises(api.FblsError, match="star 1: at least six observations"):
        gpu.search_batch(states, stars[0][1], period_max=[cfg.period_max for _, cfg in stars], workers=workers)


def test_fused_batch_with_ranges_matches_ranged_search(gpu):
    """Ranged searches (the proposal path's second step) fused over a batch."""
    stars = _stars(5, seed=23)
    base = stars[0][1]
    pmax = [cfg.period_max for _, cfg in stars]
    ranges = [[(0.9, 1.3), (4.0, 6.5)], None, [(2.0, 2.2)], [(0.5, 20.0)], [(7.5, 9.0), (11.0, 12.5)]]
    want = [gpu.signal_search(st, cfg, ranges=rg) for (st, cfg), rg in zip(stars, ranges)]
    got = gpu.search_batch([st for st, _ in stars], base, period_max=pmax, workers=0, ranges=ranges)
    for (rows, glen, templates), (wrows, wglen, wstats) in zip(got, want):
        assert glen == wglen
        assert templates == sum(s["templates_scanned"] for s in wstats)
        assert np.array_equal(rows, wrows)


def test_signal_search_reports_every_row_when_the_buffer_is_short(gpu):
    """With room for fewer rows than it finds, signal_search writes as many as
    fit and reports the full count."""
    import ctypes as C
    from fbls_b200 import _native as N
    c, cfg = synth.single_sector(), synth.single_sector_config()
    st = api.prepared_family(c.time, c.flux, c.flux_err, cfg)
    want = gpu.signal_search(st, cfg)[0]
    assert want.shape[0] > 3
    dev = gpu.upload(st)
    cc, keep = api._config(cfg)
    d, r = np.ascontiguousarray(st.durations), np.ascontiguousarray(st.rho)
    rows = np.full((2, 5), -1.0)
    n, glen, nb = C.c_uint32(0), C.c_uint64(0), C.c_uint32(0)
    stats = (N.ScanStats * 64)()
    rc = gpu.lib.fbls_signal_search(gpu.ctx, dev.handle, d.ctypes.data_as(N.c_double_p),
                                    r.ctypes.data_as(N.c_double_p), len(d), C.byref(cc),
                                    rows.ctypes.data_as(C.POINTER(N.Row)), 2, C.byref(n), C.byref(glen), stats,
                                    C.byref(nb))
    assert rc == 0
    assert n.value == want.shape[0]
    assert np.array_equal(rows, want[:2])
    dev.free()


def test_fused_batch_uploads_every_star(gpu):
    """The fused batch uploads a group's host families together (planned on
    several threads): results equal those of the same stars uploaded
    beforehand, for a batch large enough to plan in parallel."""
    stars = _stars(40, seed=31, max_sectors=1)
    base = stars[0][1]
    pmax = [cfg.period_max for _, cfg in stars]
    states = [st for st, _ in stars]
    devs = [gpu.upload(st) for st in states]
    want = gpu.search_batch(states, base, period_max=pmax, devs=devs, workers=0)
    got = gpu.search_batch(states, base, period_max=pmax, workers=0)
    for (rows, glen, templates), (wrows, wglen, wtemplates) in zip(got, want):
        assert glen == wglen and templates == wtemplates
        assert np.array_equal(rows, wrows)
    for d in devs:
        d.free()


@pytest.mark.parametrize("knobs", [{"fold_steal": 1}, {"batch_no_fill": 1}, {"fold_steal": 1, "batch_no_fill": 1}])
def test_work_stealing_and_whole_groups_give_the_same_rows(gpu, knobs):
    # The batch's walking-fold jobs by a persistent grid that takes units from
    # a counter (fold_steal) against a CTA per unit, and with each pass's
    # period groups kept whole (batch_no_fill) against groups cut to fill the
    # SMs pass by pass: the same rows bit for bit.
    from fbls_b200 import autotune
    rng = np.random.default_rng(31)
    stars = []
    for _ in range(24):
        c = synth.survey_star(rng)
        cfg = synth.survey_config(c)
        stars.append((api.prepared_family(c.time, c.flux, c.flux_err, cfg), cfg.period_max))
    base = synth.survey_config(synth.survey_star(np.random.default_rng(0)))
    saved = autotune.current()
    try:
        autotune.apply({**saved, "fold_steal": 0, "batch_no_fill": 0})
        want = gpu.search_batch([s for s, _ in stars], base, period_max=[p for _, p in stars], workers=0)
        autotune.apply({**saved, **knobs})
        got = gpu.search_batch([s for s, _ in stars], base, period_max=[p for _, p in stars], workers=0)
    finally:
        autotune.apply(saved)
    for (r1, g1, t1), (r2, g2, t2) in zip(got, want):
        assert np.array_equal(r1, r2) and g1 == g2 and t1 == t2


@pytest.mark.parametrize("threads,lockstep,pair,group", [
    (128, 0, 0, 0), (256, 3, 0, 0), (512, 4096, 0, 0), (1024, 3, 0, 0), (512, 0, 1, 0), (256, 3, 1, 0),
    (512, 4096, 1, 0),
    # group caps that give a period fewer lanes than a warp (down to 8)
    (1024, 0, 0, 128), (128, 3, 0, 16), (512, 0, 1, 128), (1024, 4096, 0, 64)])
def test_fold_cta_size_and_lockstep_give_the_same_rows(gpu, threads, lockstep, pair, group):
    # The walking fold at every CTA size, lockstep threshold, form (one or
    # two periods per lane) and group cap the tuning table allows, in both the per-star
    # search and the batch's job launches (where shapes of several CTA sizes
    # and forms share a wave), with and without work stealing: the same rows
    # bit for bit as the built-in shape.
    from fbls_b200 import autotune
    rng = np.random.default_rng(37)
    stars = []
    for _ in range(12):
        c = synth.survey_star(rng)
        cfg = synth.survey_config(c)
        stars.append((api.prepared_family(c.time, c.flux, c.flux_err, cfg), cfg.period_max))
    base = synth.survey_config(synth.survey_star(np.random.default_rng(0)))
    one = synth.single_sector()
    one_cfg = synth.single_sector_config()
    one_st = api.prepared_family(one.time, one.flux, one.flux_err, one_cfg)
    saved = autotune.current()
    try:
        autotune.reset()
        want = gpu.search_batch([s for s, _ in stars], base, period_max=[p for _, p in stars], workers=0)
        want_one = gpu.signal_search(one_st, one_cfg)
        # every class but the smallest at the CTA size under test, so a wave mixes sizes
        classes = {str(c): threads for c in range(7, 16)}
        for steal in (0, 1):
            autotune.apply({"fold_threads": classes, "lockstep_min": {str(c): lockstep for c in range(32)} if lockstep
                            else {}, "fold_pair": {c: pair for c in classes} if pair else {}, "fold_steal": steal,
                            "fold_group_max": {str(c): group for c in range(32)} if group else {}})
            got = gpu.search_batch([s for s, _ in stars], base, period_max=[p for _, p in stars], workers=0)
            for (r1, g1, t1), (r2, g2, t2) in zip(got, want):
                assert np.array_equal(r1, r2) and g1 == g2 and t1 == t2
        got_one = gpu.signal_search(one_st, one_cfg)
        assert np.array_equal(got_one[0], want_one[0]) and got_one[1] == want_one[1]
    finally:
        autotune.apply(saved)


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_fused_tile_scan_equals_the_separate_kernels(gpu, mode):
    # The walking fold scanning and merging its own tiles from the prefix
    # rows it keeps in shared memory (fused_scan) against the fold writing
    # the rows to device memory and k_scan_tiles and k_merge reading them
    # back (the default): the same records,
    # scores, depths and flags bit for bit, in each precision mode, for a
    # multi-band star (nb from 96 to 1,920, several period groups per CTA)
    # and a batch of survey stars (the job launches).
    import dataclasses
    from fbls_b200 import autotune
    one = synth.single_sector()
    cfg = dataclasses.replace(synth.single_sector_config(), precision_mode=mode)
    st = api.prepared_family(one.time, one.flux, one.flux_err, cfg)
    grid, bands = api.band_plan(st, cfg)
    rng = np.random.default_rng(41)
    stars = []
    for _ in range(8):
        c = synth.survey_star(rng)
        sc = synth.survey_config(c)
        stars.append((api.prepared_family(c.time, c.flux, c.flux_err, sc), sc.period_max))
    base = dataclasses.replace(synth.survey_config(synth.survey_star(np.random.default_rng(0))), precision_mode=mode)
    saved = autotune.current()
    out = {}
    try:
        dev = gpu.upload(st)
        # (fused, steal): fused scans in a CTA per unit and in the persistent
        # work-stealing grid (one launch covering fold, scan and merge).
        for fused, steal in ((0, 0), (1, 0), (1, 1)):
            autotune.apply({**saved, "fused_scan": fused, "fold_steal": steal})
            banks = [gpu.scan_bank(dev, b["periods"][:3000], api.bank_for(b, cfg), nb, precision_mode=mode)
                     for b in bands for nb in (b["nb"] // 2, b["nb"])]
            rows = gpu.signal_search(st, cfg, dev=dev)
            batch = gpu.search_batch([s for s, _ in stars], base, period_max=[p for _, p in stars], workers=0)
            out[(fused, steal)] = (banks, rows, batch)
        dev.free()
    finally:
        autotune.apply(saved)
    b0, r0, s0 = out[(0, 0)]
    for key in ((1, 0), (1, 1)):
        b1, r1, s1 = out[key]
        for x, y in zip(b1, b0):
            for u, v in zip(x[:4], y[:4]):
                assert np.array_equal(u, v, equal_nan=True)
        assert np.array_equal(r1[0], r0[0]) and r1[1] == r0[1]
        for (x, gx, tx), (y, gy, ty) in zip(s1, s0):
            assert np.array_equal(x, y) and gx == gy and tx == ty
