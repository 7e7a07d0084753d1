"""Python API of the B200 search path, mirroring the reference's host API.

    Gpu(device)                      <- Gpu::new            src/search/scan.rs:66-77
    Gpu.upload(state)                <- DeviceReady::upload src/search/scan.rs:110-124
    Gpu.scan_periods(dev, p, bank)   <- scan_periods        src/search/scan.rs:363-408
    Gpu.scan_bank(dev, p, bank, nb)  <- scan_bank           src/search/scan.rs:144-357
    Gpu.signal_search(state, cfg)    <- signal_search       src/search/scan.rs:413-473
    Gpu.compare_search(state, P, cfg)<- compare_search      src/search/evidence.rs:693-1003
    family_state(...)                <- family_state        src/prep/curve.rs:541-569
    prepared_family(...)             <- search_prepared's preparation, src/pipeline.rs:41-68
    period_grid(...)                 <- period_grid         src/search/grid.rs:5-28

Every call goes through the C ABI of libfbls_b200.so; errors raise FblsError
with the library's message (the reference's text where it has one).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .config import SearchConfig

ROW_FIELDS = ("period", "epoch", "duration", "score", "depth")


class FblsError(RuntimeError):
    """Error raised by the native library (status code and message)."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(N.c_double_p)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


@dataclasses.dataclass
class Bank:
    """Template bank of one band; mirrors Bank (scan.rs:127-139)."""
    durations: Sequence[float]
    rho: Sequence[float]
    ingress: Sequence[float] = (0.0, 0.2, 0.45)
    layers: int = 4
    threshold: float = 7.1
    shape_gate: float = 0.6 * 7.1
    phase_oversample: int = 4
    period_batch: int = 4096
    max_fold_mib: float = 1024.0
    prescan_factor: int = 2
    prescan_fraction: float = 0.7

    def _native(self):
        d, r, g = _f64(self.durations), _f64(self.rho), _f64(self.ingress)
        b = N.Bank(_dptr(d), _dptr(r), len(d), _dptr(g), len(g), self.layers, self.threshold, self.shape_gate,
                   self.phase_oversample, self.period_batch, self.max_fold_mib, self.prescan_factor,
                   self.prescan_fraction)
        return b, (d, r, g)


@dataclasses.dataclass
class FamilyState:
    """Prepared family: the Ready fields (curve.rs:46-54) and rho."""
    time: np.ndarray        # relative to origin, ascending
    v: np.ndarray
    w: np.ndarray
    baseline_norm: float
    origin: float
    residual_energy: float
    durations: np.ndarray   # days, family order
    rho: np.ndarray
    inflation: float = 1.0
    segments: int = 1

    @property
    def n(self) -> int:
        return int(self.time.shape[0])


def _config(cfg: SearchConfig):
    ing = _f64(cfg.ingress_fractions)
    c = N.Config(cfg.period_min, cfg.period_max, cfg.threshold, _dptr(ing), len(ing), cfg.shape_layers,
                 cfg.phase_oversample, cfg.shape_gate_fraction, cfg.prescan_factor, cfg.prescan_fraction,
                 cfg.period_oversample, cfg.period_batch, cfg.max_fold_mib, cfg.evidence_rtol, cfg.planet_prior,
                 cfg.binary_prior, cfg.planet_depth_scale, cfg.binary_depth_scale, cfg.diluted_binary_depth_scale,
                 math.nan if cfg.stellar_radius_solar is None else cfg.stellar_radius_solar,
                 cfg.planet_radius_scale_rj, cfg.target_flux_fraction, int(cfg.precision_mode))
    return c, ing


def period_grid(minimum: float, maximum: float, baseline: float, minimum_duration: float,
                oversample: float) -> np.ndarray:
    lib = N.load()
    count = lib.fbls_period_grid(minimum, maximum, baseline, minimum_duration, oversample, None, 0)
    if count < 0:
        raise FblsError(1, "the period grid is infinite or too large")
    out = np.empty(count, dtype=np.float64)
    lib.fbls_period_grid(minimum, maximum, baseline, minimum_duration, oversample, _dptr(out), count)
    return out


def family_state(time, flux, sigma, durations_days: Sequence[float], correlated: bool = True) -> FamilyState:
    """family_state of a prepared curve (detrended relative flux, transits
    negative, per-point errors): noise model, precision fields and rho."""
    lib = N.load()
    t, f, s = _f64(time), _f64(flux), _f64(sigma)
    d = _f64(durations_days)
    n_in = t.shape[0]
    n_out = C.c_uint32(0)
    to, vo, wo = (np.empty(max(n_in, 1)) for _ in range(3))
    scal = np.empty(5)
    rho = np.empty(max(len(d), 1))
    err = C.create_string_buffer(256)
    rc = lib.fbls_family_state(_dptr(t), _dptr(f), _dptr(s), n_in, _dptr(d), len(d), int(correlated),
                               C.byref(n_out), _dptr(to), _dptr(vo), _dptr(wo), _dptr(scal), _dptr(rho), err, 256)
    if rc:
        raise FblsError(rc, err.value.decode())
    n = n_out.value
    return FamilyState(to[:n].copy(), vo[:n].copy(), wo[:n].copy(), float(scal[0]), float(scal[1]), float(scal[2]),
                       d.copy(), rho[:len(d)].copy(), float(scal[3]), int(scal[4]))


def _opt_f64(a):
    return None if a is None else _f64(a)


def _opt_i64(a):
    return None if a is None else np.ascontiguousarray(np.asarray(a, dtype=np.int64))


@dataclasses.dataclass
class NoiseModel:
    """DiagonalNoise (curve.rs:89-198): relative times, deficit, variance,
    group per observation, origin, inflation, segments."""
    time: np.ndarray
    deficit: np.ndarray
    variance: np.ndarray
    group: np.ndarray
    origin: float
    inflation: float
    segments: int


def fit_segment_noise(time, flux, err=None, group=None, bin_minutes: float = 0.0, gap_days: float = 0.75) -> NoiseModel:
    """The diagonal noise model of raw mission flux (host only)."""
    lib = N.load()
    t, f, e, g = _f64(time), _f64(flux), _opt_f64(err), _opt_i64(group)
    n_in = t.shape[0]
    to, do, vo = (np.empty(max(n_in, 1)) for _ in range(3))
    go = np.empty(max(n_in, 1), dtype=np.int64)
    scal = np.empty(3)
    n_out = C.c_uint32(0)
    msg = C.create_string_buffer(256)
    rc = lib.fbls_fit_segment_noise(_dptr(t), _dptr(f), None if e is None else _dptr(e),
                                    None if g is None else g.ctypes.data_as(C.POINTER(C.c_int64)), n_in,
                                    float(bin_minutes), float(gap_days), C.byref(n_out), _dptr(to), _dptr(do),
                                    _dptr(vo), go.ctypes.data_as(C.POINTER(C.c_int64)), _dptr(scal), msg, 256)
    if rc:
        raise FblsError(rc, msg.value.decode())
    n = n_out.value
    return NoiseModel(to[:n].copy(), do[:n].copy(), vo[:n].copy(), go[:n].copy(), float(scal[0]), float(scal[1]),
                      int(scal[2]))


def segment_edges(time, gap: float) -> np.ndarray:
    """Distance to the nearer edge of each gap-separated segment (curve.rs:332-345)."""
    t = _f64(time)
    out = np.empty_like(t)
    rc = N.load().fbls_segment_edges(_dptr(t), t.shape[0], float(gap), _dptr(out))
    if rc:
        raise FblsError(rc, "segment_edges")
    return out


def detrending_windows(durations, minimum: float, factor: float, maximum: float) -> List[Tuple[float, List[int]]]:
    """(window, duration indices) sorted by window (curve.rs:349-370)."""
    d = _f64(durations)
    w = np.empty(max(len(d), 1))
    fam = np.empty(max(len(d), 1), dtype=np.uint32)
    k = C.c_uint32(0)
    rc = N.load().fbls_detrending_windows(_dptr(d), len(d), float(minimum), float(factor), float(maximum), _dptr(w),
                                          fam.ctypes.data_as(N.c_uint32_p), C.byref(k))
    if rc:
        raise FblsError(rc, "detrending_windows")
    return [(float(w[j]), [i for i in range(len(d)) if fam[i] == j]) for j in range(k.value)]


@dataclasses.dataclass
class PreparedCurve:
    """One detrended curve of prepare_families (curve.rs:384-425)."""
    time: np.ndarray      # absolute
    flux: np.ndarray      # detrended relative flux
    sigma: np.ndarray
    window_days: float
    clipped: int
    indices: np.ndarray   # durations searched on this curve


def prepared_family(time, flux, flux_err, cfg: SearchConfig) -> FamilyState:
    """search_prepared's single family holding every duration (pipeline.rs:41-68)."""
    return family_state(time, flux, flux_err, cfg.durations_days(), cfg.correlated_noise)


class DeviceReady:
    """A family's fields resident on the GPU (DeviceReady, scan.rs:101-124)."""

    def __init__(self, gpu: "Gpu", handle: int, state: FamilyState):
        self.gpu = gpu
        self.handle = handle
        self.n = state.n
        self.origin = state.origin
        self.baseline_norm = state.baseline_norm

    def free(self) -> None:
        if self.handle:
            N.load().fbls_free_ready(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Gpu:
    """One device context and stream (Gpu, scan.rs:39-99)."""

    _tuning_loaded = False

    def __init__(self, device: int = 0, tuned: bool = True):
        self.lib = N.load()
        status = C.c_int(0)
        self.ctx = self.lib.fbls_create(device, C.byref(status))
        if not self.ctx:
            raise FblsError(status.value, f"cannot create a context on device {device}")
        self.device = device
        if tuned and not Gpu._tuning_loaded:
            # The measured launch-shape table (fbls_b200.autotune), when it was
            # measured on this device model; the rules apply otherwise.
            Gpu._tuning_loaded = True
            try:
                from . import autotune
                autotune.load_for(autotune.device_name(device))
            except (ImportError, RuntimeError):
                pass

    def close(self) -> None:
        if self.ctx:
            self.lib.fbls_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int) -> None:
        if rc:
            raise FblsError(rc, self.lib.fbls_last_error(self.ctx).decode())

    def timer_start(self) -> None:
        """Records a CUDA event on the context's stream."""
        self._check(self.lib.fbls_timer_start(self.ctx))

    def timer_stop(self) -> float:
        """Milliseconds of device time on the context's stream since timer_start."""
        ms = C.c_float(0.0)
        self._check(self.lib.fbls_timer_stop(self.ctx, C.byref(ms)))
        return float(ms.value)

    def set_kernel_timing(self, enable: bool) -> None:
        self._check(self.lib.fbls_set_kernel_timing(self.ctx, int(enable)))

    def counters(self, reset: bool = False) -> dict:
        c = N.Counters()
        self._check(self.lib.fbls_read_counters(self.ctx, C.byref(c), int(reset)))
        return c.as_dict()

    def upload(self, state: FamilyState) -> DeviceReady:
        t, v, w = _f64(state.time), _f64(state.v), _f64(state.w)
        h = C.c_void_p()
        self._check(self.lib.fbls_upload_ready(self.ctx, _dptr(t), _dptr(v), _dptr(w), t.shape[0],
                                               state.baseline_norm, state.origin, state.residual_energy,
                                               C.byref(h)))
        return DeviceReady(self, h.value, state)

    def scan_bank(self, dev: DeviceReady, periods, bank: Bank, nb: int, precision_mode: int = 0):
        """Every period's winner at nb bins: (records Px9, score, depth, flags, stats)."""
        p = _f64(periods)
        P = p.shape[0]
        rec = np.empty((P, 9))
        score = np.empty(P)
        depth = np.empty(P)
        flags = np.empty(P, dtype=np.uint32)
        st = N.ScanStats()
        b, keep = bank._native()
        rc = self.lib.fbls_scan_bank(self.ctx, dev.handle, _dptr(p), P, C.byref(b), nb, precision_mode, _dptr(rec),
                                     _dptr(score), _dptr(depth), flags.ctypes.data_as(N.c_uint32_p), C.byref(st))
        self._check(rc)
        return rec, score, depth, flags, st.as_dict()

    def scan_periods(self, dev: DeviceReady, periods, bank: Bank, precision_mode: int = 0):
        """Rows (N x 5: period, epoch, duration, score, depth) at or above the threshold, and ScanStats."""
        p = _f64(periods)
        P = p.shape[0]
        rows = (N.Row * max(P, 1))()
        n = C.c_uint32(0)
        st = N.ScanStats()
        b, keep = bank._native()
        self._check(self.lib.fbls_scan_periods(self.ctx, dev.handle, _dptr(p), P, C.byref(b), precision_mode, rows,
                                               C.byref(n), C.byref(st)))
        return _rows_array(rows, n.value), st.as_dict()

    def coarse_map(self, dev: DeviceReady, periods, durations, rho, oversample: float = 2.0,
                   bin_days: float = 0.0) -> np.ndarray:
        """Best box score over phases per (period, duration): P x nd float32."""
        p, d, r = _f64(periods), _f64(durations), _f64(rho)
        out = np.empty((p.shape[0], d.shape[0]), dtype=np.float32)
        self._check(self.lib.fbls_coarse_map(self.ctx, dev.handle, _dptr(p), p.shape[0], _dptr(d), _dptr(r),
                                             d.shape[0], float(oversample), float(bin_days),
                                             out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def coarse_map_batch(self, devs: Sequence[DeviceReady], periods: Sequence, durations: Sequence, rho: Sequence,
                         oversample: float = 2.0, workers: int = 8, bin_days: float = 0.0) -> List[np.ndarray]:
        """coarse_map of many uploaded families: on `workers` host threads,
        or (workers == 0) all together in shared job launches."""
        count = len(devs)
        jobs = (N.MapJob * max(count, 1))()
        keep, outs = [], []
        for i in range(count):
            p, d, r = _f64(periods[i]), _f64(durations[i]), _f64(rho[i])
            o = np.empty((p.shape[0], d.shape[0]), dtype=np.float32)
            keep += [p, d, r]
            outs.append(o)
            j = jobs[i]
            j.ready, j.periods, j.P = devs[i].handle, _dptr(p), p.shape[0]
            j.durations, j.rho, j.nd = _dptr(d), _dptr(r), d.shape[0]
            j.oversample = float(oversample)
            j.bin_days = float(bin_days)
            j.out = o.ctypes.data_as(C.POINTER(C.c_float))
        self._check(self.lib.fbls_coarse_map_batch(self.ctx, jobs, count, int(workers)))
        return outs

    def prepare_families(self, time, flux, err, group, cfg: SearchConfig) -> List[PreparedCurve]:
        """prepare_families (curve.rs:384-425): raw flux to one detrended
        curve per detrending window of cfg's durations (raw mode,
        pipeline.rs:27-37); the biweight detrend runs on the GPU."""
        t, f, e, g = _f64(time), _f64(flux), _opt_f64(err), _opt_i64(group)
        n = t.shape[0]
        d = _f64(cfg.durations_days())
        pc = N.PrepConfig(cfg.bin_minutes, cfg.window_days, cfg.window_factor, cfg.window_max_days, cfg.clip_sigma,
                          cfg.edge_trim_windows)
        outs = (N.FamilyOut * max(len(d), 1))()
        bufs = []
        for k in range(len(d)):
            arr = [np.empty(max(n, 1)) for _ in range(3)] + [np.empty(max(len(d), 1), dtype=np.uint32)]
            bufs.append(arr)
            outs[k].time, outs[k].flux, outs[k].sigma = (_dptr(a) for a in arr[:3])
            outs[k].indices = arr[3].ctypes.data_as(N.c_uint32_p)
        nf = C.c_uint32(0)
        self._check(self.lib.fbls_prepare_families(self.ctx, _dptr(t), _dptr(f), None if e is None else _dptr(e),
                                                   None if g is None else g.ctypes.data_as(C.POINTER(C.c_int64)), n,
                                                   _dptr(d), len(d), C.byref(pc), outs, C.byref(nf)))
        res = []
        for k in range(nf.value):
            o, arr = outs[k], bufs[k]
            m = o.n
            res.append(PreparedCurve(arr[0][:m].copy(), arr[1][:m].copy(), arr[2][:m].copy(), float(o.window_days),
                                     int(o.clipped), arr[3][:o.n_indices].copy()))
        return res

    def biweight_flatten(self, time, relative_flux, window: float, gap: float = 0.5, c: float = 5.0,
                         iterations: int = 10) -> np.ndarray:
        """biweight_flatten_gpu (curve.rs:256-329): (1 + relative_flux) over
        its biweight location in a sliding window, minus 1."""
        t, f = _f64(time), _f64(relative_flux)
        out = np.empty_like(t)
        self._check(self.lib.fbls_biweight_flatten(self.ctx, _dptr(t), _dptr(f), t.shape[0], float(window),
                                                   float(gap), float(c), int(iterations), _dptr(out)))
        return out

    def single_event_search(self, state: FamilyState, cfg: SearchConfig, capacity: int = 131072,
                            dev: Optional[DeviceReady] = None):
        """single_event_search (events.rs:18-153): rows (period inf, epoch,
        duration, score, depth) of every template above threshold at one
        trial period longer than the baseline, and the EventStats dict."""
        own = dev is None
        if own:
            dev = self.upload(state)
        try:
            c, keep = _config(cfg)
            d, r = _f64(state.durations), _f64(state.rho)
            out = np.empty((max(int(capacity), 1), 5))  # the pipeline's capacity (pipeline.rs:14)
            n = C.c_uint32(0)
            st = N.EventStats()
            self._check(self.lib.fbls_single_event_search(self.ctx, dev.handle, _dptr(d), _dptr(r), len(d),
                                                          C.byref(c), int(capacity),
                                                          out.ctypes.data_as(C.POINTER(N.Row)), C.byref(n),
                                                          C.byref(st)))
            return out[: n.value].copy(), st.as_dict()
        finally:
            if own:
                dev.free()

    def rescore_rows(self, dev: DeviceReady, excluded, rows) -> np.ndarray:
        """(R, 3) box sums a, hp, norm of rows (R x 3: period, epoch, duration)
        over the family's observations with excluded == 0 (rescore_rows,
        kernels.rs:936-990)."""
        r = _f64(rows).reshape(-1, 3)
        ex = np.ascontiguousarray(excluded, dtype=np.uint8)
        if ex.shape[0] != dev.n:
            raise ValueError("excluded must have one entry per family observation")
        out = np.empty((r.shape[0], 3))
        self._check(self.lib.fbls_rescore_rows(self.ctx, dev.handle, ex.ctypes.data_as(C.POINTER(C.c_uint8)),
                                               _dptr(r), r.shape[0], _dptr(out)))
        return out

    def count_rows(self, time, excluded, rows) -> np.ndarray:
        """(R, 2) in-transit counts of rows over an ascending time vector, and
        of those the not-excluded ones (count_rows, kernels.rs:993-1042)."""
        t = _f64(time)
        r = _f64(rows).reshape(-1, 3)
        ex = np.ascontiguousarray(excluded, dtype=np.uint8)
        if ex.shape[0] != t.shape[0]:
            raise ValueError("excluded must have one entry per time")
        out = np.empty((r.shape[0], 2), dtype=np.uint32)
        self._check(self.lib.fbls_count_rows(self.ctx, _dptr(t), t.shape[0], ex.ctypes.data_as(C.POINTER(C.c_uint8)),
                                             _dptr(r), r.shape[0], out.ctypes.data_as(N.c_uint32_p)))
        return out

    def coarse_features(self, devs: Sequence[DeviceReady], periods: Sequence, durations: Sequence, rho: Sequence,
                        offsets: Sequence[int], T: int, oversample: float = 2.0, bin_days: float = 0.0,
                        device: bool = False):
        """The proposal network's input (channels, len(devs), T) float32: each
        star's coarse map (channels = its durations), log1p'd and standardised
        per channel, at positions [offset, offset + len(periods)) of its row.
        device=True returns it as a torch tensor on the context's GPU (copied
        there device to device), else as a numpy array."""
        count = len(devs)
        channels = len(durations[0]) if count else 1
        jobs = (N.MapJob * max(count, 1))()
        keep = []
        for i in range(count):
            p, d, r = _f64(periods[i]), _f64(durations[i]), _f64(rho[i])
            keep += [p, d, r]
            j = jobs[i]
            j.ready, j.periods, j.P = devs[i].handle, _dptr(p), p.shape[0]
            j.durations, j.rho, j.nd = _dptr(d), _dptr(r), d.shape[0]
            j.oversample = float(oversample)
            j.bin_days = float(bin_days)
        offs = np.ascontiguousarray(offsets, dtype=np.uint32)
        if device:
            import torch
            x = torch.empty((channels, count, T), dtype=torch.float32, device=f"cuda:{self.device}")
            ptr = C.cast(C.c_void_p(x.data_ptr()), C.POINTER(C.c_float))
        else:
            x = np.empty((channels, count, T), dtype=np.float32)
            ptr = x.ctypes.data_as(C.POINTER(C.c_float))
        self._check(self.lib.fbls_coarse_features(self.ctx, jobs, count, offs.ctypes.data_as(N.c_uint32_p),
                                                  channels, T, ptr))
        return x

    def search_batch(self, states: Sequence[FamilyState], cfg: SearchConfig, period_max: Optional[Sequence[float]] = None,
                     devs: Optional[Sequence[DeviceReady]] = None, workers: int = 4,
                     ranges: Optional[Sequence[Optional[Sequence[Tuple[float, float]]]]] = None):
        """signal_search over many stars: [(rows N x 5, grid length,
        templates)] per star. workers >= 1 host threads each take one star at
        a time on a stream of their own; workers == 0 searches groups of stars
        together with job launches that cover every star of a group.
        period_max overrides cfg.period_max per star; devs are uploaded
        families (else the host arrays are uploaded); ranges restrict a star's
        search to period ranges [lo, hi)."""
        count = len(states)
        stars = (N.Star * max(count, 1))()
        keep = []
        # One row buffer for the batch, room for every grid period of each star
        # (rows cannot outnumber them); only the rows written are touched.
        caps = []
        for i, s in enumerate(states):
            pm = math.nan if period_max is None else float(period_max[i])
            c1 = dataclasses.replace(cfg, period_max=pm) if math.isfinite(pm) else cfg
            caps.append(max(1, _grid_count(s, c1)))
        offs = np.concatenate([[0], np.cumsum(caps)])
        rows_all = np.empty((int(offs[-1]), 5))
        for i, s in enumerate(states):
            st = stars[i]
            if devs is not None:
                st.ready = devs[i].handle
            else:
                t, v, w = _f64(s.time), _f64(s.v), _f64(s.w)
                keep += [t, v, w]
                st.time, st.v, st.w = _dptr(t), _dptr(v), _dptr(w)
                st.n = t.shape[0]
            st.baseline_norm, st.origin, st.residual_energy = s.baseline_norm, s.origin, s.residual_energy
            d, r = _f64(s.durations), _f64(s.rho)
            keep += [d, r]
            st.durations, st.rho, st.nd = _dptr(d), _dptr(r), len(d)
            pm = math.nan if period_max is None else float(period_max[i])
            st.period_max = pm
            st.rows = rows_all[offs[i]:].ctypes.data_as(C.POINTER(N.Row))
            st.capacity = caps[i]
            if ranges is not None and ranges[i]:
                rg = _f64(np.asarray(ranges[i], dtype=np.float64).reshape(-1))
                keep.append(rg)
                st.ranges = _dptr(rg)
                st.n_ranges = rg.shape[0] // 2
        c, ck = _config(cfg)
        self._check(self.lib.fbls_search_batch(self.ctx, stars, count, C.byref(c), int(workers)))
        out = []
        for i in range(count):
            st = stars[i]
            out.append((rows_all[offs[i]:offs[i] + st.n_rows].copy(), int(st.grid_len), int(st.templates)))
        return out

    def signal_search(self, state: FamilyState, cfg: SearchConfig, dev: Optional[DeviceReady] = None,
                      ranges: Optional[Sequence[Tuple[float, float]]] = None):
        """signal_search: (rows N x 5, grid length, per-band ScanStats); with
        ranges, only the grid periods in those [lo, hi) ranges are scanned."""
        own = dev is None
        if own:
            dev = self.upload(state)
        try:
            c, keep = _config(cfg)
            d, r = _f64(state.durations), _f64(state.rho)
            cap = max(1, _grid_count(state, cfg))  # rows cannot outnumber grid periods
            n = C.c_uint32(0)
            glen = C.c_uint64(0)
            stats = (N.ScanStats * 64)()
            nb = C.c_uint32(0)
            rg = _f64(np.asarray(ranges if ranges else [], dtype=np.float64).reshape(-1))
            rows = np.empty((cap, 5))  # not touched beyond the rows written
            self._check(self.lib.fbls_signal_search_ranges(self.ctx, dev.handle, _dptr(d), _dptr(r), len(d),
                                                           C.byref(c), _dptr(rg), rg.shape[0] // 2,
                                                           rows.ctypes.data_as(C.POINTER(N.Row)), cap, C.byref(n),
                                                           C.byref(glen), stats, C.byref(nb)))
            return rows[:n.value].copy(), int(glen.value), [stats[i].as_dict() for i in range(nb.value)]
        finally:
            if own:
                dev.free()

    def compare_search(self, state: FamilyState, period: float, cfg: SearchConfig,
                       dev: Optional[DeviceReady] = None) -> List[dict]:
        """Evidence rows (0, 1 or 2 dicts of EvidenceRow fields) at one period."""
        own = dev is None
        if own:
            dev = self.upload(state)
        try:
            c, keep = _config(cfg)
            d, r = _f64(state.durations), _f64(state.rho)
            rows = (N.EvidenceRow * 2)()
            n = C.c_uint32(0)
            self._check(self.lib.fbls_compare_search(self.ctx, dev.handle, _dptr(d), _dptr(r), len(d), float(period),
                                                     C.byref(c), rows, C.byref(n)))
            return [rows[i].as_dict() for i in range(n.value)]
        finally:
            if own:
                dev.free()


    def precision_bins(self, dev: DeviceReady, scales, nb: int) -> dict:
        """Bin forms of the precision study (fbls_precision_bins): mismatches
        of the f32 and double-single bin products against the fold's f64
        product, and of the double-single form with its exact fallback."""
        sc = _f64(scales)
        out = (C.c_uint64 * 5)()
        self._check(self.lib.fbls_precision_bins(self.ctx, dev.handle, _dptr(sc), sc.shape[0], int(nb), out))
        keys = ("pairs", "f32_mismatches", "double_single_mismatches", "fallbacks", "fallback_mismatches")
        return {k: int(v) for k, v in zip(keys, out)}

    def compare_batch(self, candidates: Sequence[Tuple[FamilyState, float]], cfg: SearchConfig,
                      devs: Optional[Sequence[DeviceReady]] = None) -> List[List[dict]]:
        """Evidence rows of many (family, period) candidates in one batch
        (fbls_compare_batch): for each candidate the rows compare_search gives.
        devs: the families already uploaded (one per candidate), else each
        distinct family is uploaded for the call."""
        uploaded: List[DeviceReady] = []
        try:
            if devs is None:
                seen = {}
                devs = []
                for st, _ in candidates:
                    if id(st) not in seen:
                        seen[id(st)] = self.upload(st)
                        uploaded.append(seen[id(st)])
                    devs.append(seen[id(st)])
            c, keep = _config(cfg)
            jobs = (N.EvidenceJob * max(1, len(candidates)))()
            arrays = []
            for i, ((st, period), dev) in enumerate(zip(candidates, devs)):
                d, r = _f64(st.durations), _f64(st.rho)
                arrays.append((d, r))
                jobs[i].ready = dev.handle
                jobs[i].period = float(period)
                jobs[i].durations = _dptr(d)
                jobs[i].rho = _dptr(r)
                jobs[i].nd = len(d)
            self._check(self.lib.fbls_compare_batch(self.ctx, jobs, len(candidates), C.byref(c)))
            return [[jobs[i].rows[k].as_dict() for k in range(jobs[i].n_rows)] for i in range(len(candidates))]
        finally:
            for dev in uploaded:
                dev.free()


def _grid_count(state: FamilyState, cfg: SearchConfig) -> int:
    """Length of the period grid signal_search scans (an upper bound on its rows)."""
    dmin = float(np.min(state.durations))
    baseline = float(state.time[-1])
    maximum = min(cfg.period_max, baseline)
    minimum = max(cfg.period_min, 4.0 * dmin * (1.0 + 1e-9))
    if maximum <= minimum:
        return 0
    return int(N.load().fbls_period_grid(minimum, maximum, baseline, dmin, cfg.period_oversample, None, 0))


def _rows_array(rows, n: int) -> np.ndarray:
    if n == 0:
        return np.zeros((0, 5))
    buf = np.ctypeslib.as_array(C.cast(rows, N.c_double_p), shape=(n * 5,))
    return buf.reshape(n, 5).copy()


def band_plan(state: FamilyState, cfg: SearchConfig) -> Tuple[np.ndarray, List[dict]]:
    """The grid and octave bands signal_search scans (scan.rs:418-471):
    (grid, [{periods, durations, rho, nb}])."""
    order = np.argsort(state.durations, kind="stable")
    ds = state.durations[order]
    rs = state.rho[order]
    baseline = float(state.time[-1])
    maximum = min(cfg.period_max, baseline)
    minimum = max(cfg.period_min, 4.0 * ds[0] * (1.0 + 1e-9))
    if maximum <= minimum:
        return np.zeros(0), []
    grid = period_grid(minimum, maximum, baseline, float(ds[0]), cfg.period_oversample)
    bands = []
    lo = grid[0]
    last = grid[-1]
    while lo <= last:
        hi = lo * 2.0
        sel = grid[(grid >= lo) & (grid < hi)]
        chosen = ds < lo / 4.0
        if sel.size and chosen.any():
            d = ds[chosen]
            nb = max(8, int(math.ceil(cfg.phase_oversample * sel[-1] / d.min())))
            bands.append({"periods": sel, "durations": d, "rho": rs[chosen], "nb": nb})
        lo = hi
    return grid, bands


def bank_for(band: dict, cfg: SearchConfig) -> Bank:
    """The Bank signal_search builds for one band (scan.rs:453-465)."""
    gate = cfg.shape_gate_fraction * cfg.threshold if cfg.ingress_fractions[0] == 0.0 else 0.0
    return Bank(durations=band["durations"], rho=band["rho"], ingress=tuple(cfg.ingress_fractions),
                layers=cfg.shape_layers, threshold=cfg.threshold, shape_gate=gate,
                phase_oversample=cfg.phase_oversample, period_batch=cfg.period_batch,
                max_fold_mib=cfg.max_fold_mib, prescan_factor=cfg.prescan_factor,
                prescan_fraction=cfg.prescan_fraction)
