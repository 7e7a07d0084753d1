"""Seeded synthetic light curves for the workloads the path is measured on.

The reference validates on real TESS curves that are not available here; the
workloads below stand in for them with the shapes, sizes and value
distributions of the configurations the path is specified on:

  single_sector  one 27.4 d sector at 120 s with a 1 d mid-sector gap
                 (~19k points), white noise 1e-3, one box at P = 3.7 d,
                 1500 ppm, 2.5 h; 12 durations log-spaced 0.5-12 h;
                 periods 0.5-13.7 d.
  multi_sector   13 contiguous 27.4 d sectors at 120 s, each with a 1 d gap
                 (~250k points), white 8e-4 plus AR(1) red noise (rho 0.95,
                 sigma 3e-4), one box at P = 17.3 d, 400 ppm, 5 h;
                 20 durations 0.5-15 h; periods 0.5-20 d.
  survey_star    one star of the batched population: geometric(0.4) sectors
                 capped at 13, cadence in {120, 200, 600} s, white noise
                 log-uniform 2e-4-5e-3 plus AR(1) (rho 0.9), a box on 30%.
  survey_star_full  the survey-scale batch's star: the same population with
                 a box on 8% and an eclipsing-binary-like pair (primary and
                 secondary at phase 0.5, unequal depths 1-20%) on 2%.

Flux is returned as relative flux (transits negative) with flux_err, the
prepared-mode input of the reference (pipeline.rs:41-68).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

from .config import SearchConfig

SECTOR_DAYS = 27.4
GAP_DAYS = 1.0
T0 = 2458000.0  # an arbitrary BJD origin


@dataclasses.dataclass
class Curve:
    time: np.ndarray
    flux: np.ndarray
    flux_err: np.ndarray
    period: Optional[float] = None     # injected period (days)
    epoch: Optional[float] = None      # injected mid-transit time (BJD)
    depth: Optional[float] = None      # injected depth (relative)
    duration: Optional[float] = None   # injected duration (days)
    label: str = ""


def sector_times(sectors: int, cadence_s: float, start: float = T0) -> np.ndarray:
    """Contiguous sectors of 27.4 d with a 1 d gap at mid-sector."""
    step = cadence_s / 86400.0
    per = int(round(SECTOR_DAYS / step))
    base = np.arange(per) * step
    half = SECTOR_DAYS / 2.0
    keep = ~((base >= half - GAP_DAYS / 2.0) & (base < half + GAP_DAYS / 2.0))
    one = base[keep]
    return np.concatenate([start + s * SECTOR_DAYS + one for s in range(sectors)])


def _ar1_fast(rng: np.random.Generator, n: int, rho: float, sigma: float) -> np.ndarray:
    """Stationary AR(1) series x_t = rho x_(t-1) + e_t with marginal standard
    deviation sigma, evaluated in short blocks with the closed form
    x_t = rho^t x_0 + sum_k rho^(t-k) e_k (blocks keep rho^-t well scaled)."""
    e = rng.normal(0.0, sigma * math.sqrt(1.0 - rho * rho), n)
    out = np.empty(n)
    x = rng.normal(0.0, sigma)
    block = 64
    powers = rho ** np.arange(1, block + 1)
    for s in range(0, n, block):
        seg = e[s:s + block]
        m = seg.shape[0]
        scaled = seg / powers[:m]
        acc = np.cumsum(scaled) * powers[:m]
        out[s:s + m] = acc + powers[:m] * x
        x = out[s + m - 1]
    return out


def inject_box(time: np.ndarray, flux: np.ndarray, period: float, epoch: float, duration: float,
               depth: float) -> np.ndarray:
    phase = np.remainder(time - epoch + 0.5 * period, period) - 0.5 * period
    out = flux.copy()
    out[np.abs(phase) <= duration / 2.0] -= depth
    return out


def single_sector(seed: int = 1) -> Curve:
    rng = np.random.default_rng(seed)
    t = sector_times(1, 120.0)
    sigma = 1e-3
    flux = rng.normal(0.0, sigma, t.shape[0])
    period, depth, duration = 3.7, 1500e-6, 2.5 / 24.0
    epoch = T0 + rng.uniform(0.0, period)
    flux = inject_box(t, flux, period, epoch, duration, depth)
    return Curve(t, flux, np.full_like(t, sigma), period, epoch, depth, duration, "single_sector")


def multi_sector(seed: int = 2, sectors: int = 13) -> Curve:
    rng = np.random.default_rng(seed)
    t = sector_times(sectors, 120.0)
    n = t.shape[0]
    flux = rng.normal(0.0, 8e-4, n) + _ar1_fast(rng, n, 0.95, 3e-4)
    period, depth, duration = 17.3, 400e-6, 5.0 / 24.0
    epoch = T0 + rng.uniform(0.0, period)
    flux = inject_box(t, flux, period, epoch, duration, depth)
    err = np.full(n, math.sqrt(8e-4 ** 2 + 3e-4 ** 2))
    return Curve(t, flux, err, period, epoch, depth, duration, "multi_sector")


def survey_star(rng: np.random.Generator, inject_fraction: float = 0.3) -> Curve:
    sectors = min(int(rng.geometric(0.4)), 13)
    cadence = float(rng.choice([120.0, 200.0, 600.0]))
    t = sector_times(sectors, cadence, start=T0 + rng.uniform(0.0, 10.0))
    n = t.shape[0]
    sigma = math.exp(rng.uniform(math.log(2e-4), math.log(5e-3)))
    flux = rng.normal(0.0, sigma, n) + _ar1_fast(rng, n, 0.9, 0.3 * sigma)
    c = Curve(t, flux, np.full(n, sigma), label=f"{sectors}x{int(cadence)}s")
    if rng.uniform() < inject_fraction:
        baseline = t[-1] - t[0]
        pmax = min(20.0, baseline / 2.0)
        period = math.exp(rng.uniform(math.log(0.5), math.log(pmax)))
        depth = math.exp(rng.uniform(math.log(100e-6), math.log(1e-2)))
        # Duration at solar density: 13 h (P / 365 d)^(1/3), times U(0.5, 2).
        duration = 13.0 / 24.0 * (period / 365.25) ** (1.0 / 3.0) * rng.uniform(0.5, 2.0)
        epoch = t[0] + rng.uniform(0.0, period)
        c.flux = inject_box(t, flux, period, epoch, duration, depth)
        c.period, c.epoch, c.depth, c.duration = period, epoch, depth, duration
    return c


def inject_pair(time: np.ndarray, flux: np.ndarray, period: float, epoch: float, duration: float,
                primary: float, secondary: float) -> np.ndarray:
    """An eclipsing-binary-like pair: a primary box at epoch and a secondary
    box half a period later, of depths `primary` and `secondary`."""
    out = inject_box(time, flux, period, epoch, duration, primary)
    return inject_box(time, out, period, epoch + 0.5 * period, duration, secondary)


def survey_star_full(rng: np.random.Generator, box_fraction: float = 0.08, pair_fraction: float = 0.02) -> Curve:
    """One star of the survey-scale batch: the batching population (as
    survey_star) with a box on `box_fraction` of the stars and an
    eclipsing-binary-like pair on `pair_fraction`: primary and secondary boxes
    at phases 0 and 0.5 with unequal depths, each log-uniform in 1-20 %
    (redrawn until they differ by at least 10 %), period log-uniform 0.5 d to
    min(20 d, baseline / 2), duration as for the boxes."""
    c = survey_star(rng, inject_fraction=0.0)
    u = rng.uniform()
    baseline = c.time[-1] - c.time[0]
    pmax = min(20.0, baseline / 2.0)
    period = math.exp(rng.uniform(math.log(0.5), math.log(pmax)))
    duration = 13.0 / 24.0 * (period / 365.25) ** (1.0 / 3.0) * rng.uniform(0.5, 2.0)
    epoch = c.time[0] + rng.uniform(0.0, period)
    if u < box_fraction:
        depth = math.exp(rng.uniform(math.log(100e-6), math.log(1e-2)))
        c.flux = inject_box(c.time, c.flux, period, epoch, duration, depth)
        c.period, c.epoch, c.depth, c.duration, c.label = period, epoch, depth, duration, c.label + " box"
    elif u < box_fraction + pair_fraction:
        while True:
            d1, d2 = (math.exp(rng.uniform(math.log(0.01), math.log(0.2))) for _ in range(2))
            if abs(d1 - d2) >= 0.1 * max(d1, d2):
                break
        c.flux = inject_pair(c.time, c.flux, period, epoch, duration, d1, d2)
        c.period, c.epoch, c.depth, c.duration = period, epoch, max(d1, d2), duration
        c.label += f" pair {d1:.3f}/{d2:.3f}"
    return c


def single_sector_config() -> SearchConfig:
    """Search configuration of the single-sector workload (prepared mode)."""
    d = [0.5 * 24.0 ** (i / 11.0) for i in range(12)]
    return SearchConfig(period_min=0.5, period_max=13.7, durations_hours=d)


def multi_sector_config() -> SearchConfig:
    """Search configuration of the 13-sector workload (prepared mode)."""
    d = [0.5 * 30.0 ** (i / 19.0) for i in range(20)]
    return SearchConfig(period_min=0.5, period_max=20.0, durations_hours=d)


def survey_config(curve: Curve) -> SearchConfig:
    d = [0.5 * 30.0 ** (i / 19.0) for i in range(20)]
    baseline = float(curve.time[-1] - curve.time[0])
    return SearchConfig(period_min=0.5, period_max=min(20.0, baseline / 2.0), durations_hours=d)


def small_curve(seed: int = 3, days: float = 6.0, cadence_s: float = 600.0, sigma: float = 1e-3,
                period: float = 1.3, depth: float = 3e-3, duration: float = 2.0 / 24.0) -> Curve:
    """A few-day curve for fast parity tests (the oracle runs it in seconds)."""
    rng = np.random.default_rng(seed)
    step = cadence_s / 86400.0
    t = T0 + np.arange(int(days / step)) * step
    gap = (t - T0 > days * 0.45) & (t - T0 < days * 0.45 + 0.3)
    t = t[~gap]
    flux = rng.normal(0.0, sigma, t.shape[0])
    epoch = T0 + rng.uniform(0.0, period)
    flux = inject_box(t, flux, period, epoch, duration, depth)
    return Curve(t, flux, np.full_like(t, sigma), period, epoch, depth, duration, "small")


def small_config() -> SearchConfig:
    return SearchConfig(period_min=0.4, period_max=2.9, durations_hours=[0.75, 1.2, 2.0, 3.0])
