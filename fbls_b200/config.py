"""Search configuration; mirrors SearchConfig (src/config.rs:6-139).

Times are days unless the field name says hours. Defaults are the
reference's (config.rs:45-88); validation follows config.rs:91-131.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional


def _default_durations() -> List[float]:
    # 0.5 h x 1.25^i, i = 0..12, rounded half-to-even at 1e-6 h (config.rs:50-52).
    return [round(0.5 * 1.25 ** i * 1e6) / 1e6 for i in range(13)]


@dataclasses.dataclass
class SearchConfig:
    period_min: float = 0.3
    period_max: float = 10.0
    durations_hours: List[float] = dataclasses.field(default_factory=_default_durations)
    threshold: float = 7.1
    bin_minutes: float = 10.0
    window_days: float = 0.4
    window_factor: float = 3.0
    window_max_days: float = 3.5
    edge_trim_windows: float = 0.5
    clip_sigma: float = 4.0
    correlated_noise: bool = True
    ingress_fractions: List[float] = dataclasses.field(default_factory=lambda: [0.0, 0.2, 0.45])
    shape_layers: int = 4
    phase_oversample: int = 4
    shape_gate_fraction: float = 0.6
    prescan_factor: int = 2
    prescan_fraction: float = 0.7
    period_oversample: float = 3.0
    max_candidates: int = 20
    period_batch: int = 4096
    max_fold_mib: float = 1024.0
    passes: int = 3
    min_events: int = 2
    single_events: bool = True
    model_comparison: bool = True
    evidence_candidates: int = 32
    evidence_rtol: float = 1e-12
    planet_log_odds_min: float = 0.0
    planet_prior: float = 0.01
    binary_prior: float = 0.01
    planet_depth_scale: float = 0.01
    binary_depth_scale: float = 0.1
    diluted_binary_depth_scale: float = 0.01
    stellar_radius_solar: Optional[float] = None
    planet_radius_scale_rj: float = 1.0
    target_flux_fraction: float = 1.0
    # Not in the reference: 0 = its mixed-precision scan (f32 pre-rank, f64
    # winner and rescans), 1 = f64 ranking throughout.
    precision_mode: int = 0

    def validate(self) -> None:
        """Raises ValueError with the reference's message (config.rs:91-131)."""
        if not (0.0 < self.period_min < self.period_max):
            raise ValueError("require 0 < period_min < period_max")
        if not self.durations_hours or any(not (math.isfinite(d) and d > 0.0) for d in self.durations_hours):
            raise ValueError("durations_hours must contain positive finite values")
        if min(self.durations_hours) / 24.0 >= self.period_min / 4.0:
            raise ValueError("minimum duration must be below one quarter of period_min")
        if not self.ingress_fractions or any(not (0.0 <= x < 0.5) for x in self.ingress_fractions):
            raise ValueError("ingress fractions must be in [0, 0.5)")
        if (self.shape_layers < 1 or self.phase_oversample < 1 or self.period_batch < 1 or self.passes < 1
                or self.prescan_factor < 1):
            raise ValueError("invalid integer search parameter")
        if not (0.0 < self.prescan_fraction <= 1.0):
            raise ValueError("prescan_fraction must be in (0, 1]")

    def durations_days(self) -> List[float]:
        """Sorted unique durations in days (config.rs:134-139)."""
        d = sorted(h / 24.0 for h in self.durations_hours)
        out: List[float] = []
        for x in d:
            if not out or out[-1] != x:
                out.append(x)
        return out
