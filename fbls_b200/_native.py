"""ctypes binding of the C ABI declared in include/fbls_b200.h.

The library is built in-tree (fbls_b200/lib/libfbls_b200.so). There is no
fallback: if the library is missing or fails to load, importing the compute
API raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libfbls_b200.so"

c_double_p = C.POINTER(C.c_double)
c_uint32_p = C.POINTER(C.c_uint32)
c_uint64_p = C.POINTER(C.c_uint64)


class Bank(C.Structure):
    _fields_ = [
        ("durations", c_double_p),
        ("rho", c_double_p),
        ("nd", C.c_uint32),
        ("ingress", c_double_p),
        ("ns", C.c_uint32),
        ("layers", C.c_uint32),
        ("threshold", C.c_double),
        ("shape_gate", C.c_double),
        ("phase_oversample", C.c_uint32),
        ("period_batch", C.c_uint32),
        ("max_fold_mib", C.c_double),
        ("prescan_factor", C.c_uint32),
        ("prescan_fraction", C.c_double),
    ]


class Row(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("period", "epoch", "duration", "score", "depth")]


class Star(C.Structure):
    _fields_ = [
        ("ready", C.c_void_p),
        ("time", C.POINTER(C.c_double)),
        ("v", C.POINTER(C.c_double)),
        ("w", C.POINTER(C.c_double)),
        ("n", C.c_uint32),
        ("baseline_norm", C.c_double),
        ("origin", C.c_double),
        ("residual_energy", C.c_double),
        ("durations", C.POINTER(C.c_double)),
        ("rho", C.POINTER(C.c_double)),
        ("nd", C.c_uint32),
        ("period_max", C.c_double),
        ("rows", C.POINTER(Row)),
        ("capacity", C.c_uint32),
        ("n_rows", C.c_uint32),
        ("grid_len", C.c_uint64),
        ("templates", C.c_uint64),
        ("status", C.c_int),
        ("ranges", C.POINTER(C.c_double)),
        ("n_ranges", C.c_uint32),
    ]


class MapJob(C.Structure):
    _fields_ = [
        ("ready", C.c_void_p),
        ("periods", C.POINTER(C.c_double)),
        ("P", C.c_uint32),
        ("durations", C.POINTER(C.c_double)),
        ("rho", C.POINTER(C.c_double)),
        ("nd", C.c_uint32),
        ("oversample", C.c_double),
        ("bin_days", C.c_double),
        ("out", C.POINTER(C.c_float)),
        ("status", C.c_int),
    ]


class ScanStats(C.Structure):
    _fields_ = [
        ("periods", C.c_uint64),
        ("prescan_survivors", C.c_uint64),
        ("phase_bins", C.c_uint64),
        ("batches", C.c_uint64),
        ("templates_scanned", C.c_uint64),
        ("exact_tile_retries", C.c_uint64),
        ("tile_rescans", C.c_uint64),
        ("seconds", C.c_double),
        ("seconds_fold", C.c_double),
        ("seconds_cumulative", C.c_double),
        ("seconds_scan", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Config(C.Structure):
    _fields_ = [
        ("period_min", C.c_double),
        ("period_max", C.c_double),
        ("threshold", C.c_double),
        ("ingress_fractions", c_double_p),
        ("n_ingress", C.c_uint32),
        ("shape_layers", C.c_uint32),
        ("phase_oversample", C.c_uint32),
        ("shape_gate_fraction", C.c_double),
        ("prescan_factor", C.c_uint32),
        ("prescan_fraction", C.c_double),
        ("period_oversample", C.c_double),
        ("period_batch", C.c_uint32),
        ("max_fold_mib", C.c_double),
        ("evidence_rtol", C.c_double),
        ("planet_prior", C.c_double),
        ("binary_prior", C.c_double),
        ("planet_depth_scale", C.c_double),
        ("binary_depth_scale", C.c_double),
        ("diluted_binary_depth_scale", C.c_double),
        ("stellar_radius_solar", C.c_double),
        ("planet_radius_scale_rj", C.c_double),
        ("target_flux_fraction", C.c_double),
        ("precision_mode", C.c_uint32),
    ]


class EvidenceRow(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "period", "epoch", "duration", "snr", "depth", "planet_log_odds", "log_bf_planet_noise",
        "log_bf_binary_noise", "binary_secondary_ratio", "binary_secondary_phase", "binary_odd_even_ratio",
        "binary_period_days", "ingress_fraction")] + [("selection_flags", C.c_uint32)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class EvidenceJob(C.Structure):
    _fields_ = [("ready", C.c_void_p), ("period", C.c_double), ("durations", C.POINTER(C.c_double)),
                ("rho", C.POINTER(C.c_double)), ("nd", C.c_uint32), ("rows", EvidenceRow * 2),
                ("n_rows", C.c_uint32), ("status", C.c_int)]


class Tuning(C.Structure):
    _fields_ = [("fold_group_max", C.c_uint32 * 32), ("launch_periods", C.c_uint32), ("fold_steal", C.c_uint32),
                ("fold_threads", C.c_uint32 * 32), ("lockstep_min", C.c_uint32 * 32), ("fused_scan", C.c_uint32),
                ("map_lockstep_min", C.c_uint32), ("fold_pair", C.c_uint32 * 32), ("map_threads", C.c_uint32),
                ("map_group_max", C.c_uint32), ("batch_no_fill", C.c_uint32)]


class PrepConfig(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("bin_minutes", "window_min", "window_factor", "window_max", "clip_sigma",
                                           "edge_trim")]


class FamilyOut(C.Structure):
    _fields_ = [("time", C.POINTER(C.c_double)), ("flux", C.POINTER(C.c_double)), ("sigma", C.POINTER(C.c_double)),
                ("n", C.c_uint32), ("window_days", C.c_double), ("clipped", C.c_uint32),
                ("indices", C.POINTER(C.c_uint32)), ("n_indices", C.c_uint32)]


class EventStats(C.Structure):
    _fields_ = [("templates_scanned", C.c_uint64), ("threshold_survivors", C.c_uint64), ("overflow", C.c_int)]

    def as_dict(self) -> dict:
        return {"templates_scanned": int(self.templates_scanned),
                "threshold_survivors": int(self.threshold_survivors), "overflow": bool(self.overflow)}


class Counters(C.Structure):
    _fields_ = [
        ("launches", C.c_uint64),
        ("fold_launches", C.c_uint64),
        ("fold_ms", C.c_double),
        ("fold_bytes", C.c_double),
        ("scan_launches", C.c_uint64),
        ("scan_ms", C.c_double),
        ("scan_bytes", C.c_double),
        ("fold_updates", C.c_uint64),
        ("rescore_launches", C.c_uint64),
        ("rescore_ms", C.c_double),
        ("detrend_ms", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


# Every entry point declared in include/fbls_b200.h: name -> (restype, argtypes).
SIGNATURES = {
    "fbls_version": (C.c_char_p, []),
    "fbls_create": (C.c_void_p, [C.c_int, C.POINTER(C.c_int)]),
    "fbls_destroy": (None, [C.c_void_p]),
    "fbls_last_error": (C.c_char_p, [C.c_void_p]),
    "fbls_upload_ready": (C.c_int, [C.c_void_p, c_double_p, c_double_p, c_double_p, C.c_uint32, C.c_double,
                                    C.c_double, C.c_double, C.POINTER(C.c_void_p)]),
    "fbls_free_ready": (None, [C.c_void_p]),
    "fbls_scan_periods": (C.c_int, [C.c_void_p, C.c_void_p, c_double_p, C.c_uint32, C.POINTER(Bank), C.c_uint32,
                                    C.POINTER(Row), c_uint32_p, C.POINTER(ScanStats)]),
    "fbls_scan_bank": (C.c_int, [C.c_void_p, C.c_void_p, c_double_p, C.c_uint32, C.POINTER(Bank), C.c_uint32,
                                 C.c_uint32, c_double_p, c_double_p, c_double_p, c_uint32_p,
                                 C.POINTER(ScanStats)]),
    "fbls_compare_search": (C.c_int, [C.c_void_p, C.c_void_p, c_double_p, c_double_p, C.c_uint32, C.c_double,
                                      C.POINTER(Config), C.POINTER(EvidenceRow), c_uint32_p]),
    "fbls_compare_batch": (C.c_int, [C.c_void_p, C.POINTER(EvidenceJob), C.c_uint32, C.POINTER(Config)]),
    "fbls_scan_bank_static": (C.c_int, [C.c_int, c_double_p, c_double_p, c_double_p, C.c_uint32, C.c_double,
                                        c_double_p, C.c_uint32, C.POINTER(Bank), C.c_uint32, C.c_uint32,
                                        c_double_p, c_double_p, c_double_p, c_uint32_p, C.c_char_p,
                                        C.c_uint32]),
    "fbls_set_tuning": (C.c_int, [C.POINTER(Tuning)]),
    "fbls_get_tuning": (C.c_int, [C.POINTER(Tuning)]),
    "fbls_precision_bins": (C.c_int, [C.c_void_p, C.c_void_p, c_double_p, C.c_uint32, C.c_uint32,
                                      C.POINTER(C.c_uint64)]),
    "fbls_timer_start": (C.c_int, [C.c_void_p]),
    "fbls_timer_stop": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "fbls_set_kernel_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "fbls_read_counters": (C.c_int, [C.c_void_p, C.POINTER(Counters), C.c_int]),
    "fbls_period_grid": (C.c_int64, [C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, c_double_p,
                                     C.c_int64]),
    "fbls_family_state": (C.c_int, [c_double_p, c_double_p, c_double_p, C.c_uint32, c_double_p, C.c_uint32, C.c_int,
                                    c_uint32_p, c_double_p, c_double_p, c_double_p, c_double_p, c_double_p,
                                    C.c_char_p, C.c_uint32]),
    "fbls_signal_search": (C.c_int, [C.c_void_p, C.c_void_p, c_double_p, c_double_p, C.c_uint32,
                                     C.POINTER(Config), C.POINTER(Row), C.c_uint32, c_uint32_p, c_uint64_p,
                                     C.POINTER(ScanStats), c_uint32_p]),
    "fbls_signal_search_ranges": (C.c_int, [C.c_void_p, C.c_void_p, c_double_p, c_double_p, C.c_uint32,
                                            C.POINTER(Config), c_double_p, C.c_uint32, C.POINTER(Row), C.c_uint32,
                                            c_uint32_p, c_uint64_p, C.POINTER(ScanStats), c_uint32_p]),
    "fbls_search_batch": (C.c_int, [C.c_void_p, C.POINTER(Star), C.c_uint32, C.POINTER(Config), C.c_uint32]),
    "fbls_coarse_map": (C.c_int, [C.c_void_p, C.c_void_p, c_double_p, C.c_uint32, c_double_p, c_double_p, C.c_uint32,
                                  C.c_double, C.c_double, C.POINTER(C.c_float)]),
    "fbls_coarse_map_batch": (C.c_int, [C.c_void_p, C.POINTER(MapJob), C.c_uint32, C.c_uint32]),
    "fbls_coarse_features": (C.c_int, [C.c_void_p, C.POINTER(MapJob), C.c_uint32, c_uint32_p, C.c_uint32,
                                       C.c_uint32, C.POINTER(C.c_float)]),
    "fbls_fit_segment_noise": (C.c_int, [c_double_p, c_double_p, c_double_p, C.POINTER(C.c_int64), C.c_uint32,
                                         C.c_double, C.c_double, c_uint32_p, c_double_p, c_double_p, c_double_p,
                                         C.POINTER(C.c_int64), c_double_p, C.c_char_p, C.c_uint32]),
    "fbls_segment_edges": (C.c_int, [c_double_p, C.c_uint32, C.c_double, c_double_p]),
    "fbls_detrending_windows": (C.c_int, [c_double_p, C.c_uint32, C.c_double, C.c_double, C.c_double, c_double_p,
                                          c_uint32_p, c_uint32_p]),
    "fbls_prepare_families": (C.c_int, [C.c_void_p, c_double_p, c_double_p, c_double_p, C.POINTER(C.c_int64),
                                        C.c_uint32, c_double_p, C.c_uint32, C.POINTER(PrepConfig),
                                        C.POINTER(FamilyOut), c_uint32_p]),
    "fbls_biweight_flatten": (C.c_int, [C.c_void_p, c_double_p, c_double_p, C.c_uint32, C.c_double, C.c_double,
                                        C.c_double, C.c_uint32, c_double_p]),
    "fbls_single_event_search": (C.c_int, [C.c_void_p, C.c_void_p, c_double_p, c_double_p, C.c_uint32,
                                           C.POINTER(Config), C.c_uint32, C.POINTER(Row), c_uint32_p,
                                           C.POINTER(EventStats)]),
    "fbls_rescore_rows": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint8), c_double_p, C.c_uint32,
                                    c_double_p]),
    "fbls_count_rows": (C.c_int, [C.c_void_p, c_double_p, C.c_uint32, C.POINTER(C.c_uint8), c_double_p, C.c_uint32,
                                  c_uint32_p]),
    # proposal network kernels: device pointers passed as integers
    "fbls_nn_gemm": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int] + [C.c_longlong] * 9
                     + [C.c_int, C.c_float, C.c_float, C.c_void_p]),
    "fbls_nn_im2col": (C.c_int, [C.c_void_p, C.c_void_p] + [C.c_int] * 5 + [C.c_void_p]),
    "fbls_nn_col2im": (C.c_int, [C.c_void_p, C.c_void_p] + [C.c_int] * 5 + [C.c_void_p]),
    "fbls_nn_bias_relu_pool": (C.c_int, [C.c_void_p] * 4 + [C.c_int] * 4 + [C.c_void_p]),
    "fbls_nn_bias_relu_pool_bwd": (C.c_int, [C.c_void_p] * 5 + [C.c_int] * 4 + [C.c_void_p]),
    "fbls_nn_bias_gelu_pool": (C.c_int, [C.c_void_p] * 4 + [C.c_int] * 4 + [C.c_void_p]),
    "fbls_nn_bias_gelu_pool_bwd": (C.c_int, [C.c_void_p] * 6 + [C.c_int] * 4 + [C.c_void_p]),
    "fbls_nn_head": (C.c_int, [C.c_void_p] * 7 + [C.c_int] * 4 + [C.c_void_p]),
    "fbls_nn_head_bwd": (C.c_int, [C.c_void_p] * 6 + [C.c_int] * 4 + [C.c_void_p]),
    "fbls_nn_adam": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_float, C.c_float,
                               C.c_float, C.c_float, C.c_int, C.c_void_p]),
    "fbls_nn_adamw": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_float, C.c_float,
                                C.c_float, C.c_float, C.c_float, C.c_int, C.c_void_p]),
}

_lib = None


def load() -> C.CDLL:
    """Loads the native library (once). Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"fbls_b200 native library not built: {LIB_PATH} (run python -m fbls_b200.build)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
