"""ctypes binding of the C ABI declared in include/quantkos_b200.h.

The shared library is the in-tree ``libquantkos_b200.so`` built by
``python -m quantkos_b200.build``; importing this module on a machine without
it raises ImportError (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libquantkos_b200.so"

QK_MAX_PAYOFFS = 8

# status codes
QK_OK = 0
QK_ERR_INVALID_ARG = 1
QK_ERR_CUDA = 2
QK_ERR_OUT_OF_MEMORY = 3
QK_ERR_UNSUPPORTED = 4
QK_ERR_TIMEOUT = 5
QK_ERR_CAPACITY = 6
QK_ERR_NO_DEVICE = 7
QK_ERR_PARSE = 8
QK_ERR_STATE = 9
QK_ERR_CANCELLED = 10

# enums (quantkos::Implemented order)
HESTON, BATES = 0, 1
EULER, IMPLICIT_MILSTEIN, ANDERSEN_QE = 0, 1, 2
(EUROPEAN, ASIAN, BARRIER_UP_OUT, BARRIER_DOWN_OUT, BARRIER_UP_IN, BARRIER_DOWN_IN,
 LOOKBACK_FLOATING, LOOKBACK_FIXED, BINARY_CASH, BINARY_ASSET, AMERICAN) = range(11)
CALL, PUT = 0, 1
FP64, FP32 = 0, 1
LSM_LAGUERRE3, LSM_POLY_SV = 0, 1
GREEK_DELTA_GAMMA, GREEK_VEGA_VOMMA, GREEK_VANNA, GREEK_RHO, GREEK_THETA = 1, 2, 4, 8, 16
GREEK_ALL = 31


class Payoff(C.Structure):
    _fields_ = [("type", C.c_int32), ("right", C.c_int32), ("strike", C.c_double), ("barrier", C.c_double)]


class Contract(C.Structure):
    _fields_ = [
        ("S0", C.c_double), ("v0", C.c_double), ("r", C.c_double), ("q", C.c_double),
        ("model", C.c_int32), ("scheme", C.c_int32),
        ("kappa", C.c_double), ("theta", C.c_double), ("sigma", C.c_double), ("rho", C.c_double),
        ("lambda_j", C.c_double), ("mu_j", C.c_double), ("sigma_j", C.c_double),
        ("psi_c", C.c_double), ("T", C.c_double),
        ("n_steps", C.c_int32), ("normalize", C.c_int32),
        ("n_paths", C.c_int64), ("seed", C.c_uint64), ("stream", C.c_uint64),
        ("precision", C.c_int32), ("n_payoffs", C.c_int32),
        ("payoffs", Payoff * QK_MAX_PAYOFFS),
        ("lsm_basis", C.c_int32), ("lsm_dates", C.c_int32),
        ("antithetic", C.c_int32), ("reserved_", C.c_int32),
    ]


class Greeks(C.Structure):
    _fields_ = [("mask", C.c_int32), ("vega_mode", C.c_int32), ("bump_S_rel", C.c_double),
                ("bump_vol", C.c_double), ("bump_r_abs", C.c_double), ("bump_T_abs", C.c_double)]


class PayoffResult(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("price", "std_error", "prob_itm", "delta", "gamma", "vega", "vomma", "vanna", "rho", "theta")]


class Result(C.Structure):
    _fields_ = [("status", C.c_int32), ("n_payoffs", C.c_int32), ("n_paths", C.c_int64),
                ("path_steps", C.c_double), ("p", PayoffResult * QK_MAX_PAYOFFS)]


class Timing(C.Structure):
    _fields_ = [("device_ms", C.c_double), ("paths_ms", C.c_double), ("reduce_ms", C.c_double),
                ("launches", C.c_int64), ("path_steps", C.c_double), ("h2d_bytes", C.c_int64),
                ("d2h_bytes", C.c_int64)]


TUNE_KINDS = 12


class TuneReport(C.Structure):
    _fields_ = [("n_kinds", C.c_int32), ("precision", C.c_int32 * TUNE_KINDS), ("model", C.c_int32 * TUNE_KINDS),
                ("scheme", C.c_int32 * TUNE_KINDS), ("tiles_per_warp", C.c_int32 * TUNE_KINDS),
                ("guided_tail", C.c_int32 * TUNE_KINDS), ("paths_per_lane", C.c_int32 * TUNE_KINDS),
                ("best_ms", C.c_double * TUNE_KINDS),
                ("default_ms", C.c_double * TUNE_KINDS), ("candidates", C.c_int32),
                ("block_size", C.c_int32 * TUNE_KINDS)]


class ServeStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("rejected", C.c_int64),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("p999_ms", C.c_double), ("max_ms", C.c_double),
                ("contracts_per_s", C.c_double), ("path_steps_per_s", C.c_double),
                ("batches", C.c_int64), ("busy_s", C.c_double), ("reserved_mib", C.c_int64)]


class Config(C.Structure):
    _fields_ = [
        ("S0", C.c_double), ("v0", C.c_double), ("r", C.c_double), ("q", C.c_double),
        ("opt_type", C.c_int32), ("opt_right", C.c_int32), ("K", C.c_double), ("B", C.c_double),
        ("model", C.c_int32),
        ("heston_k", C.c_double), ("heston_theta", C.c_double), ("heston_sigma", C.c_double), ("heston_rho", C.c_double),
        ("bates_k", C.c_double), ("bates_theta", C.c_double), ("bates_sigma", C.c_double), ("bates_rho", C.c_double),
        ("bates_lambda", C.c_double), ("bates_mu", C.c_double), ("bates_sigma_j", C.c_double),
        ("scheme", C.c_int32),
        ("t_end", C.c_double), ("inp_dt", C.c_double), ("dt", C.c_double),
        ("n_steps", C.c_int32), ("normalize", C.c_int32), ("n_paths", C.c_int32), ("batch_size", C.c_int32),
        ("seed", C.c_uint64), ("max_vram_mb", C.c_int64), ("max_cpu_ram_mb", C.c_int64),
        ("analyze_distribution", C.c_int32), ("greeks_mask", C.c_int32),
        ("bump_S_rel", C.c_double), ("bump_vol_abs", C.c_double), ("bump_r_abs", C.c_double), ("bump_T_abs", C.c_double),
        ("verbosity", C.c_int32), ("format", C.c_int32),
        ("out_dir", C.c_char * 256), ("paths_file", C.c_char * 256), ("log_file", C.c_char * 256),
        ("precision", C.c_int32), ("engine", C.c_int32), ("lsm_basis", C.c_int32), ("lsm_dates", C.c_int32),
        ("vega_mode", C.c_int32), ("stream", C.c_uint64), ("antithetic", C.c_int32), ("reserved_", C.c_int32),
    ]


class ServeRecord(C.Structure):
    _fields_ = [("ticket", C.c_int64), ("wave", C.c_int64), ("lane", C.c_int32), ("wave_requests", C.c_int32),
                ("submit_s", C.c_double), ("admit_ms", C.c_double), ("latency_ms", C.c_double),
                ("wave_ms", C.c_double), ("wave_est_ms", C.c_double), ("est_ms", C.c_double)]


class ServeOptions(C.Structure):
    _fields_ = [("hbm_budget_mib", C.c_int64), ("max_batch", C.c_int32), ("lanes", C.c_int32), ("wave_ms", C.c_double),
                ("reserve_mib", C.c_int64), ("plain_fp64", C.c_int32), ("pad_", C.c_int32)]


_P = C.POINTER
_VP = C.c_void_p

# name -> (restype, argtypes); every symbol declared in include/quantkos_b200.h
SIGNATURES = {
    "qk_version": (C.c_char_p, []),
    "qk_last_error": (C.c_char_p, []),
    "qk_create": (C.c_int, [C.c_int32, _P(_VP)]),
    "qk_destroy": (C.c_int, [_VP]),
    "qk_get_stream": (C.c_int, [_VP, _P(_VP)]),
    "qk_last_timing": (C.c_int, [_VP, _P(Timing)]),
    "qk_autotune": (C.c_int, [_VP, _P(Contract), C.c_int32, _P(Greeks), C.c_int32, _P(TuneReport)]),
    "qk_tune_set": (C.c_int, [_VP, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "qk_tune_set_block": (C.c_int, [_VP, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "qk_tune_reset": (C.c_int, [_VP]),
    "qk_measure_sfu": (C.c_int, [_VP, _P(C.c_double)]),
    "qk_validate": (C.c_int, [_P(Contract), _P(Greeks)]),
    "qk_price_plain": (C.c_int, [_VP, _P(Contract), _P(Greeks), _P(Result)]),
    "qk_price_batch": (C.c_int, [_VP, _P(Contract), C.c_int32, _P(Greeks), _P(Result)]),
    "qk_batch_prepare": (C.c_int, [_VP, _P(Contract), C.c_int32, _P(Greeks)]),
    "qk_batch_run": (C.c_int, [_VP]),
    "qk_batch_fetch": (C.c_int, [_VP, _P(Result), C.c_int32]),
    "qk_price_noalloc": (C.c_int, [_P(Contract), _VP, _P(Result)]),
    "qk_payoff_trace": (C.c_int, [_P(Payoff), _P(C.c_double), C.c_int32, C.c_double, C.c_int32, _P(C.c_double)]),
    "qk_payoffs_range": (C.c_int, [_VP, _P(Contract), C.c_int64, C.c_int64, _P(C.c_double)]),
    "qk_lsm_date": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int64, _P(C.c_double),
                              _P(C.c_double), _P(C.c_double), C.c_double, C.c_double, C.c_double, C.c_double,
                              _P(C.c_double), _P(C.c_int32)]),
    "qk_lsm_solve": (C.c_int, [C.c_int32, _P(C.c_double), _P(C.c_double), _P(C.c_int32)]),
    "qk_paths_write": (C.c_int, [C.c_char_p, C.c_int32, C.c_int64, C.c_int32, C.c_double, C.c_double,
                                 _P(C.c_double)]),
    "qk_step_trace": (C.c_int, [C.c_int32, _P(Contract), _P(C.c_double), _P(C.c_double), C.c_int32, C.c_int32,
                                _P(C.c_double), _P(C.c_double)]),
    "qk_paths_dump": (C.c_int, [_VP, _P(Contract), C.c_int64, C.c_int64, _P(C.c_double), _P(C.c_double)]),
    "qk_config_default": (C.c_int, [_P(Config)]),
    "qk_config_parse_file": (C.c_int, [C.c_char_p, _P(Config)]),
    "qk_config_parse_string": (C.c_int, [C.c_char_p, _P(Config)]),
    "qk_config_validate": (C.c_int, [_P(Config)]),
    "qk_config_to_contract": (C.c_int, [_P(Config), _P(Contract), _P(Greeks)]),
    "qk_run_config": (C.c_int, [_VP, _P(Config), _P(Result), _P(C.c_double)]),
    "qk_serve_start": (C.c_int, [_VP, C.c_int64, C.c_int32, _P(_VP)]),
    "qk_serve_start_ex": (C.c_int, [_VP, _P(ServeOptions), _P(_VP)]),
    "qk_serve_records": (C.c_int, [_VP, _P(ServeRecord), C.c_int64, _P(C.c_int64)]),
    "qk_serve_submit": (C.c_int, [_VP, _P(Contract), _P(Greeks), _P(C.c_int64)]),
    "qk_serve_poll": (C.c_int, [_VP, C.c_int64, C.c_int32, _P(C.c_int32), _P(Result)]),
    "qk_serve_cancel": (C.c_int, [_VP, C.c_int64, _P(C.c_int32)]),
    "qk_serve_stats_get": (C.c_int, [_VP, _P(ServeStats)]),
    "qk_serve_stop": (C.c_int, [_VP]),
}


def load(path: Path | str | None = None) -> C.CDLL:
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"{p} is not built; run `python -m quantkos_b200.build` (no CPU fallback exists)")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = load()
    return _lib
