"""TEST INFRASTRUCTURE: ctypes binding of the reference-code harness
(oracle/ref_harness/qkref_harness.cpp -> oracle/_ref/libqkref{64,32}.so).

These libraries are the reference's own headers compiled against the project's
host shim of Kokkos (OpenMP on the host cores).  They exist where the reference
checkout was present at build time; callers check :func:`available`.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB64 = HERE / "_ref" / "libqkref64.so"
LIB32 = HERE / "_ref" / "libqkref32.so"


class RefConfig(C.Structure):
    _fields_ = [("S0", C.c_double), ("v0", C.c_double), ("r", C.c_double), ("q", C.c_double),
                ("opt_type", C.c_int32), ("opt_right", C.c_int32), ("K", C.c_double), ("B", C.c_double),
                ("model", C.c_int32), ("scheme", C.c_int32),
                ("kappa", C.c_double), ("theta", C.c_double), ("sigma", C.c_double), ("rho", C.c_double),
                ("lambda_j", C.c_double), ("mu_j", C.c_double), ("sigma_j", C.c_double),
                ("T", C.c_double), ("dt_in", C.c_double),
                ("normalize", C.c_int32), ("n_paths", C.c_int32), ("batch_size", C.c_int32),
                ("analyze_distribution", C.c_int32),
                ("seed", C.c_uint64), ("max_vram_mb", C.c_int64), ("max_cpu_ram_mb", C.c_int64),
                ("greeks_mask", C.c_int32), ("pad_", C.c_int32),
                ("bump_S_rel", C.c_double), ("bump_vol_abs", C.c_double), ("bump_r_abs", C.c_double),
                ("bump_T_abs", C.c_double)]


class RefResult(C.Structure):
    _fields_ = [("price", C.c_double), ("std_error", C.c_double), ("prob_itm", C.c_double),
                ("pct", C.c_double * 15),
                ("delta", C.c_double), ("gamma", C.c_double), ("vega", C.c_double), ("vomma", C.c_double),
                ("vanna", C.c_double), ("rho", C.c_double), ("theta", C.c_double),
                ("n_steps", C.c_int32), ("pad_", C.c_int32), ("dt", C.c_double), ("seconds", C.c_double)]


_libs: dict[int, C.CDLL] = {}


def available() -> bool:
    return LIB64.exists() and LIB32.exists()


def lib(real_bytes: int = 8) -> C.CDLL:
    if real_bytes not in _libs:
        path = LIB64 if real_bytes == 8 else LIB32
        if not path.exists():
            raise ImportError(f"{path} not built (needs the reference checkout at build time)")
        L = C.CDLL(str(path))
        dp = C.POINTER(C.c_double)
        L.qkref_step_trace.argtypes = [C.POINTER(RefConfig), dp, dp, C.c_int, C.c_int, dp, dp, C.POINTER(C.c_int)]
        L.qkref_price.argtypes = [C.POINTER(RefConfig), C.POINTER(RefResult)]
        L.qkref_exact_call.argtypes = [C.POINTER(RefConfig), C.c_int, C.c_double, dp]
        L.qkref_lsm_solve.argtypes = [dp, dp, C.c_double, C.c_int, dp]
        L.qkref_laguerre.argtypes = [C.c_double, C.c_int, dp]
        L.qkref_payoff.argtypes = [C.c_int, C.c_int, dp, C.c_int, C.c_double, C.c_double, C.c_double, dp]
        L.qkref_last_error.restype = C.c_char_p
        L.qkref_set_threads.argtypes = [C.c_int]
        L.qkref_read_paths.argtypes = [C.c_char_p, C.c_char_p, C.c_double, dp, C.c_int, C.POINTER(C.c_int)]
        L.qkref_get_threads.restype = C.c_int
        _libs[real_bytes] = L
    return _libs[real_bytes]


def set_threads(n: int) -> None:
    """Thread count of the reference's OpenMP loops in both builds.  Its generator pool
    holds one state per thread, so a fixed count gives the same draws on any machine."""
    for rb in (8, 4):
        lib(rb).qkref_set_threads(int(n))


def get_threads() -> int:
    return int(lib(8).qkref_get_threads())


def config(**kw) -> RefConfig:
    """RefConfig with the reference's UInputs defaults (include/core/config/Config.hpp:50-623), then kw."""
    c = RefConfig(S0=100.0, v0=1.0, r=0.05, q=0.0, opt_type=0, opt_right=0, K=100.0, B=100.0, model=0, scheme=0,
                  kappa=2.0, theta=0.04, sigma=0.3, rho=-0.7, lambda_j=0.1, mu_j=-0.1, sigma_j=0.15,
                  T=1.0, dt_in=0.2, normalize=1, n_paths=1000, batch_size=0, analyze_distribution=0,
                  seed=184467440737095, max_vram_mb=256, max_cpu_ram_mb=4000, greeks_mask=0, pad_=0,
                  bump_S_rel=0.001, bump_vol_abs=0.01, bump_r_abs=1e-4, bump_T_abs=1.0 / 365.0)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def from_contract(k, **kw) -> RefConfig:
    """RefConfig equivalent of an engine contract (first payoff leg)."""
    c = config(S0=k.S0, v0=k.v0, r=k.r, q=k.q, opt_type=k.payoffs[0].type, opt_right=k.payoffs[0].right,
               K=k.payoffs[0].strike, B=k.payoffs[0].barrier, model=k.model, scheme=k.scheme, kappa=k.kappa,
               theta=k.theta, sigma=k.sigma, rho=k.rho, lambda_j=k.lambda_j, mu_j=k.mu_j, sigma_j=k.sigma_j,
               T=k.T, dt_in=k.T / k.n_steps, normalize=k.normalize, n_paths=int(k.n_paths), seed=int(k.seed))
    for a, v in kw.items():
        setattr(c, a, v)
    return c


def step_trace(real_bytes: int, cfg: RefConfig, z: np.ndarray, u: np.ndarray):
    """SDEScheme<M,S>::evolve_step with fed draws; dt = cfg.dt_in."""
    z = np.ascontiguousarray(z, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64)
    n = z.shape[0]
    S, v = np.empty(n), np.empty(n)
    used = (C.c_int * n)()
    dp = C.POINTER(C.c_double)
    rc = lib(real_bytes).qkref_step_trace(C.byref(cfg), z.ctypes.data_as(dp), u.ctypes.data_as(dp), u.shape[1], n,
                                          S.ctypes.data_as(dp), v.ctypes.data_as(dp), used)
    if rc != 0:
        raise RuntimeError(f"qkref_step_trace rc={rc}: {lib(real_bytes).qkref_last_error()}")
    return S, v, np.array(used[:])


def price(cfg: RefConfig, real_bytes: int = 8) -> dict:
    r = RefResult()
    rc = lib(real_bytes).qkref_price(C.byref(cfg), C.byref(r))
    if rc != 0:
        raise RuntimeError(f"qkref_price: {lib(real_bytes).qkref_last_error().decode()}")
    out = {f: getattr(r, f) for f, _ in RefResult._fields_ if f not in ("pct", "pad_")}
    out["pct"] = list(r.pct)
    return out


def exact_call(cfg: RefConfig, kind: int, phi_max: float = 0.0) -> float:
    p = C.c_double()
    rc = lib(8).qkref_exact_call(C.byref(cfg), kind, phi_max, C.byref(p))
    if rc != 0:
        raise RuntimeError(lib(8).qkref_last_error().decode())
    return p.value


def lsm_solve(M: np.ndarray, B: np.ndarray, count: float) -> np.ndarray:
    nb = len(B)
    M = np.ascontiguousarray(M, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    out = np.empty(nb)
    dp = C.POINTER(C.c_double)
    lib(8).qkref_lsm_solve(M.ctypes.data_as(dp), B.ctypes.data_as(dp), count, nb, out.ctypes.data_as(dp))
    return out


def laguerre(X: float, nb: int = 4, real_bytes: int = 8) -> np.ndarray:
    out = np.empty(nb)
    lib(real_bytes).qkref_laguerre(X, nb, out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def payoff(opt_type: int, right: int, S: np.ndarray, S0: float, K: float, B: float, real_bytes: int = 8) -> float:
    S = np.ascontiguousarray(S, dtype=np.float64)
    out = C.c_double()
    rc = lib(real_bytes).qkref_payoff(opt_type, right, S.ctypes.data_as(C.POINTER(C.c_double)), len(S), S0, K, B,
                                      C.byref(out))
    if rc != 0:
        raise RuntimeError("qkref_payoff")
    return out.value


def read_paths(directory: str, filename: str, t: float, max_n: int, real_bytes: int = 8) -> np.ndarray:
    """The reference's BinReader: every path's spot at time t (real units) from a .paths file."""
    out = np.empty(max_n)
    n = C.c_int()
    rc = lib(real_bytes).qkref_read_paths(directory.encode(), filename.encode(), t,
                                          out.ctypes.data_as(C.POINTER(C.c_double)), max_n, C.byref(n))
    if rc != 0:
        raise RuntimeError(f"qkref_read_paths: {lib(real_bytes).qkref_last_error().decode()}")
    return out[:n.value]
