"""TEST INFRASTRUCTURE: ctypes binding of the C oracle (oracle/qk_oracle.c).

Contract / Greeks / Result structures are the engine's public C layouts
(include/quantkos_b200.h), re-declared here so the oracle does not depend on the
engine package.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libqkoracle.so"
QK_MAX_PAYOFFS = 8


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


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} not built (python -m quantkos_b200.build)")
        L = C.CDLL(str(LIB_PATH))
        dp = C.POINTER(C.c_double)
        L.qko_philox.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.qko_step_trace.argtypes = [C.c_int, C.POINTER(Contract), dp, dp, C.c_int, C.c_int, dp, dp]
        L.qko_paths.argtypes = [C.POINTER(Contract), C.c_int64, C.c_int64, dp, dp]
        L.qko_payoffs.argtypes = [C.POINTER(Contract), C.c_int, dp]
        L.qko_price.argtypes = [C.POINTER(Contract), C.POINTER(Greeks), C.POINTER(Result)]
        L.qko_exact_call.argtypes = [C.c_int, C.POINTER(Contract), C.c_double, dp]
        L.qko_lsm_solve_reference.argtypes = [dp, dp, C.c_double, C.c_int, dp]
        L.qko_gl_nodes.argtypes = [dp, dp]
        L.qko_payoff_path.argtypes = [C.POINTER(Payoff), dp, C.c_int, C.c_double, C.c_int, dp]
        _lib = L
    return _lib


def as_oracle(c) -> Contract:
    """Copy an engine contract (same layout) into the oracle's structure."""
    o = Contract()
    C.memmove(C.byref(o), C.byref(c), C.sizeof(Contract))
    return o


def as_greeks(g) -> Greeks | None:
    if g is None:
        return None
    o = Greeks()
    C.memmove(C.byref(o), C.byref(g), C.sizeof(Greeks))
    return o


def philox(ctr, key) -> tuple[int, int, int, int]:
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().qko_philox(c, k, o)
    return tuple(int(x) for x in o)


def step_trace(precision: int, contract, z: np.ndarray, u: np.ndarray | None = None):
    z = np.ascontiguousarray(z, dtype=np.float64)
    n = z.shape[0]
    if u is None:
        u = np.zeros((n, 1))
    u = np.ascontiguousarray(u, dtype=np.float64)
    S, v = np.empty(n), np.empty(n)
    dp = C.POINTER(C.c_double)
    rc = lib().qko_step_trace(precision, C.byref(as_oracle(contract)), z.ctypes.data_as(dp), u.ctypes.data_as(dp),
                              u.shape[1], n, S.ctypes.data_as(dp), v.ctypes.data_as(dp))
    if rc != 0:
        raise RuntimeError(f"qko_step_trace rc={rc}")
    return S, v


def paths(contract, first: int, count: int):
    c = as_oracle(contract)
    S = np.empty((count, c.n_steps))
    v = np.empty((count, c.n_steps))
    dp = C.POINTER(C.c_double)
    if lib().qko_paths(C.byref(c), first, count, S.ctypes.data_as(dp), v.ctypes.data_as(dp)) != 0:
        raise RuntimeError("qko_paths failed")
    return S, v


def payoffs(contract, leg: int = 0) -> np.ndarray:
    c = as_oracle(contract)
    out = np.empty(c.n_paths)
    lib().qko_payoffs(C.byref(c), leg, out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def payoff_path(opt_type: int, right: int, S: np.ndarray, S0: float, K: float, B: float, fp32: bool = False) -> float:
    """The oracle's payoff of one leg on a fed spot sequence S_1..S_n (trackers start at S0)."""
    S = np.ascontiguousarray(S, dtype=np.float64)
    ps = Payoff(opt_type, right, K, B)
    out = C.c_double()
    if lib().qko_payoff_path(C.byref(ps), S.ctypes.data_as(C.POINTER(C.c_double)), len(S), S0, int(fp32),
                             C.byref(out)) != 0:
        raise RuntimeError("qko_payoff_path failed")
    return out.value


def price(contract, greeks=None) -> dict:
    out = Result()
    g = as_greeks(greeks)
    rc = lib().qko_price(C.byref(as_oracle(contract)), C.byref(g) if g is not None else None, C.byref(out))
    if rc != 0:
        raise RuntimeError(f"qko_price rc={rc}")
    legs = [{f: getattr(out.p[k], f) for f, _ in PayoffResult._fields_} for k in range(out.n_payoffs)]
    return {"n_paths": int(out.n_paths), "path_steps": out.path_steps, "legs": legs}


def exact_call(kind: int, contract, phi_max: float = 0.0) -> float:
    """kind 0 Black-Scholes, 1 Heston (GL64 on [0, phi_max=100]), 2 Bates (50-wide chunks to 8000)."""
    p = C.c_double()
    lib().qko_exact_call(kind, C.byref(as_oracle(contract)), phi_max, C.byref(p))
    return p.value


def lsm_solve_reference(M: np.ndarray, B: np.ndarray, count: float) -> np.ndarray:
    nb = len(B)
    M = np.ascontiguousarray(M, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    out = np.empty(nb)
    dp = C.POINTER(C.c_double)
    lib().qko_lsm_solve_reference(M.ctypes.data_as(dp), B.ctypes.data_as(dp), count, nb, out.ctypes.data_as(dp))
    return out


def gl_nodes() -> tuple[np.ndarray, np.ndarray]:
    x, w = np.empty(64), np.empty(64)
    dp = C.POINTER(C.c_double)
    lib().qko_gl_nodes(x.ctypes.data_as(dp), w.ctypes.data_as(dp))
    return x, w
