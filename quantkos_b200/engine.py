"""Python host API over the C ABI, with the reference's names.

The reference's public surface (paths relative to the reference project) and
its counterpart here:

* ``quantkos::Config::UInputs`` (include/core/config/Config.hpp:677-775)  -> :class:`UInputs`
* ``quantkos::Config::Parser::parse`` (src/IO/ConfigParser.cpp:36-294)  -> :meth:`Parser.parse`
* ``MCDispatcher(UInputs).launch_montecarlo()`` (include/core/engine/Distpatcher.hpp:78)
  -> :class:`MCDispatcher`
* ``MCResults`` / ``MCOpPrices`` / ``MCGreeks`` (MCEngine.hpp:93-135, OptionPricer.hpp:50-70)
  -> :class:`MCResults`, :class:`MCOpPrices`, :class:`MCGreeks`
* ``SDEScheme<M,S>::evolve_step`` with fed draws -> :func:`step_trace`

Errors follow the reference: validation problems raise ``ValueError`` (its
``std::invalid_argument``), everything else ``RuntimeError``.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np

from . import _lib as L


class QuantKosError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class QuantKosInvalidArgument(ValueError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def check(status: int, what: str = "") -> None:
    if status == L.QK_OK:
        return
    msg = (L.lib().qk_last_error() or b"").decode(errors="replace")
    text = f"{what}: {msg}" if what else msg
    if status in (L.QK_ERR_INVALID_ARG, L.QK_ERR_PARSE):
        raise QuantKosInvalidArgument(status, text)
    raise QuantKosError(status, text)


# ----------------------------------------------------------------------------- handle
class Handle:
    """Owns one device context, one CUDA stream and the device arenas."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        check(L.lib().qk_create(device, C.byref(self._h)), "qk_create")
        self.device = device

    @property
    def ptr(self) -> C.c_void_p:
        if not self._h:
            raise RuntimeError("handle destroyed")
        return self._h

    def close(self) -> None:
        if self._h:
            L.lib().qk_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self) -> "Handle":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    def stream(self) -> int:
        s = C.c_void_p()
        check(L.lib().qk_get_stream(self.ptr, C.byref(s)))
        return int(s.value or 0)

    def last_timing(self) -> dict:
        t = L.Timing()
        check(L.lib().qk_last_timing(self.ptr, C.byref(t)))
        return {"device_ms": t.device_ms, "paths_ms": t.paths_ms, "reduce_ms": t.reduce_ms,
                "launches": int(t.launches), "path_steps": t.path_steps, "h2d_bytes": int(t.h2d_bytes),
                "d2h_bytes": int(t.d2h_bytes)}

    def measure_sfu(self) -> float:
        """Measured MUFU operations per second of this device."""
        x = C.c_double()
        check(L.lib().qk_measure_sfu(self.ptr, C.byref(x)), "qk_measure_sfu")
        return x.value

    def autotune(self, contracts: Sequence[L.Contract], greeks: L.Greeks | None = None, reps: int = 2) -> list[dict]:
        """Time every launch shape per kernel kind on a sample and keep the fastest (qk_autotune)."""
        n = len(contracts)
        arr = (L.Contract * n)(*contracts)
        rep = L.TuneReport()
        check(L.lib().qk_autotune(self.ptr, arr, n, C.byref(greeks) if greeks else None, reps, C.byref(rep)),
              "qk_autotune")
        return [{"precision": rep.precision[k], "model": rep.model[k], "scheme": rep.scheme[k],
                 "tiles_per_warp": rep.tiles_per_warp[k], "guided_tail": rep.guided_tail[k],
                 "paths_per_lane": rep.paths_per_lane[k], "block_size": rep.block_size[k],
                 "best_ms": rep.best_ms[k], "default_ms": rep.default_ms[k]} for k in range(rep.n_kinds)]

    def tune_reset(self) -> None:
        """Back to the default launch shape of every kernel kind."""
        check(L.lib().qk_tune_reset(self.ptr), "qk_tune_reset")

    def tune_set(self, precision: int, model: int, scheme: int, tiles_per_warp: int, guided_tail: bool,
                 paths_per_lane: int = 1, block_size: int | None = None) -> None:
        check(L.lib().qk_tune_set(self.ptr, precision, model, scheme, tiles_per_warp, int(guided_tail),
                                  paths_per_lane), "qk_tune_set")
        if block_size is not None:
            check(L.lib().qk_tune_set_block(self.ptr, precision, model, scheme, block_size), "qk_tune_set_block")


_default: Handle | None = None


def default_handle() -> Handle:
    global _default
    if _default is None:
        _default = Handle(0)
    return _default


# ----------------------------------------------------------------------------- contracts
def payoff(type: int = L.EUROPEAN, right: int = L.CALL, strike: float = 100.0, barrier: float = 100.0) -> L.Payoff:
    return L.Payoff(type, right, strike, barrier)


def make_contract(*, S0=100.0, v0=0.04, r=0.03, q=0.0, model=L.HESTON, scheme=L.EULER, kappa=2.0, theta=0.04,
                  sigma=0.3, rho=-0.7, lambda_j=0.0, mu_j=0.0, sigma_j=0.0, psi_c=1.5, T=1.0, n_steps=252,
                  normalize=True, n_paths=100_000, seed=42, stream=0, precision=L.FP32,
                  payoffs: Sequence[L.Payoff] | None = None, lsm_basis=L.LSM_LAGUERRE3, lsm_dates=0,
                  antithetic=False) -> L.Contract:
    c = L.Contract()
    c.S0, c.v0, c.r, c.q = S0, v0, r, q
    c.model, c.scheme = model, scheme
    c.kappa, c.theta, c.sigma, c.rho = kappa, theta, sigma, rho
    c.lambda_j, c.mu_j, c.sigma_j, c.psi_c = lambda_j, mu_j, sigma_j, psi_c
    c.T, c.n_steps, c.normalize = T, int(n_steps), int(bool(normalize))
    c.n_paths, c.seed, c.stream, c.precision = int(n_paths), int(seed), int(stream), int(precision)
    legs = list(payoffs) if payoffs else [payoff()]
    if not 1 <= len(legs) <= L.QK_MAX_PAYOFFS:
        raise ValueError("1..8 payoff legs")
    c.n_payoffs = len(legs)
    for i, p in enumerate(legs):
        c.payoffs[i] = p
    c.lsm_basis, c.lsm_dates = lsm_basis, lsm_dates
    c.antithetic = int(bool(antithetic))
    return c


def make_greeks(mask=L.GREEK_ALL, vega_mode=0, bump_S_rel=0.001, bump_vol=0.01, bump_r_abs=1e-4,
                bump_T_abs=1.0 / 365.0) -> L.Greeks:
    return L.Greeks(mask, vega_mode, bump_S_rel, bump_vol, bump_r_abs, bump_T_abs)


def result_to_dict(r: L.Result) -> dict:
    legs = []
    for k in range(r.n_payoffs):
        p = r.p[k]
        legs.append({f: getattr(p, f) for f, _ in L.PayoffResult._fields_})
    return {"status": r.status, "n_paths": int(r.n_paths), "path_steps": r.path_steps, "legs": legs}


def price_plain(contract: L.Contract, greeks: L.Greeks | None = None, handle: Handle | None = None) -> dict:
    """The drop-in: one contract, all-FP64, one kernel launch per pricing (bumps included)."""
    h = handle or default_handle()
    out = L.Result()
    check(L.lib().qk_price_plain(h.ptr, C.byref(contract), C.byref(greeks) if greeks else None, C.byref(out)),
          "qk_price_plain")
    return result_to_dict(out)


def price_batch(contracts: Sequence[L.Contract], greeks: L.Greeks | None = None,
                handle: Handle | None = None) -> list[dict]:
    """The batched mixed-precision engine: every contract and bump in one persistent launch."""
    h = handle or default_handle()
    n = len(contracts)
    arr = (L.Contract * n)(*contracts)
    out = (L.Result * n)()
    check(L.lib().qk_price_batch(h.ptr, arr, n, C.byref(greeks) if greeks else None, out), "qk_price_batch")
    return [result_to_dict(out[i]) for i in range(n)]


def price_noalloc(contract: L.Contract, stream: int = 0) -> dict:
    """Base price of one forward contract without any device allocation (fixed scratch).

    For callers that may not allocate GPU memory while pricing; see qk_price_noalloc in
    include/quantkos_b200.h for the size limit and the rules of use."""
    out = L.Result()
    check(L.lib().qk_price_noalloc(C.byref(contract), C.c_void_p(stream or None), C.byref(out)), "qk_price_noalloc")
    return result_to_dict(out)


class PreparedBatch:
    """Device-resident task set: prepare once, run many times (inputs stay in HBM)."""

    def __init__(self, contracts: Sequence[L.Contract], greeks: L.Greeks | None = None, handle: Handle | None = None):
        self.h = handle or default_handle()
        self.n = len(contracts)
        self._arr = (L.Contract * self.n)(*contracts)
        check(L.lib().qk_batch_prepare(self.h.ptr, self._arr, self.n, C.byref(greeks) if greeks else None),
              "qk_batch_prepare")

    def run(self) -> None:
        check(L.lib().qk_batch_run(self.h.ptr), "qk_batch_run")

    def fetch(self) -> list[dict]:
        out = (L.Result * self.n)()
        check(L.lib().qk_batch_fetch(self.h.ptr, out, self.n), "qk_batch_fetch")
        return [result_to_dict(out[i]) for i in range(self.n)]


def step_trace(precision: int, contract: L.Contract, z: np.ndarray, u: np.ndarray | None = None
               ) -> tuple[np.ndarray, np.ndarray]:
    """Run SDEScheme<M,S>::evolve_step n times on the device with fed draws.

    z: (n, 3) = (Z1, Z2, Zjump) per step; u: (n, umax) Poisson uniforms per step."""
    z = np.ascontiguousarray(z, dtype=np.float64)
    n = z.shape[0]
    if u is None:
        u = np.zeros((n, 1))
    u = np.ascontiguousarray(u, dtype=np.float64)
    umax = u.shape[1]
    S = np.empty(n)
    v = np.empty(n)
    dp = C.POINTER(C.c_double)
    check(L.lib().qk_step_trace(precision, C.byref(contract), z.ctypes.data_as(dp), u.ctypes.data_as(dp), umax, n,
                                S.ctypes.data_as(dp), v.ctypes.data_as(dp)), "qk_step_trace")
    return S, v


def paths(contract: L.Contract, first: int, count: int, handle: Handle | None = None
          ) -> tuple[np.ndarray, np.ndarray]:
    """Spot (real units) and variance paths exactly as the pricing kernels generate them."""
    h = handle or default_handle()
    S = np.empty((count, contract.n_steps))
    v = np.empty((count, contract.n_steps))
    dp = C.POINTER(C.c_double)
    check(L.lib().qk_paths_dump(h.ptr, C.byref(contract), first, count, S.ctypes.data_as(dp), v.ctypes.data_as(dp)),
          "qk_paths_dump")
    return S, v


# ----------------------------------------------------------------------------- reference-named layer
_OPT_TYPES = ["European", "Asian", "BarrierUpAndOut", "BarrierDownAndOut", "BarrierUpAndIn", "BarrierDownAndIn",
              "LookbackFloatingStrike", "LookbackFixedStrike", "BinaryCashOrNothing", "BinaryAssetOrNothing",
              "American"]


class UInputs:
    """quantkos::Config::UInputs: the full configuration tree (flat fields of qk_config)."""

    def __init__(self, cfg: L.Config | None = None):
        if cfg is None:
            cfg = L.Config()
            check(L.lib().qk_config_default(C.byref(cfg)))
        object.__setattr__(self, "_c", cfg)

    def __getattr__(self, name):
        c = object.__getattribute__(self, "_c")
        val = getattr(c, name)
        return val.decode() if isinstance(val, bytes) else val

    def __setattr__(self, name, value):
        if isinstance(value, str):
            value = value.encode()
        setattr(self._c, name, value)

    def validate(self) -> "UInputs":
        check(L.lib().qk_config_validate(C.byref(self._c)), "UInputs::validate")
        return self

    def to_contract(self) -> tuple[L.Contract, L.Greeks]:
        k, g = L.Contract(), L.Greeks()
        check(L.lib().qk_config_to_contract(C.byref(self._c), C.byref(k), C.byref(g)))
        return k, g

    @property
    def raw(self) -> L.Config:
        return self._c


class Parser:
    @staticmethod
    def parse(path: str) -> UInputs:
        cfg = L.Config()
        check(L.lib().qk_config_parse_file(str(path).encode(), C.byref(cfg)), "Parser::parse")
        return UInputs(cfg)

    @staticmethod
    def parse_string(text: str) -> UInputs:
        cfg = L.Config()
        check(L.lib().qk_config_parse_string(text.encode(), C.byref(cfg)), "Parser::parse")
        return UInputs(cfg)


@dataclass
class MCOpPrices:
    option_price: float
    standard_error: float
    prob_itm: float
    percentiles: dict = field(default_factory=dict)
    is_computed: bool = True


@dataclass
class MCGreeks:
    delta: float = 0.0
    gamma: float = 0.0
    vega: float = 0.0
    vomma: float = 0.0
    vanna: float = 0.0
    rho: float = 0.0
    theta: float = 0.0


@dataclass
class MCResults:
    MCConfig: UInputs
    OptionPrice: MCOpPrices
    Greeks: MCGreeks
    Timing: dict


_PCT_NAMES = ["p0", "p1", "p5", "p10", "p20", "p30", "p40", "median", "p60", "p70", "p80", "p90", "p95", "p99", "p100"]


class MCDispatcher:
    """MCDispatcher(UInputs).launch_montecarlo() -> MCResults."""

    def __init__(self, config: UInputs, handle: Handle | None = None):
        self.config = config
        self.handle = handle or default_handle()

    def launch_montecarlo(self) -> MCResults:
        out = L.Result()
        pct = (C.c_double * 15)()
        check(L.lib().qk_run_config(self.handle.ptr, C.byref(self.config.raw), C.byref(out), pct),
              "MCDispatcher::launch_montecarlo")
        p = out.p[0]
        pcts = {n: pct[i] for i, n in enumerate(_PCT_NAMES)} if self.config.analyze_distribution else {}
        return MCResults(self.config, MCOpPrices(p.price, p.std_error, p.prob_itm, pcts),
                         MCGreeks(p.delta, p.gamma, p.vega, p.vomma, p.vanna, p.rho, p.theta),
                         self.handle.last_timing())


# ----------------------------------------------------------------------------- serving
class Server:
    """Continuous-batching request loop (qk_serve_*)."""

    def __init__(self, handle: Handle | None = None, hbm_budget_mib: int = 0, max_batch: int = 256, lanes: int = 0,
                 wave_ms: float = 0.0, reserve_mib: int = 0, plain_fp64: bool = False):
        """lanes: host threads whose waves run on the GPU at once (0 = 4); wave_ms: estimated GPU time at
        which a lane closes a wave (0 = 2.5 ms); reserve_mib: HBM mapped into the device pool at the start and
        held until stop, from which the lanes' buffers grow (0 = the budget, -1 = none); plain_fp64: serve
        every request alone with the plain FP64 method (for comparing the methods on one stream)."""
        self.handle = handle or default_handle()
        self._s = C.c_void_p()
        opt = L.ServeOptions(hbm_budget_mib, max_batch, lanes, wave_ms, reserve_mib, int(bool(plain_fp64)), 0)
        check(L.lib().qk_serve_start_ex(self.handle.ptr, C.byref(opt), C.byref(self._s)), "qk_serve_start_ex")

    def submit(self, contract: L.Contract, greeks: L.Greeks | None = None) -> int:
        t = C.c_int64()
        check(L.lib().qk_serve_submit(self._s, C.byref(contract), C.byref(greeks) if greeks else None, C.byref(t)),
              "qk_serve_submit")
        return t.value

    def poll(self, ticket: int, wait_ms: int = 0) -> dict | None:
        done = C.c_int32()
        out = L.Result()
        check(L.lib().qk_serve_poll(self._s, ticket, wait_ms, C.byref(done), C.byref(out)), "qk_serve_poll")
        return result_to_dict(out) if done.value else None

    def cancel(self, ticket: int) -> bool:
        """Withdraw a request still waiting for admission (its poll then raises QK_ERR_CANCELLED)."""
        c = C.c_int32()
        check(L.lib().qk_serve_cancel(self._s, ticket, C.byref(c)), "qk_serve_cancel")
        return bool(c.value)

    def records(self) -> list[dict]:
        """Per-request accounting of the completed requests (qk_serve_records)."""
        n = C.c_int64()
        check(L.lib().qk_serve_records(self._s, None, 0, C.byref(n)), "qk_serve_records")
        arr = (L.ServeRecord * max(n.value, 1))()
        check(L.lib().qk_serve_records(self._s, arr, n.value, C.byref(n)), "qk_serve_records")
        return [{f: getattr(arr[i], f) for f, _ in L.ServeRecord._fields_} for i in range(n.value)]

    def stats(self) -> dict:
        s = L.ServeStats()
        check(L.lib().qk_serve_stats_get(self._s, C.byref(s)))
        return {f: getattr(s, f) for f, _ in L.ServeStats._fields_}

    def stop(self) -> None:
        if self._s:
            L.lib().qk_serve_stop(self._s)
            self._s = C.c_void_p()

    def __enter__(self) -> "Server":
        return self

    def __exit__(self, *exc) -> None:
        self.stop()


def n_steps_for(T: float, dt: float) -> int:
    """TimeConfig::validate: N = ceil(T/dt)."""
    return int(math.ceil(T / dt))
