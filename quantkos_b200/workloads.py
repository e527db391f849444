"""Seeded synthetic generators for the benchmark workloads.

* :func:`plain_heston_euler` — the plain-method case: one European call, Heston
  Euler, 1,048,576 paths x 252 steps, FP64, seed 42.
* :func:`bates_qe_five_payoffs` — one Bates/QE contract, 16,777,216 paths x 252
  steps, five payoff legs in one pass, FP32.
* :func:`american_lsm` — American put by Longstaff-Schwartz, Heston QE, 4,194,304
  paths x 250 steps, 50 exercise dates, basis {1,S,S^2,S^3,v,Sv}, seed 7.
* :func:`mixed_batch` — 4096 contracts drawn with seed 123 (Heston/Bates, Euler/
  Milstein/QE, European/Asian/barrier/binary, log-uniform path counts) with the
  full set of finite-difference Greeks.
* :func:`serving_stream` — Poisson arrivals of pricing requests drawn like the
  mixed batch with a 30% share of American puts.

Choices the workload descriptions leave open are fixed here: S0 = 100,
r = 0.03, q = 0; calls and puts 50/50; the barrier leg is an up-and-out call
with B ~ U[1.15, 1.5] S0 or a down-and-out put with B ~ U[0.5, 0.85] S0; the
binary leg is cash-or-nothing; Bates jumps
lambda ~ U[0.05, 0.5], muJ ~ U[-0.15, 0.05], sigmaJ ~ U[0.05, 0.2]; Greeks bump
1% of S0, 1% of v0 (relative v0 bump, vega per unit of variance), 1 bp of r and
one day (1/365) of T.
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib as L
from .engine import make_contract, make_greeks, payoff


def plain_heston_euler() -> L.Contract:
    return make_contract(S0=100.0, v0=0.04, r=0.03, q=0.0, model=L.HESTON, scheme=L.EULER, kappa=2.0, theta=0.04,
                         sigma=0.3, rho=-0.7, T=1.0, n_steps=252, n_paths=1_048_576, seed=42, precision=L.FP64,
                         payoffs=[payoff(L.EUROPEAN, L.CALL, 100.0)])


def bates_qe_five_payoffs(n_paths: int = 16_777_216, stream: int = 0, precision: int = L.FP32) -> L.Contract:
    legs = [payoff(L.EUROPEAN, L.CALL, 100.0), payoff(L.ASIAN, L.CALL, 100.0),
            payoff(L.BARRIER_UP_OUT, L.CALL, 100.0, 130.0), payoff(L.LOOKBACK_FLOATING, L.PUT, 100.0),
            payoff(L.BINARY_CASH, L.CALL, 105.0)]
    return make_contract(S0=100.0, v0=0.04, r=0.03, q=0.0, model=L.BATES, scheme=L.ANDERSEN_QE, kappa=2.0,
                         theta=0.04, sigma=0.3, rho=-0.7, lambda_j=0.1, mu_j=-0.05, sigma_j=0.10, psi_c=1.5, T=1.0,
                         n_steps=252, n_paths=n_paths, seed=42, stream=stream, precision=precision, payoffs=legs)


def american_lsm(n_paths: int = 4_194_304, precision: int = L.FP32, basis: int = L.LSM_POLY_SV,
                 dates: int = 50) -> L.Contract:
    return make_contract(S0=100.0, v0=0.04, r=0.03, q=0.0, model=L.HESTON, scheme=L.ANDERSEN_QE, kappa=2.0,
                         theta=0.04, sigma=0.3, rho=-0.7, T=1.0, n_steps=250, n_paths=n_paths, seed=7,
                         precision=precision, payoffs=[payoff(L.AMERICAN, L.PUT, 100.0)], lsm_basis=basis,
                         lsm_dates=dates)


def batch_greeks() -> L.Greeks:
    return make_greeks(L.GREEK_ALL, vega_mode=1, bump_S_rel=0.01, bump_vol=0.01, bump_r_abs=1e-4,
                       bump_T_abs=1.0 / 365.0)


def _draw_contract(rng: np.random.Generator, i: int, precision: int, american_share: float = 0.0,
                   path_range=(1e4, 2e6), american_paths=(1e5, 4e6)) -> L.Contract:
    model = L.BATES if rng.random() < 0.5 else L.HESTON
    scheme = int(rng.integers(0, 3))
    K = float(rng.uniform(80.0, 120.0))
    T = float(rng.uniform(0.1, 2.0))
    n_steps = int(math.ceil(252.0 * T))
    v0 = float(rng.uniform(0.01, 0.09))
    theta = float(rng.uniform(0.01, 0.09))
    kappa = float(rng.uniform(0.5, 4.0))
    sigma = float(rng.uniform(0.1, 0.8))
    rho = float(rng.uniform(-0.9, -0.1))
    lam = float(rng.uniform(0.05, 0.5))
    muj = float(rng.uniform(-0.15, 0.05))
    sj = float(rng.uniform(0.05, 0.2))
    right = int(rng.integers(0, 2))
    kind = int(rng.integers(0, 4))
    lo, hi = path_range
    n_paths = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
    b_up = float(rng.uniform(1.15, 1.5)) * 100.0
    b_dn = float(rng.uniform(0.5, 0.85)) * 100.0
    american = american_share > 0.0 and rng.random() < american_share
    if american:
        lo, hi = american_paths
        n_paths = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        leg = payoff(L.AMERICAN, L.PUT, K)
        n_steps = 50 * int(math.ceil(252.0 * T / 50.0))  # a multiple of the 50 exercise dates
        return make_contract(S0=100.0, v0=v0, r=0.03, q=0.0, model=model, scheme=scheme, kappa=kappa, theta=theta,
                             sigma=sigma, rho=rho, lambda_j=lam if model == L.BATES else 0.0, mu_j=muj, sigma_j=sj,
                             T=T, n_steps=n_steps, n_paths=n_paths, seed=123, stream=i, precision=precision,
                             payoffs=[leg], lsm_basis=L.LSM_POLY_SV, lsm_dates=50)
    if kind == 0:
        leg = payoff(L.EUROPEAN, right, K)
    elif kind == 1:
        leg = payoff(L.ASIAN, right, K)
    elif kind == 2:
        leg = payoff(L.BARRIER_UP_OUT, L.CALL, K, b_up) if right == L.CALL else payoff(L.BARRIER_DOWN_OUT, L.PUT, K, b_dn)
    else:
        leg = payoff(L.BINARY_CASH, right, K)
    return make_contract(S0=100.0, v0=v0, r=0.03, q=0.0, model=model, scheme=scheme, kappa=kappa, theta=theta,
                         sigma=sigma, rho=rho, lambda_j=lam if model == L.BATES else 0.0, mu_j=muj, sigma_j=sj, T=T,
                         n_steps=n_steps, n_paths=n_paths, seed=123, stream=i, precision=precision, payoffs=[leg])


def mixed_batch(n: int = 4096, seed: int = 123, precision: int = L.FP32) -> list[L.Contract]:
    rng = np.random.default_rng(seed)
    return [_draw_contract(rng, i, precision) for i in range(n)]


def serving_stream(n: int = 20_000, rate_per_s: float = 2000.0, seed: int = 123, precision: int = L.FP32
                   ) -> tuple[np.ndarray, list[L.Contract]]:
    """(arrival times in seconds, contracts): Poisson arrivals, 30% American puts via LSM."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_per_s, n)
    arrivals = np.cumsum(gaps)
    contracts = [_draw_contract(rng, i, precision, american_share=0.3) for i in range(n)]
    return arrivals, contracts


def path_steps(contracts, greeks: L.Greeks | None = None) -> float:
    """Path-steps a set of contracts costs, counting the Greek bumps (11 extra tasks with all Greeks)."""
    tasks = 1
    if greeks is not None and greeks.mask:
        tasks += 2 * bool(greeks.mask & L.GREEK_DELTA_GAMMA) + 2 * bool(greeks.mask & L.GREEK_VEGA_VOMMA) \
            + 2 * bool(greeks.mask & L.GREEK_RHO) + 1 * bool(greeks.mask & L.GREEK_THETA) \
            + 4 * bool(greeks.mask & L.GREEK_VANNA)
    return float(sum(c.n_paths * c.n_steps for c in contracts)) * tasks
