"""Cases on which prices and Greeks are compared with the reference's own engine.

The reference side is its whole pricing path (MCDispatcher -> ForwardMCRunner /
ForwardBackwardMCRunner -> execute_mc_framework, include/core/engine/*.hpp),
compiled from its headers against the host shim (oracle/_ref).  Each side draws
from its own generator, so results agree in distribution only: the comparison is
|a - b| <= 3 combined standard errors (the reference's 3-SE rule,
include/tests/TestsUtils.hpp:124-165).

The reference's shim pool holds one generator state per OpenMP thread under a
static schedule, so its draws depend on the thread count; the comparisons pin it
(REF_THREADS) and are therefore the same on every machine.

Greeks: the standard error of a finite-difference Greek is taken from independent
replications (different seeds): mean over GREEK_REPS pricings, SE = sample
standard deviation / sqrt(GREEK_REPS), on each side.  24 replications of 20,000
paths rather than fewer, larger ones: the SE estimate itself needs the degrees of
freedom (with 12 it came out at half the exact per-path SE for one vanna).
Under Bates the reference's Theta loses common random numbers (Knuth's Poisson
loop consumes a dt-dependent number of uniforms, so the T-bumped repricing
drifts onto other draws); its SE is then about 15 times the engine's and is
what the comparison uses.
"""
from __future__ import annotations

import math

import numpy as np

REF_THREADS = 8
K_SE = 3.0
GREEK_REPS = 24
GREEK_NAMES = ("delta", "gamma", "vega", "vomma", "vanna", "rho", "theta")

# (model, scheme) pairs of the all-payoff price comparison
PRICE_KINDS = ((1, 2), (0, 0), (0, 1))


def strike_barrier(opt_type: int) -> tuple[float, float]:
    """A barrier level that the paths cross often: above S0 for the up barriers,
    below for the down ones."""
    if opt_type in (2, 4):
        return 100.0, 120.0
    if opt_type in (3, 5):
        return 100.0, 85.0
    return 100.0, 100.0


def price_case(make_contract, L, model: int, scheme: int, opt_type: int, right: int, n_paths: int = 100_000,
               precision=None):
    K, B = strike_barrier(opt_type)
    return make_contract(S0=100.0, v0=0.05, r=0.03, q=0.01, model=model, scheme=scheme, kappa=3.0, theta=0.05,
                         sigma=0.5, rho=-0.7, lambda_j=0.5 if model else 0.0, mu_j=-0.1, sigma_j=0.12, T=0.5,
                         n_steps=32, n_paths=n_paths, seed=31, precision=L.FP64 if precision is None else precision,
                         payoffs=[L.Payoff(opt_type, right, K, B)])


def ref_price_seed(opt_type: int, right: int) -> int:
    return 1000 + 10 * opt_type + right


# Greeks: (model, scheme, type, right, K, B); bumps larger than the reference defaults so
# that second-order Greeks are resolved with a few hundred thousand paths in all
GREEK_CASES = ((0, 2, 0, 0, 100.0, 100.0), (1, 0, 1, 1, 100.0, 100.0), (0, 1, 2, 0, 100.0, 125.0),
               (1, 2, 7, 0, 100.0, 100.0))
GREEK_BUMPS = dict(bump_S_rel=0.01, bump_vol=0.02, bump_r_abs=1e-3, bump_T_abs=2.0 / 365.0)


def greek_case(make_contract, L, model, scheme, opt_type, right, K, B, rep: int, n_paths: int = 20_000,
               precision=None):
    return make_contract(S0=100.0, v0=0.05, r=0.03, q=0.01, model=model, scheme=scheme, kappa=3.0, theta=0.05,
                         sigma=0.5, rho=-0.7, lambda_j=0.5 if model else 0.0, mu_j=-0.1, sigma_j=0.12, T=0.5,
                         n_steps=24, n_paths=n_paths, seed=1500 + rep, precision=L.FP64 if precision is None else precision,
                         payoffs=[L.Payoff(opt_type, right, K, B)])


def ref_greek_config(qkref, contract, rep: int):
    b = GREEK_BUMPS
    return qkref.from_contract(contract, seed=10000 + rep, greeks_mask=31, bump_S_rel=b["bump_S_rel"],
                               bump_vol_abs=b["bump_vol"], bump_r_abs=b["bump_r_abs"], bump_T_abs=b["bump_T_abs"])


def replicated(rows: list[list[float]]) -> tuple[np.ndarray, np.ndarray]:
    """Mean and standard error over replications (rows) of each column."""
    a = np.asarray(rows, dtype=float)
    return a.mean(axis=0), a.std(axis=0, ddof=1) / math.sqrt(a.shape[0])


# American put, reference mode (Laguerre basis on S/K, every step an exercise date):
# (model, scheme, K, steps)
AMERICAN_CASES = ((0, 2, 100.0, 50), (0, 0, 110.0, 40), (1, 1, 90.0, 30))


def american_case(make_contract, L, model, scheme, K, steps, n_paths: int = 400_000, precision=None):
    return make_contract(S0=100.0, v0=0.04, r=0.05, q=0.0, model=model, scheme=scheme, kappa=2.0, theta=0.04,
                         sigma=0.3, rho=-0.7, lambda_j=0.3 if model else 0.0, mu_j=-0.1, sigma_j=0.1, T=1.0,
                         n_steps=steps, n_paths=n_paths, seed=77, precision=L.FP64 if precision is None else precision,
                         payoffs=[L.Payoff(L.AMERICAN, L.PUT, K, 0.0)], lsm_basis=L.LSM_LAGUERRE3, lsm_dates=0)


def z_score(a: float, b: float, se_a: float, se_b: float) -> float:
    s = math.hypot(se_a, se_b)
    return abs(a - b) / s if s > 0 else (0.0 if a == b else math.inf)
