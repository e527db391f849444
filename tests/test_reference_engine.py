"""CPU: the oracle against the reference's own engine (oracle/_ref).

* payoffs: the oracle's payoff path on fed spot sequences equals PayoffTracker
  (include/core/options/Payoff.hpp:84-243) on the reference-generated fixtures and
  on random non-monotone sequences that cross the barriers, FP64 and FP32, to 1e-12;
* prices of every payoff type and right under three (model, scheme) pairs, Greeks
  (all seven, by replication) and the reference-mode American put agree with the
  reference's pricing path within 3 combined standard errors.

The same comparisons run engine-against-reference on the GPU in
test_gpu_reference_engine.py.
"""
import math

import numpy as np
import pytest

import refcases as RC
from helpers import load


@pytest.fixture(scope="module")
def pinned_ref(ref):
    ref.set_threads(RC.REF_THREADS)
    return ref


def _api():
    from quantkos_b200 import _lib as L
    from quantkos_b200.engine import make_contract, make_greeks
    return L, make_contract, make_greeks


def test_oracle_payoff_path_on_reference_fixtures(oracle):
    """Every reference-generated PayoffTracker case (10 types x 2 rights, random sequences)."""
    cases = load("payoff_cases.json")
    assert len(cases) == 120
    for c in cases:
        got = oracle.payoff_path(c["type"], c["right"], np.array(c["S"]), c["S0"], c["K"], c["B"])
        assert math.isclose(got, c["payoff"], rel_tol=1e-12, abs_tol=1e-15), (c, got)


def test_oracle_payoff_path_matches_reference_live(oracle, ref):
    """Random walks of 1..40 steps with barriers placed where the walks cross them, every
    type and right, against the reference's PayoffTracker in both of its builds."""
    rng = np.random.default_rng(2024)
    crossed = {2: 0, 3: 0}
    for _ in range(200):
        m = int(rng.integers(1, 41))
        S = np.exp(np.cumsum(rng.normal(0.0, 0.05, m)))
        K = float(rng.uniform(0.85, 1.15))
        B = float(rng.uniform(0.8, 0.97)) if rng.uniform() < 0.5 else float(rng.uniform(1.03, 1.25))
        crossed[2] += int(max(1.0, S.max()) >= B > 1.0)
        crossed[3] += int(min(1.0, S.min()) <= B < 1.0)
        for t in range(10):
            for right in (0, 1):
                want = ref.payoff(t, right, S, 1.0, K, B)
                got = oracle.payoff_path(t, right, S, 1.0, K, B)
                assert math.isclose(got, want, rel_tol=1e-12, abs_tol=1e-15), (t, right, S, K, B)
                want32 = ref.payoff(t, right, S, 1.0, K, B, real_bytes=4)
                got32 = oracle.payoff_path(t, right, S, 1.0, K, B, fp32=True)
                assert math.isclose(got32, want32, rel_tol=1e-12, abs_tol=1e-15), (t, right, S, K, B)
    assert crossed[2] > 20 and crossed[3] > 20  # the barrier logic is exercised on both sides


@pytest.mark.parametrize("model,scheme", RC.PRICE_KINDS)
def test_prices_every_payoff_vs_reference_engine(oracle, pinned_ref, model, scheme):
    L, make_contract, _ = _api()
    for t in range(10):
        for right in (0, 1):
            k = RC.price_case(make_contract, L, model, scheme, t, right)
            o = oracle.price(k)["legs"][0]
            r = pinned_ref.price(pinned_ref.from_contract(k, seed=RC.ref_price_seed(t, right)))
            z = RC.z_score(o["price"], r["price"], o["std_error"], r["std_error"])
            assert z <= RC.K_SE, (model, scheme, t, right, o, r)
            assert abs(o["std_error"] / r["std_error"] - 1.0) < 0.25


@pytest.mark.parametrize("case", RC.GREEK_CASES)
def test_greeks_vs_reference_engine(oracle, pinned_ref, case):
    """All seven Greeks (and the price) by central differences under common random
    numbers on each side; SE of each finite difference from 12 replications."""
    L, make_contract, make_greeks = _api()
    b = RC.GREEK_BUMPS
    g = make_greeks(L.GREEK_ALL, vega_mode=0, bump_S_rel=b["bump_S_rel"], bump_vol=b["bump_vol"],
                    bump_r_abs=b["bump_r_abs"], bump_T_abs=b["bump_T_abs"])
    cols = ("price",) + RC.GREEK_NAMES
    o_rows, r_rows = [], []
    for rep in range(RC.GREEK_REPS):
        k = RC.greek_case(make_contract, L, *case, rep)
        o = oracle.price(k, g)["legs"][0]
        r = pinned_ref.price(RC.ref_greek_config(pinned_ref, k, rep))
        o_rows.append([o[c] for c in cols])
        r_rows.append([r[c] for c in cols])
    mo, so = RC.replicated(o_rows)
    mr, sr = RC.replicated(r_rows)
    for j, c in enumerate(cols):
        assert RC.z_score(mo[j], mr[j], so[j], sr[j]) <= RC.K_SE, (case, c, mo[j], so[j], mr[j], sr[j])


@pytest.mark.parametrize("case", RC.AMERICAN_CASES)
def test_american_reference_mode_vs_reference_engine(oracle, pinned_ref, case):
    """Longstaff-Schwartz with the reference's Laguerre basis at every step against
    ForwardBackwardMCRunner (include/core/engine/ForwardBackwardMC.hpp:204-255)."""
    L, make_contract, _ = _api()
    k = RC.american_case(make_contract, L, *case)
    o = oracle.price(k)["legs"][0]
    r = pinned_ref.price(pinned_ref.from_contract(k, seed=4242))
    assert RC.z_score(o["price"], r["price"], o["std_error"], r["std_error"]) <= RC.K_SE, (case, o, r)
    assert abs(o["std_error"] / r["std_error"] - 1.0) < 0.1
    assert abs(o["prob_itm"] - r["prob_itm"]) < 0.01
