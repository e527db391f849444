"""GPU parity: the CUDA path through the C ABI against the oracle and the
reference's golden fixtures.

Tolerances (stated per test):
* per-step scheme outputs vs the reference's own code: 1e-12 (FP64), 1e-5 (FP32);
* FP64 kernels vs the oracle on the same Philox paths: 1e-12 on paths, 1e-9 on prices;
* FP32 kernels vs the FP32 oracle: 1e-4 relative on paths over <=64 steps, prices
  within 0.05 standard errors;
* statistical checks vs closed forms / the reference's published values: 3 combined SE
  (plus the reference's own bias allowance where it has one).
"""
import math

import numpy as np
import pytest

from tests.helpers import TOL_STEP_FP32, TOL_STEP_FP64, case_contract, load, step_err, within_se

pytestmark = pytest.mark.gpu


def test_step_trace_matches_reference_golden(qk, handle):
    """One step on fed draws against the reference's own FP64 and FP32 builds: FP64 within
    1e-12; FP32 within 1e-5 of the reference's FP32 build.  Where the reference's two builds
    themselves differ by more than 1e-5 (11 of the 600 cases: variance 0 to 1e-4 at a
    vol-of-vol of 0.9, where FP32 rounding moves a QE step across a regime threshold), the
    FP32 step must agree with one of the two builds."""
    cases = load("step_cases.json")
    worst = {0: 0.0, 1: 0.0}
    n_boundary = 0
    for c in cases:
        k = case_contract(qk.make_contract, c)
        z = np.array([c["z"]])
        u = np.array([c["u"]])
        for prec in (qk.FP64, qk.FP32):
            S, v = qk.step_trace(prec, k, z, u)
            if prec == qk.FP64:
                e = step_err(S[0], v[0], c["S_out64"], c["v_out64"], c["v"])
                assert e <= TOL_STEP_FP64, (c, e)
            else:
                e = step_err(S[0], v[0], c["S_out32"], c["v_out32"], c["v"])
                if step_err(c["S_out32"], c["v_out32"], c["S_out64"], c["v_out64"], c["v"]) > TOL_STEP_FP32:
                    n_boundary += 1
                    e = min(e, step_err(S[0], v[0], c["S_out64"], c["v_out64"], c["v"]))
                assert e <= TOL_STEP_FP32, (c, e)
            worst[prec] = max(worst[prec], e)
    assert n_boundary == 11
    print("worst per-step error FP64 %.2e FP32 %.2e" % (worst[0], worst[1]))


def test_step_trace_trajectory_matches_oracle(qk, handle, oracle):
    rng = np.random.default_rng(3)
    for model in (0, 1):
        for scheme in (0, 1, 2):
            k = qk.make_contract(S0=1.0, v0=0.04, model=model, scheme=scheme, lambda_j=20.0 if model else 0.0,
                                 mu_j=-0.05, sigma_j=0.1, n_steps=252, normalize=False)
            z = rng.standard_normal((252, 3))
            u = rng.uniform(size=(252, 8))
            for prec, tol in ((qk.FP64, 1e-12), (qk.FP32, 2e-4)):
                Sg, vg = qk.step_trace(prec, k, z, u)
                So, vo = oracle.step_trace(prec, k, z, u)
                np.testing.assert_allclose(Sg, So, rtol=tol)
                np.testing.assert_allclose(vg, vo, rtol=tol * 10, atol=tol * 0.04)


def test_step_trace_rejects_uniform_overflow(qk, handle):
    k = qk.make_contract(S0=1.0, v0=0.04, model=qk.BATES, lambda_j=1.0, n_steps=1, T=1.0 / 252, normalize=False)
    z = np.zeros((1, 3))
    u = np.full((1, 2), 0.9999999)  # Knuth's loop wants more than 2 uniforms
    with pytest.raises(ValueError, match="umax"):
        qk.step_trace(qk.FP64, k, z, u)


@pytest.mark.parametrize("model,scheme", [(m, s) for m in (0, 1) for s in (0, 1, 2)])
def test_paths_match_oracle(qk, handle, oracle, model, scheme):
    k = qk.make_contract(S0=100.0, v0=0.04, model=model, scheme=scheme, lambda_j=3.0 if model else 0.0, mu_j=-0.05,
                         sigma_j=0.1, n_steps=64, T=0.5, n_paths=5000, seed=0xC0FFEE12345, stream=7)
    for prec, tol in ((qk.FP64, 1e-12), (qk.FP32, 1e-4)):
        k.precision = prec
        Sg, vg = qk.paths(k, 1000, 257, handle)
        So, vo = oracle.paths(k, 1000, 257)
        np.testing.assert_allclose(Sg, So, rtol=tol)
        np.testing.assert_allclose(vg, vo, rtol=tol * 20, atol=tol * 0.04)


ALL_LEGS = [(t, r) for t in range(10) for r in (0, 1)]


def _legs(qk, subset):
    return [qk.payoff(t, r, 100.0 if t not in (8, 9) else 103.0, 115.0 if t in (2, 4) else 90.0) for t, r in subset]


@pytest.mark.parametrize("model,scheme", [(0, 0), (0, 2), (1, 1), (1, 2)])
def test_plain_fp64_prices_match_oracle(qk, handle, oracle, model, scheme):
    for chunk in (ALL_LEGS[:8], ALL_LEGS[8:16], ALL_LEGS[16:]):
        k = qk.make_contract(model=model, scheme=scheme, lambda_j=0.5 if model else 0.0, mu_j=-0.1, sigma_j=0.15,
                             n_steps=48, n_paths=20_000, seed=12345, precision=qk.FP64, payoffs=_legs(qk, chunk))
        g = qk.price_plain(k, None, handle)
        o = oracle.price(k)
        for a, b in zip(g["legs"], o["legs"]):
            assert math.isclose(a["price"], b["price"], rel_tol=1e-9, abs_tol=1e-12), (a, b)
            assert math.isclose(a["std_error"], b["std_error"], rel_tol=1e-7, abs_tol=1e-12)
            assert a["prob_itm"] == pytest.approx(b["prob_itm"], abs=1e-4)


@pytest.mark.parametrize("model,scheme", [(0, 1), (1, 2)])
def test_batch_fp32_prices_match_fp32_oracle(qk, handle, oracle, model, scheme):
    k = qk.make_contract(model=model, scheme=scheme, lambda_j=0.5 if model else 0.0, mu_j=-0.1, sigma_j=0.15,
                         n_steps=48, n_paths=20_000, seed=777, precision=qk.FP32, payoffs=_legs(qk, ALL_LEGS[:8]))
    g = qk.price_batch([k], None, handle)[0]
    o = oracle.price(k)
    for a, b in zip(g["legs"], o["legs"]):
        assert abs(a["price"] - b["price"]) <= 0.05 * b["std_error"] + 1e-7, (a, b)


def test_multi_payoff_pass_equals_single_legs(qk, handle):
    legs = [qk.payoff(qk.EUROPEAN, qk.CALL, 100.0), qk.payoff(qk.ASIAN, qk.CALL, 100.0),
            qk.payoff(qk.BARRIER_UP_OUT, qk.CALL, 100.0, 130.0), qk.payoff(qk.LOOKBACK_FLOATING, qk.PUT, 100.0),
            qk.payoff(qk.BINARY_CASH, qk.CALL, 105.0)]
    base = dict(model=qk.BATES, scheme=qk.ANDERSEN_QE, lambda_j=0.1, mu_j=-0.05, sigma_j=0.1, n_paths=65_536,
                n_steps=252, seed=42)
    together = qk.price_batch([qk.make_contract(payoffs=legs, **base)], None, handle)[0]["legs"]
    for i, leg in enumerate(legs):
        alone = qk.price_batch([qk.make_contract(payoffs=[leg], **base)], None, handle)[0]["legs"][0]
        assert together[i]["price"] == pytest.approx(alone["price"], rel=1e-12, abs=1e-14)


def test_launch_shape_invariance(qk, handle):
    """A contract's price does not depend on what else is in the batch (tile plan / paths per thread)."""
    k = qk.make_contract(scheme=qk.ANDERSEN_QE, n_paths=300_001, n_steps=100, seed=99, stream=5, precision=qk.FP64)
    alone = qk.price_batch([k], None, handle)[0]["legs"][0]["price"]
    others = [qk.make_contract(n_paths=2_000_000, n_steps=200, seed=1 + i, stream=100 + i) for i in range(4)]
    mixed = qk.price_batch(others[:2] + [k] + others[2:], None, handle)[2]["legs"][0]["price"]
    plain = qk.price_plain(k, None, handle)["legs"][0]["price"]
    assert mixed == pytest.approx(alone, rel=1e-13)
    assert plain == pytest.approx(alone, rel=1e-13)


def test_block_size_changes_no_result(qk, handle):
    """Threads per block of the pricing kernel (128, 256, 512 in FP32; 128, 256 in FP64) only
    change which warps run the tiles: every tile covers the same paths and writes the same
    record, so every price, standard error and Greek is bit for bit the same; the autotuner's
    choice reports a valid block size."""
    legs = [qk.payoff(qk.EUROPEAN, qk.CALL, 100.0), qk.payoff(qk.ASIAN, qk.PUT, 95.0),
            qk.payoff(qk.BARRIER_UP_OUT, qk.CALL, 100.0, 125.0)]
    g = qk.make_greeks(qk.GREEK_ALL, bump_S_rel=0.01, bump_vol=0.02, bump_r_abs=1e-3, bump_T_abs=2 / 365)
    key = lambda r: [(leg[f] for f in ("price", "std_error", "delta", "gamma", "vega", "vanna", "theta"))
                     for leg in r["legs"]]
    for prec, blocks in ((qk.FP32, (128, 256, 512)), (qk.FP64, (128, 256))):
        ks = [qk.make_contract(model=qk.BATES, scheme=s, lambda_j=0.3, mu_j=-0.1, sigma_j=0.1, n_paths=n,
                               n_steps=40, seed=17, stream=i, precision=prec, payoffs=legs)
              for i, (s, n) in enumerate(((qk.ANDERSEN_QE, 400_003), (qk.EULER, 77_777), (qk.IMPLICIT_MILSTEIN, 150_000)))]
        results = []
        try:
            for b in blocks:
                for s in (qk.EULER, qk.IMPLICIT_MILSTEIN, qk.ANDERSEN_QE):
                    handle.tune_set(prec, qk.BATES, s, 24, False, 2 if prec == qk.FP32 else 1, block_size=b)
                rs = qk.price_batch(ks, g, handle)
                results.append([[list(x) for x in key(r)] for r in rs])
        finally:
            handle.tune_reset()
        for other in results[1:]:
            assert other == results[0]
    with pytest.raises(qk.QuantKosInvalidArgument):
        handle.tune_set(qk.FP64, qk.HESTON, qk.EULER, 24, False, 1, block_size=512)
    rep = handle.autotune([qk.make_contract(n_paths=200_000, n_steps=32, precision=qk.FP32)], None, reps=1)
    assert rep[0]["block_size"] in (128, 256, 512)
    handle.tune_reset()


def test_greeks_match_oracle(qk, handle, oracle):
    g = qk.make_greeks(qk.GREEK_ALL, bump_S_rel=0.01, bump_vol=0.02, bump_r_abs=0.001, bump_T_abs=7 / 365)
    for otype in (qk.EUROPEAN, qk.ASIAN, qk.BARRIER_DOWN_OUT):
        k = qk.make_contract(scheme=qk.ANDERSEN_QE, n_steps=32, n_paths=20_000, seed=4242, precision=qk.FP64,
                             payoffs=[qk.payoff(otype, qk.CALL, 100.0, 85.0)])
        got = qk.price_plain(k, g, handle)["legs"][0]
        want = oracle.price(k, g)["legs"][0]
        for f in ("price", "delta", "gamma", "vega", "vomma", "vanna", "rho", "theta"):
            assert got[f] == pytest.approx(want[f], rel=1e-7, abs=1e-9), f
        batched = qk.price_batch([k], g, handle)[0]["legs"][0]
        for f in ("price", "delta", "gamma", "vega", "vomma", "vanna", "rho", "theta"):
            assert batched[f] == pytest.approx(want[f], rel=1e-7, abs=1e-9), f


def test_greeks_crn_exactness(qk, handle):
    """Bumped tasks reuse the base contract's random numbers.  Prices are homogeneous in (S0, K)
    under the same multiplicative path factors, so the spot-up task (S0 = 1.001 normalised,
    K = 1) must equal a separately priced contract with S0 = 100.1, K = 100 on the same stream:
    p_up = p0 + delta h + gamma h^2 / 2 recovered from the Greeks matches it."""
    base = dict(n_paths=100_000, n_steps=64, precision=qk.FP64, seed=5, stream=3)
    k = qk.make_contract(**base)
    k_up = qk.make_contract(S0=100.0 * 1.001, **base)
    pd = qk.price_batch([k], qk.make_greeks(qk.GREEK_DELTA_GAMMA, bump_S_rel=0.001), handle)[0]["legs"][0]
    p0 = qk.price_batch([k], None, handle)[0]["legs"][0]["price"]
    assert pd["price"] == p0
    h = 100.0 * 0.001
    p_up = p0 + pd["delta"] * h + 0.5 * pd["gamma"] * h * h
    p_sep = qk.price_batch([k_up], None, handle)[0]["legs"][0]["price"]
    assert p_up == pytest.approx(p_sep, rel=1e-9)


@pytest.mark.parametrize("basis", [0, 1])
def test_lsm_matches_oracle(qk, handle, oracle, basis):
    k = qk.make_contract(S0=100.0, v0=0.04, scheme=qk.ANDERSEN_QE, n_steps=50, n_paths=20_000, seed=7,
                         precision=qk.FP64, payoffs=[qk.payoff(qk.AMERICAN, qk.PUT, 100.0)], lsm_basis=basis,
                         lsm_dates=0 if basis == 0 else 10)
    g = qk.price_plain(k, None, handle)["legs"][0]
    o = oracle.price(k)["legs"][0]
    assert abs(g["price"] - o["price"]) <= 0.02 * o["std_error"] + 1e-9, (g, o)
    assert g["std_error"] == pytest.approx(o["std_error"], rel=0.05)


def test_lsm_fp32_close_to_fp64(qk, handle):
    base = dict(S0=100.0, v0=0.04, scheme=qk.ANDERSEN_QE, n_steps=250, n_paths=200_000, seed=7,
                payoffs=[qk.payoff(qk.AMERICAN, qk.PUT, 100.0)], lsm_basis=qk.LSM_POLY_SV, lsm_dates=50)
    p64 = qk.price_plain(qk.make_contract(precision=qk.FP64, **base), None, handle)["legs"][0]
    p32 = qk.price_batch([qk.make_contract(precision=qk.FP32, **base)], None, handle)[0]["legs"][0]
    assert abs(p64["price"] - p32["price"]) < 0.2 * p64["std_error"]
    euro = qk.price_plain(qk.make_contract(precision=qk.FP64, **{**base, "payoffs": [qk.payoff(0, 1, 100.0)]}),
                          None, handle)["legs"][0]
    assert p64["price"] > euro["price"]  # early-exercise premium of the put


@pytest.mark.parametrize("right,q,n_paths,dates", [
    (1, 0.0, 50_003, 20),     # put; paths neither a multiple of 4 nor of the 1024-path chunk
    (0, 0.08, 80_000, 25),    # call with a dividend yield (early exercise pays)
    (1, 0.0, 30_001, 0),      # put, every step an exercise date
])
def test_lsm_fp32_poly_sv_cases_close_to_fp64(qk, handle, right, q, n_paths, dates):
    """The FP32 slab with the 6-term basis runs its own sweep arithmetic (FP32 on path
    pairs, partial sums folded into FP64); same draws priced by the FP64 drop-in."""
    base = dict(S0=100.0, v0=0.04, q=q, scheme=qk.ANDERSEN_QE, n_steps=100, n_paths=n_paths, seed=11,
                payoffs=[qk.payoff(qk.AMERICAN, right, 100.0)], lsm_basis=qk.LSM_POLY_SV, lsm_dates=dates)
    p64 = qk.price_plain(qk.make_contract(precision=qk.FP64, **base), None, handle)["legs"][0]
    p32 = qk.price_batch([qk.make_contract(precision=qk.FP32, **base)], None, handle)[0]["legs"][0]
    assert abs(p64["price"] - p32["price"]) < 0.25 * p64["std_error"], (p32, p64)
    assert p32["std_error"] == pytest.approx(p64["std_error"], rel=0.02)
    euro = qk.price_plain(qk.make_contract(precision=qk.FP64, **{**base, "payoffs": [qk.payoff(0, right, 100.0)]}),
                          None, handle)["legs"][0]
    assert p64["price"] >= euro["price"] - 2.0 * euro["std_error"]  # early exercise adds value


@pytest.mark.parametrize("model,scheme", [(0, 0), (0, 1), (0, 2), (1, 0), (1, 1), (1, 2)])
def test_prices_vs_closed_form(qk, handle, oracle, model, scheme):
    """European call within 3 SE of the Gil-Pelaez price (HestonTest/BatesTest parameters, 512 steps)."""
    d = load("reference_tests.json")["heston_call_rouah_p28"]["params"]
    k = qk.make_contract(S0=100.0, v0=d["v0"], r=d["r"], q=d["q"], model=model, scheme=scheme, kappa=d["kappa"],
                         theta=d["theta"], sigma=d["sigma"], rho=d["rho"], lambda_j=0.11 if model else 0.0,
                         mu_j=-0.15, sigma_j=0.11, T=0.5, n_steps=512, n_paths=1_000_000, seed=2026,
                         precision=qk.FP32, payoffs=[qk.payoff(0, 0, 100.0)])
    exact = oracle.exact_call(2 if model else 1, k)
    got = qk.price_batch([k], None, handle)[0]["legs"][0]
    assert abs(got["price"] - exact) <= 3.0 * got["std_error"], (got, exact)


@pytest.mark.parametrize("model,scheme", [(0, 0), (0, 1), (0, 2), (1, 0), (1, 1), (1, 2)])
def test_black_scholes_limit(qk, handle, oracle, model, scheme):
    """include/tests/Options/BlackScholesTest.hpp: kappa = theta = sigma = 0 (and no jumps) leaves
    the variance at v0, so every model and scheme prices the Black-Scholes call within 3 SE."""
    k = qk.make_contract(S0=100.0, v0=0.04, r=0.04, q=0.0, model=model, scheme=scheme, kappa=0.0, theta=0.0,
                         sigma=0.0, rho=0.0, lambda_j=0.0, T=1.0, n_steps=64, n_paths=1_000_000, seed=31,
                         precision=qk.FP32, payoffs=[qk.payoff(qk.EUROPEAN, qk.CALL, 100.0)])
    exact = oracle.exact_call(0, k)
    got = qk.price_batch([k], None, handle)[0]["legs"][0]
    assert abs(got["price"] - exact) <= 3.0 * got["std_error"], (got, exact)


def test_american_put_reference_table(qk, handle):
    """include/tests/Options/AmericanOption.hpp: LSM put vs published values, tolerance
    3 SE + max(2% ref, 0.005); Heston implicit Milstein, 1000 steps, 500k paths."""
    d = load("reference_tests.json")["american_put_table"]
    p = d["params"]
    contracts = []
    for S0 in sorted(float(s) for s in d["S0_to_price"]):
        contracts.append(qk.make_contract(S0=S0, v0=p["v0"], r=p["r"], q=p["q"], scheme=qk.IMPLICIT_MILSTEIN,
                                          kappa=p["kappa"], theta=p["theta"], sigma=p["sigma"], rho=p["rho"],
                                          T=p["T"], n_steps=p["n_steps"], n_paths=500_000, seed=88471920573105,
                                          precision=qk.FP32, payoffs=[qk.payoff(qk.AMERICAN, qk.PUT, p["K"])],
                                          lsm_basis=qk.LSM_LAGUERRE3, lsm_dates=0))
    res = qk.price_batch(contracts, None, handle)
    for c, r in zip(contracts, res):
        ref = d["S0_to_price"][str(c.S0)]
        leg = r["legs"][0]
        tol = 3.0 * leg["std_error"] + max(0.02 * ref, 0.005)
        assert abs(leg["price"] - ref) <= tol, (c.S0, leg, ref)


def test_asian_benchmark_published_value(qk, handle):
    """benchmarks/configs/bench_asian_option_price_no_greeks.yaml: 5M paths, 365 QE steps,
    published 5.110195 +- 0.003025; ours within 3 combined SE (different random streams)."""
    d = load("reference_tests.json")["asian_benchmark"]
    p = d["params"]
    k = qk.make_contract(S0=p["S0"], v0=p["v0"], r=p["r"], q=p["q"], scheme=qk.ANDERSEN_QE, kappa=p["kappa"],
                         theta=p["theta"], sigma=p["sigma"], rho=p["rho"], T=p["T"], n_steps=p["n_steps"],
                         n_paths=p["n_paths"], seed=88471920573105, precision=qk.FP32,
                         payoffs=[qk.payoff(qk.ASIAN, qk.CALL, p["K"])])
    leg = qk.price_batch([k], None, handle)[0]["legs"][0]
    assert within_se(leg["price"], d["price"], leg["std_error"], d["std_error"], 3.0), leg
    assert leg["prob_itm"] * 100 == pytest.approx(d["prob_itm_pct"], abs=0.3)


def test_no_noise_drift_all_pairs(qk, handle):
    """include/tests/Options/NoNoiseTest.hpp: sigma = kappa = theta = v0 = 0 => S_T = S0 e^{(r-q)T}
    on every path (tol 1e-8 FP64, 5e-3 FP32)."""
    want = 100.0 * math.exp((0.05 - 0.02) * 1.0)
    for model in (0, 1):
        for scheme in (0, 1, 2):
            for prec, tol in ((qk.FP64, 1e-8), (qk.FP32, 5e-3)):
                k = qk.make_contract(S0=100.0, v0=0.0, r=0.05, q=0.02, model=model, scheme=scheme, kappa=0.0,
                                     theta=0.0, sigma=0.0, rho=0.0, lambda_j=0.0, mu_j=0.0, sigma_j=0.0, T=1.0,
                                     n_steps=365, n_paths=100, precision=prec)
                S, _ = qk.paths(k, 0, 100, handle)
                assert np.all(np.abs(S[:, -1] - want) <= tol), (model, scheme, prec)


def test_normal_draw_moments(qk, handle):
    """GaussianRNGenTest: mean within 0.005 of 0 and variance within 0.01 of 1, recovered
    exactly from constant-variance paths (rho = 0, kappa = sigma = 0: log S increments are
    -v dt/2 + sqrt(v dt) Z2)."""
    v, n, T = 0.04, 64, 1.0
    k = qk.make_contract(S0=1.0, v0=v, r=0.0, q=0.0, kappa=0.0, theta=0.0, sigma=0.0, rho=0.0, T=T, n_steps=n,
                         n_paths=200_000, precision=qk.FP64, normalize=False)
    S, _ = qk.paths(k, 0, 200_000, handle)
    dt = T / n
    logs = np.diff(np.log(np.concatenate([np.ones((S.shape[0], 1)), S], axis=1)), axis=1)
    Z = (logs + 0.5 * v * dt) / math.sqrt(v * dt)
    assert abs(Z.mean()) < 0.005 and abs(Z.var() - 1.0) < 0.01
    assert abs(np.mean(Z ** 3)) < 0.02 and abs(np.mean(Z ** 4) - 3.0) < 0.05


def test_put_call_parity_greeks(qk, handle):
    """include/tests/Options/PutCallParityTest.hpp structural parities (QE, daily steps, 1e6 paths)."""
    K, T, r = 100.0, 1.0, 0.05
    base = dict(S0=100.0, v0=0.04, r=r, q=0.0, scheme=qk.ANDERSEN_QE, T=T, n_steps=365, n_paths=1_000_000,
                seed=184467440737095, precision=qk.FP32)
    g = qk.make_greeks(qk.GREEK_ALL, bump_S_rel=0.02, bump_vol=0.03, bump_r_abs=0.005, bump_T_abs=7.0 / 365.0)
    call, put = qk.price_batch([qk.make_contract(payoffs=[qk.payoff(0, 0, K)], **base),
                                qk.make_contract(payoffs=[qk.payoff(0, 1, K)], **base)], g, handle)
    C, P = call["legs"][0], put["legs"][0]
    se = C["std_error"]
    disc = math.exp(-r * T)

    def tol(scale, mult):  # compute_greek_tol (PutCallParityTest.hpp:120-132)
        return max(0.01 * max(abs(scale), 1.0), mult * se, 1e-4)

    assert abs(C["delta"] - P["delta"] - 1.0) <= tol(1.0, 3.3)
    assert abs(C["gamma"] - P["gamma"]) <= tol(1.0, 3.3)
    assert abs(C["vega"] - P["vega"]) <= tol(1.0, 3.3)
    assert abs(C["vanna"] - P["vanna"]) <= tol(1.0, 3.3)
    assert abs(C["rho"] - P["rho"] - K * T * disc) <= tol(K * T * disc, 3.3)
    assert abs(C["theta"] - P["theta"] + r * K * disc) <= tol(r * K * disc, 5.0)


def test_invalid_contract_raises(qk, handle):
    k = qk.make_contract()
    k.payoffs[0].strike = -1.0
    with pytest.raises(ValueError, match="StrikePrice"):
        qk.price_batch([k], None, handle)
    k = qk.make_contract(n_paths=0)
    with pytest.raises(ValueError, match="N_Paths"):
        qk.price_plain(k, None, handle)


def test_timing_and_launch_count(qk, handle):
    ks = [qk.make_contract(n_paths=100_000, seed=i + 1) for i in range(16)]
    qk.price_batch(ks, qk.make_greeks(qk.GREEK_ALL), handle)
    t = handle.last_timing()
    assert t["launches"] == 3  # one persistent path kernel + the two-level merge for 16 contracts x 12 tasks
    assert t["device_ms"] > 0 and t["path_steps"] == pytest.approx(16 * 12 * 100_000 * 252)
    qk.price_plain(ks[0], qk.make_greeks(qk.GREEK_ALL), handle)
    assert handle.last_timing()["launches"] == 12 + 2  # one FP64 launch per task, then the two-level merge


@pytest.mark.parametrize("model,scheme", [(0, 2), (1, 2), (1, 0)])
def test_antithetic_pairs_match_oracle(qk, handle, oracle, model, scheme):
    """Antithetic pairs (not in the reference): pair k shares path k's draws, its second member
    with every normal negated; estimates over pair averages, against the oracle's pairs."""
    base = dict(model=model, scheme=scheme, lambda_j=0.5 if model else 0.0, mu_j=-0.1, sigma_j=0.15, n_steps=48,
                n_paths=20_000, seed=2024, payoffs=_legs(qk, ALL_LEGS[:8]), antithetic=True)
    k = qk.make_contract(precision=qk.FP64, **base)
    got = qk.price_plain(k, None, handle)["legs"]
    want = oracle.price(k)["legs"]
    for a, b in zip(got, want):
        assert a["price"] == pytest.approx(b["price"], rel=1e-9, abs=1e-12), (a, b)
        assert a["std_error"] == pytest.approx(b["std_error"], rel=1e-6, abs=1e-12)
        assert a["prob_itm"] == pytest.approx(b["prob_itm"], rel=1e-9, abs=1e-12)
    k32 = qk.make_contract(precision=qk.FP32, **base)
    for a, b in zip(qk.price_batch([k32], None, handle)[0]["legs"], oracle.price(k32)["legs"]):
        assert abs(a["price"] - b["price"]) <= 0.05 * b["std_error"] + 1e-7, (a, b)


def test_antithetic_greeks_match_oracle(qk, handle, oracle):
    g = qk.make_greeks(qk.GREEK_ALL, bump_S_rel=0.01, bump_vol=0.02, bump_r_abs=0.001, bump_T_abs=7 / 365)
    k = qk.make_contract(scheme=qk.ANDERSEN_QE, n_steps=32, n_paths=20_000, seed=4242, precision=qk.FP64,
                         payoffs=[qk.payoff(qk.ASIAN, qk.CALL, 100.0)], antithetic=True)
    got = qk.price_batch([k], g, handle)[0]["legs"][0]
    want = oracle.price(k, g)["legs"][0]
    for f in ("price", "delta", "gamma", "vega", "vomma", "vanna", "rho", "theta"):
        assert got[f] == pytest.approx(want[f], rel=1e-7, abs=1e-9), f


def test_antithetic_reduces_error_and_validates(qk, handle, oracle):
    base = dict(scheme=qk.ANDERSEN_QE, n_steps=64, n_paths=400_000, seed=99, precision=qk.FP32,
                payoffs=[qk.payoff(qk.EUROPEAN, qk.CALL, 100.0)])
    plain = qk.price_batch([qk.make_contract(**base)], None, handle)[0]["legs"][0]
    anti = qk.price_batch([qk.make_contract(antithetic=True, **base)], None, handle)[0]["legs"][0]
    assert anti["std_error"] < 0.8 * plain["std_error"]
    exact = oracle.exact_call(1, qk.make_contract(**base), 200.0)
    assert abs(anti["price"] - exact) <= 3.0 * anti["std_error"] + 5e-3
    with pytest.raises(ValueError, match="even"):
        qk.price_batch([qk.make_contract(antithetic=True, **{**base, "n_paths": 1001})], None, handle)
    with pytest.raises(RuntimeError, match="antithetic"):
        qk.price_batch([qk.make_contract(antithetic=True, **{**base, "payoffs": [qk.payoff(qk.AMERICAN, qk.PUT, 100.0)]})],
                       None, handle)


@pytest.mark.parametrize("model,scheme,lam", [(0, 0, 0.0), (0, 1, 0.0), (0, 2, 0.0), (1, 0, 0.3), (1, 1, 0.3),
                                              (1, 2, 0.3), (1, 0, 25.0), (1, 2, 25.0)])
def test_lane_modes_simulate_the_same_paths(qk, handle, model, scheme, lam):
    """A lane carrying two paths (FP32 Box-Muller, Euler and QE stepped as pairs on the paired
    FP32 pipe, rare code shared by the two paths) and a lane carrying one path simulate
    bit-identical paths: prices agree to the rounding of the FP64 moment merge, whose grouping
    of paths differs between the two shapes.  lam = 25 sends about a quarter of the steps
    through the jump code, often for both paths of a lane at once."""
    legs = [qk.payoff(qk.EUROPEAN, qk.CALL, 100.0), qk.payoff(qk.ASIAN, qk.CALL, 100.0),
            qk.payoff(qk.BARRIER_UP_OUT, qk.CALL, 100.0, 130.0), qk.payoff(qk.BINARY_CASH, qk.CALL, 105.0)]
    c = qk.make_contract(model=model, scheme=scheme, lambda_j=lam, mu_j=-0.05, sigma_j=0.1,
                         sigma=0.5, n_paths=65_537, n_steps=101, seed=5, precision=qk.FP32, payoffs=legs)
    out = []
    try:
        for lanes in (1, 2):
            handle.tune_set(qk.FP32, model, scheme, 24, False, lanes)
            out.append(qk.price_batch([c], None, handle)[0]["legs"])
    finally:
        handle.tune_reset()
    for a, b in zip(out[0], out[1]):
        assert a["price"] == pytest.approx(b["price"], rel=1e-12, abs=1e-15)
        assert a["std_error"] == pytest.approx(b["std_error"], rel=1e-9)
        assert a["prob_itm"] == pytest.approx(b["prob_itm"], rel=1e-12, abs=1e-15)


@pytest.mark.parametrize("model", [0, 1])
def test_qe_near_zero_variance_lane_modes_and_fp64(qk, handle, model):
    """QE with the Feller condition far from holding (vol-of-vol 0.9, long-run variance 0.01,
    kappa 0.5): the variance sits near zero and a large share of steps leaves the quadratic
    regime, often for one path of a lane's pair only.  Two paths per lane and one path per
    lane still simulate bit-identical paths (prices agree to the rounding of the moment
    merge), and the FP32 prices stay within one standard error of the FP64 engine on the same
    draws (three combined SE under Bates, where the two precisions decide jumps from different
    bits)."""
    legs = [qk.payoff(qk.EUROPEAN, qk.PUT, 100.0), qk.payoff(qk.ASIAN, qk.CALL, 100.0),
            qk.payoff(qk.BARRIER_DOWN_OUT, qk.PUT, 100.0, 80.0)]
    base = dict(model=model, scheme=qk.ANDERSEN_QE, v0=0.01, theta=0.01, kappa=0.5, sigma=0.9, rho=-0.7,
                lambda_j=0.2 if model else 0.0, mu_j=-0.05, sigma_j=0.1, n_paths=100_001, n_steps=126, T=0.5,
                seed=21, payoffs=legs)
    c = qk.make_contract(precision=qk.FP32, **base)
    out = []
    try:
        for lanes in (1, 2):
            handle.tune_set(qk.FP32, model, qk.ANDERSEN_QE, 24, False, lanes)
            out.append(qk.price_batch([c], None, handle)[0]["legs"])
    finally:
        handle.tune_reset()
    for a, b in zip(out[0], out[1]):
        assert a["price"] == pytest.approx(b["price"], rel=1e-12, abs=1e-15)
        assert a["std_error"] == pytest.approx(b["std_error"], rel=1e-9)
    r64 = qk.price_batch([qk.make_contract(precision=qk.FP64, **base)], None, handle)[0]["legs"]
    for a, b in zip(out[1], r64):
        assert abs(a["price"] - b["price"]) < (1.0 if model == 0 else 3.0 * 2 ** 0.5) * b["std_error"], (a, b)


def test_edge_sizes_match_oracle(qk, handle, oracle):
    """Ragged and minimal sizes: a single path, partial warps, a single step, an empty request
    list, and the largest path count a contract may have (32-bit Philox path counter)."""
    legs = [qk.payoff(qk.EUROPEAN, qk.CALL, 100.0), qk.payoff(qk.ASIAN, qk.PUT, 100.0),
            qk.payoff(qk.LOOKBACK_FLOATING, qk.CALL, 100.0)]
    for n_paths, n_steps in ((1, 1), (1, 7), (31, 3), (33, 5), (1000, 1)):
        for model, scheme in ((0, 2), (1, 0)):
            k = qk.make_contract(model=model, scheme=scheme, lambda_j=0.5 if model else 0.0, mu_j=-0.1, sigma_j=0.15,
                                 n_paths=n_paths, n_steps=n_steps, seed=99, precision=qk.FP64, payoffs=legs)
            want = oracle.price(k)["legs"]
            for got in (qk.price_plain(k, None, handle)["legs"], qk.price_batch([k], None, handle)[0]["legs"]):
                for a, b in zip(got, want):
                    assert a["price"] == pytest.approx(b["price"], rel=1e-9, abs=1e-12), (n_paths, n_steps, a, b)
                    assert a["prob_itm"] == pytest.approx(b["prob_itm"], rel=1e-12, abs=1e-15)
                    if n_paths > 1:
                        assert a["std_error"] == pytest.approx(b["std_error"], rel=1e-6, abs=1e-12)
                    else:
                        assert a["std_error"] == 0.0
    assert qk.price_batch([], None, handle) == []
    with pytest.raises(ValueError, match="N_Paths"):
        qk.price_batch([qk.make_contract(n_paths=2 ** 32)], None, handle)


def test_lsm_jobs_on_concurrent_lanes_equal_alone(qk, handle):
    """The American jobs of one call (contracts and their Greek bumps) run on several streams at
    once, each with its own working set; every result equals the contract priced alone."""
    cs = []
    for i, (n, prec, basis) in enumerate([(20_000, qk.FP32, 1), (150_000, qk.FP32, 0), (60_000, qk.FP64, 1),
                                          (8_192, qk.FP32, 1), (90_000, qk.FP64, 0)]):
        cs.append(qk.make_contract(S0=100.0, v0=0.04, scheme=qk.ANDERSEN_QE if i % 2 == 0 else qk.EULER,
                                   n_steps=50, n_paths=n, seed=7 + i, stream=i, precision=prec,
                                   payoffs=[qk.payoff(qk.AMERICAN, qk.PUT, 95.0 + 3 * i)], lsm_basis=basis,
                                   lsm_dates=0 if basis == 0 else 10))
    g = qk.make_greeks(qk.GREEK_DELTA_GAMMA, bump_S_rel=0.01)
    together = qk.price_batch(cs, g, handle)
    for c, r in zip(cs, together):
        alone = qk.price_batch([c], g, handle)[0]["legs"][0]
        leg = r["legs"][0]
        for f in ("price", "std_error", "prob_itm", "delta", "gamma"):
            assert leg[f] == pytest.approx(alone[f], rel=1e-12, abs=1e-15), f
