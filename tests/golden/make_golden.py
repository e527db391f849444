"""Generate the golden fixtures in tests/golden/ from the reference's own code.

Run (needs the reference checkout and `python -m quantkos_b200.build`, which
compiles the reference harness into oracle/_ref/):

    python tests/golden/make_golden.py

Fixtures written (all values produced by the reference code compiled against the
host shim, or read from the reference's test sources; paths relative to the
reference project):

* step_cases.json   one-step SDEScheme<M,S>::evolve_step outputs with fed draws, all
                    6 model/scheme pairs, FP64 build and FP32 build
                    (include/core/schemes/markovian/MSchemes.hpp:87-551);
* payoff_cases.json PayoffTracker final payoffs on fed spot sequences, 10 types x 2 rights
                    (include/core/options/Payoff.hpp:84-243);
* lsm_cases.json    LSMEngine::solve_system_on_host_cholesky and LaguerreBasis<4>
                    (include/core/options/LSMAmerican.hpp:157-613);
* analytic.json     Black-Scholes / Heston / Bates closed-form call prices
                    (include/core/analytical/*);
* reference_tests.json  constants the reference's tests pin: the Heston call quoted in
                    include/tests/Options/HestonTest.hpp, the American put table of
                    include/tests/Options/AmericanOption.hpp and the published Asian
                    benchmark result of benchmarks/configs/bench_asian_option_price_no_greeks.yaml,
                    parsed from those files.
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import qkref as R  # noqa: E402

from quantkos_b200.build import REFERENCE_ROOT as REF  # noqa: E402  (QK_REFERENCE_ROOT)

PARAM_SETS = [
    # name, model params (Heston core + jumps), market r, q, dt
    dict(name="config0", kappa=2.0, theta=0.04, sigma=0.3, rho=-0.7, lambda_j=0.1, mu_j=-0.05, sigma_j=0.10,
         r=0.03, q=0.0, dt=1.0 / 252),
    dict(name="rouah_p28", kappa=5.0, theta=0.05, sigma=0.5, rho=-0.8, lambda_j=0.11, mu_j=-0.15, sigma_j=0.11,
         r=0.03, q=0.02, dt=0.5 / 64),
    dict(name="rouah_p212", kappa=5.0, theta=0.16, sigma=0.9, rho=0.1, lambda_j=25.0, mu_j=-0.1, sigma_j=0.15,
         r=0.1, q=0.0, dt=0.25 / 1000),
    dict(name="high_volvol", kappa=0.7, theta=0.02, sigma=1.2, rho=-0.9, lambda_j=40.0, mu_j=0.05, sigma_j=0.3,
         r=0.05, q=0.03, dt=1.0 / 52),
    dict(name="degenerate", kappa=0.0, theta=0.0, sigma=0.0, rho=0.0, lambda_j=0.0, mu_j=0.0, sigma_j=0.0,
         r=0.05, q=0.02, dt=1.0 / 365),
]
UMAX = 8


def step_cases(rng: np.random.Generator) -> list[dict]:
    out = []
    for ps in PARAM_SETS:
        for model in (0, 1):
            for scheme in (0, 1, 2):
                n = 20
                S_in = np.exp(rng.normal(0.0, 0.3, n))
                v_in = rng.uniform(0.0005, 0.25, n)
                v_in[:4] = [0.0, 1e-9, 1e-6, 1e-4]
                z = rng.standard_normal((n, 3))
                z[4:8, 0] = [-4.0, 4.0, -2.5, 3.0]
                u = rng.uniform(0.0, 1.0, (n, UMAX))
                u = np.clip(u, 1e-6, 1.0 - 1e-6)
                for i in range(n):
                    cfg = R.config(S0=float(S_in[i]), v0=float(v_in[i]), r=ps["r"], q=ps["q"], model=model,
                                   scheme=scheme, kappa=ps["kappa"], theta=ps["theta"], sigma=ps["sigma"],
                                   rho=ps["rho"], lambda_j=ps["lambda_j"], mu_j=ps["mu_j"], sigma_j=ps["sigma_j"],
                                   T=ps["dt"], dt_in=ps["dt"])
                    case = dict(set=ps["name"], model=model, scheme=scheme, S=float(S_in[i]), v=float(v_in[i]),
                                r=ps["r"], q=ps["q"], kappa=ps["kappa"], theta=ps["theta"], sigma=ps["sigma"],
                                rho=ps["rho"], lambda_j=ps["lambda_j"], mu_j=ps["mu_j"], sigma_j=ps["sigma_j"],
                                dt=ps["dt"], z=z[i].tolist(), u=u[i].tolist())
                    ok = True
                    for rb, tag in ((8, "64"), (4, "32")):
                        try:
                            S1, v1, used = R.step_trace(rb, cfg, z[i:i + 1], u[i:i + 1])
                        except RuntimeError:
                            ok = False
                            break
                        case["S_out" + tag] = float(S1[0])
                        case["v_out" + tag] = float(v1[0])
                        case["used" + tag] = int(used[0])
                    if ok:
                        out.append(case)
    return out


def payoff_cases(rng: np.random.Generator) -> list[dict]:
    out = []
    for t in range(10):
        for right in (0, 1):
            for rep in range(6):
                n = int(rng.integers(1, 40))
                S = np.exp(np.cumsum(rng.normal(0.0, 0.04, n)))
                S0 = 1.0
                K = float(rng.uniform(0.85, 1.15))
                B = float(rng.choice([0.9, 0.95, 1.05, 1.1, 1.2]))
                val = R.payoff(t, right, S, S0, K, B, 8)
                out.append(dict(type=t, right=right, S=S.tolist(), S0=S0, K=K, B=B, payoff=val))
    return out


def lsm_cases(rng: np.random.Generator) -> dict:
    solves = []
    for rep in range(24):
        nb = 4
        count = float(rng.integers(0, 2000)) if rep % 6 else float(rng.integers(0, 4))
        X = rng.uniform(0.5, 1.0, int(max(count, 1)))
        L = np.stack([R.laguerre(float(x), nb) for x in X])
        Y = rng.uniform(0.0, 0.5, len(X))
        M = L.T @ L
        B = L.T @ Y
        if rep % 8 == 7:  # rank-deficient: duplicate column
            M = np.ones((nb, nb)) * M[0, 0]
        C = R.lsm_solve(M, B, count)
        solves.append(dict(M=M.ravel().tolist(), B=B.tolist(), count=count, C=C.tolist()))
    lag = []
    for x in np.linspace(0.0, 3.0, 31):
        lag.append(dict(X=float(x), L=R.laguerre(float(x), 4).tolist()))
    return dict(solves=solves, laguerre=lag)


def analytic() -> list[dict]:
    out = []
    sets = [
        dict(S0=100.0, K=100.0, T=0.5, v0=0.05, r=0.03, q=0.02, kappa=5.0, theta=0.05, sigma=0.5, rho=-0.8,
             lambda_j=0.11, mu_j=-0.15, sigma_j=0.11),
        dict(S0=100.0, K=100.0, T=1.0, v0=0.04, r=0.03, q=0.0, kappa=2.0, theta=0.04, sigma=0.3, rho=-0.7,
             lambda_j=0.1, mu_j=-0.05, sigma_j=0.10),
        dict(S0=100.0, K=90.0, T=2.0, v0=0.09, r=0.01, q=0.01, kappa=1.0, theta=0.06, sigma=0.6, rho=-0.3,
             lambda_j=0.5, mu_j=-0.1, sigma_j=0.2),
        dict(S0=100.0, K=115.0, T=0.25, v0=0.02, r=0.05, q=0.0, kappa=3.0, theta=0.03, sigma=0.2, rho=-0.5,
             lambda_j=0.2, mu_j=0.02, sigma_j=0.05),
    ]
    for s in sets:
        cfg = R.config(S0=s["S0"], K=s["K"], T=s["T"], v0=s["v0"], r=s["r"], q=s["q"], kappa=s["kappa"],
                       theta=s["theta"], sigma=s["sigma"], rho=s["rho"], lambda_j=s["lambda_j"], mu_j=s["mu_j"],
                       sigma_j=s["sigma_j"], dt_in=s["T"] / 10)
        d = dict(s)
        d["bs"] = R.exact_call(cfg, 0)
        d["heston"] = R.exact_call(cfg, 1)
        d["bates"] = R.exact_call(cfg, 2)
        out.append(d)
    return out


def reference_tests() -> dict:
    heston_src = (REF / "include/tests/Options/HestonTest.hpp").read_text()
    m = re.search(r"Expected European call price\s*:\s*([0-9.]+)", heston_src)
    american_src = (REF / "include/tests/Options/AmericanOption.hpp").read_text()
    table = {float(a): float(b) for a, b in re.findall(r"\{\s*([0-9.]+)\s*,\s*([0-9.]+)\s*\}", american_src)}
    bench_src = (REF / "benchmarks/configs/bench_asian_option_price_no_greeks.yaml").read_text()
    price = float(re.search(r"Estimated Option Price:\s*([0-9.]+)", bench_src).group(1))
    se = float(re.search(r"Statistical Std Error:\s*([0-9.]+)", bench_src).group(1))
    itm = float(re.search(r"Probability of ITM:\s*([0-9.]+)", bench_src).group(1))
    return {
        "heston_call_rouah_p28": {"price": float(m.group(1)), "source": "include/tests/Options/HestonTest.hpp:50-51",
                                  "params": dict(S0=100.0, K=100.0, T=0.5, v0=0.05, r=0.03, q=0.02, kappa=5.0,
                                                 theta=0.05, sigma=0.5, rho=-0.8)},
        "american_put_table": {"S0_to_price": {str(k): v for k, v in sorted(table.items())},
                               "source": "include/tests/Options/AmericanOption.hpp:115-121",
                               "tolerance": "3*SE + max(0.02*ref, 0.005) (AmericanOption.hpp:153-158)",
                               "params": dict(K=10.0, T=0.25, v0=0.0625, r=0.1, q=0.0, kappa=5.0, theta=0.16,
                                              sigma=0.9, rho=0.1, n_steps=1000, scheme="ImplicitMilstein")},
        "asian_benchmark": {"price": price, "std_error": se, "prob_itm_pct": itm,
                            "source": "benchmarks/configs/bench_asian_option_price_no_greeks.yaml:21-67",
                            "params": dict(S0=100.0, K=100.0, T=1.0, v0=0.05, r=0.03, q=0.02, kappa=5.0,
                                           theta=0.05, sigma=0.5, rho=-0.8, n_steps=365, n_paths=5_000_000,
                                           scheme="AndersonQE", type="Asian", right="Call")},
    }


def main() -> None:
    if not R.available():
        raise SystemExit("oracle/_ref not built; run python -m quantkos_b200.build with the reference present")
    rng = np.random.default_rng(20261203)
    (HERE / "step_cases.json").write_text(json.dumps(step_cases(rng)))
    (HERE / "payoff_cases.json").write_text(json.dumps(payoff_cases(rng)))
    (HERE / "lsm_cases.json").write_text(json.dumps(lsm_cases(rng)))
    (HERE / "analytic.json").write_text(json.dumps(analytic(), indent=1))
    (HERE / "reference_tests.json").write_text(json.dumps(reference_tests(), indent=1))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
