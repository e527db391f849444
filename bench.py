#!/usr/bin/env python3
"""Benchmark of the Monte Carlo hot path on B200.

Workload (one "step" = one full pricing of it): a Bates model under Andersen QE
(psi_c = 1.5), 16,777,216 paths x 252 daily steps, FP32 stepping with FP64
accumulation, five payoffs priced in one pass (European call K=100, arithmetic
Asian call K=100, up-and-out call K=100 B=130 daily monitoring, floating-strike
lookback put, cash-or-nothing binary call K=105 paying 1); S0=100, T=1, r=0.03,
q=0, v0=0.04, kappa=2, theta=0.04, sigma=0.3, rho=-0.7, lambda=0.1, muJ=-0.05,
sigmaJ=0.10.  Synthetic: the inputs are these parameters; paths come from Philox.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

For N > 1 launch with torchrun (one process per GPU); every rank prices its own
contract on its own Philox stream (weak scaling, no data-path collective); the
timed region is bracketed by a barrier and device syncs and the max over ranks is
reported.  Prints ONE JSON line on rank 0.

At N = 1 the line also carries the other workloads, each with its own clock
record: `batch_4096` (the 4096-contract mix with all seven Greeks, batched FP32
engine against the plain FP64 drop-in on every contract), `serve` /
`serve_sub_capacity` (Poisson request streams at 2,000 and 1,000 requests/s, 30%
American puts) and `serve_vs_plain` (one stream at 200 requests/s served by the
batched engine and by the plain FP64 method behind the same server: latency at equal
load).  `--no-extra` leaves them out.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_PATHS = 16_777_216
N_STEPS = 252
WORKLOAD = "bates_qe_5payoff_16777216x252_fp32"
METRIC = "path-steps/s"
# Algorithmic SFU (MUFU) work per path-step of the fused Bates-QE kernel, counted
# from the step formulas as implemented, quadratic QE branch (taken by nearly every
# step at these parameters): Box-Muller lg2, sqrt, sin, cos; QE rcp(s2),
# sqrt(x(x-1)), rcp(1+b2), sqrt(b2), rcp(term), lg2(term); spot update
# sqrt(K3 v + K4 v'), ex2.  The SFU pipe (16 lanes/clk/SM) then bounds the kernel
# at (measured SFU op rate) / 12 path-steps/s; the FP32/integer work (Philox, the
# QE algebra) fits under that bound on the 128-lane issue.
SFU_PER_STEP = 12.0
# Algorithmic scalar lane operations per path-step of the FP32 kinds (from the formulas
# as implemented; one-path-per-lane count), for the issue-slot bound (every operation,
# SFU ones included, takes an issue slot; an SM issues 4 warp instructions = 128 lane
# operations per cycle, 8 times its 16 SFU lanes):
#   Philox4x32-10: half a call per step (a call = 4 words = two steps' normal pairs):
#     10 rounds x (2 wide multiplies + 2 three-input XORs) / 2 = 20
#   Box-Muller per pair: 2 uniform conversions x 2, the log and angle scalings, 2 products
#     = 8 (+ 4 SFU: lg2, sqrt, sin, cos)
#   step: Euler 10 (+2 SFU: sqrt v, ex2), Milstein 14 (+2), QE quadratic 30 (+8: 3 rcp,
#     3 sqrt, lg2, ex2)
#   Bates: the one-compare jump test, 5; loop and counters, 3
ISSUE_OPS = {"philox": 20, "box_muller": 8, "step": {"euler": 10, "milstein": 14, "qe": 30}, "bates": 5, "loop": 3}
SFU_OPS = {"box_muller": 4, "step": {"euler": 2, "milstein": 2, "qe": 8}}


def algorithmic_ops(scheme: str, bates: bool) -> tuple[int, int]:
    """(SFU operations, issue-slot operations incl. SFU) per path-step of one FP32 kind."""
    sfu = SFU_OPS["box_muller"] + SFU_OPS["step"][scheme]
    other = ISSUE_OPS["philox"] + ISSUE_OPS["box_muller"] + ISSUE_OPS["step"][scheme] + ISSUE_OPS["loop"]
    if bates:
        other += ISSUE_OPS["bates"]
    return sfu, sfu + other
DRAM_BYTES_PER_PATH_STEP = 2.09e6 / (1_048_576 * 252)
L2_FLUSH_BYTES = 256 << 20


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-sample-paths", type=int, default=1 << 16,
                    help="reference arm: paths per timed step (each step is a bounded sample of the workload)")
    ap.add_argument("--cpu-baseline-paths", type=int, default=1 << 21,
                    help="cpu_baseline leg of our arm: paths of the one timed sample (about 10-30 s of CPU work)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison run")
    ap.add_argument("--skip-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shape")
    ap.add_argument("--shape", default=None,
                    help="launch shape 'tiles_per_warp,guided_tail,paths_per_lane' instead of the autotuner")
    ap.add_argument("--paths", type=int, default=N_PATHS,
                    help="paths per contract (the workload uses 16,777,216; smaller only for profiling captures)")
    ap.add_argument("--workload", choices=["bates5", "plain", "lsm", "batch", "serve", "kinds", "attribution",
                                           "published_asian"],
                    default="bates5",
                    help="bates5 (default): the headline line; the others measure the remaining workloads")
    ap.add_argument("--subset", type=int, default=128, help="batch: contracts priced by both engines")
    ap.add_argument("--requests", type=int, default=20_000, help="serve: number of requests")
    ap.add_argument("--rate", type=float, default=2000.0, help="serve: Poisson arrival rate (requests/s)")
    ap.add_argument("--lanes", type=int, default=0, help="serve: server lanes (0 = the library default)")
    ap.add_argument("--wave-ms", type=float, default=0.0, help="serve: wave budget in ms (0 = the library default)")
    ap.add_argument("--serve-plain", action="store_true",
                    help="serve: price every request alone with the plain FP64 method behind the same server")
    ap.add_argument("--no-extra", action="store_true",
                    help="default line without the 4096-contract batch and serving records")
    ap.add_argument("--batch-compare", type=int, default=4096,
                    help="default line: contracts of the mix priced by both engines (4096 = all)")
    return ap.parse_args()


def workload_contract(qk, rank: int = 0, precision=None, n_paths: int = N_PATHS):
    legs = [qk.payoff(qk.EUROPEAN, qk.CALL, 100.0), qk.payoff(qk.ASIAN, qk.CALL, 100.0),
            qk.payoff(qk.BARRIER_UP_OUT, qk.CALL, 100.0, 130.0), qk.payoff(qk.LOOKBACK_FLOATING, qk.PUT, 100.0),
            qk.payoff(qk.BINARY_CASH, qk.CALL, 105.0)]
    return qk.make_contract(S0=100.0, v0=0.04, r=0.03, q=0.0, model=qk.BATES, scheme=qk.ANDERSEN_QE, kappa=2.0,
                            theta=0.04, sigma=0.3, rho=-0.7, lambda_j=0.1, mu_j=-0.05, sigma_j=0.10, psi_c=1.5,
                            T=1.0, n_steps=N_STEPS, n_paths=n_paths, seed=42, stream=rank,
                            precision=qk.FP32 if precision is None else precision, payoffs=legs)


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = Path(tempfile.mkstemp(prefix="qk_clocks_", suffix=".csv")[1])

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, max_mhz_hint: float) -> dict:
        rows = []
        try:
            for line in self.path.read_text().splitlines():
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].replace(".", "").isdigit():
                    rows.append(f)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": max_mhz_hint, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows]
        mx = max(float(r[2]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [s for s in sm if s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit()) if rows else None}


# ----------------------------------------------------------------------------- CPU / reference leg
def cpu_reference_rate(sample_paths: int, repeats: int = 1) -> dict:
    """The reference's own pricing path on the host cores (oracle/_ref: reference headers over the
    OpenMP host shim), one run per payoff leg as the reference prices one payoff per run; falls back
    to the C restatement (oracle/qk_oracle.c, all legs in one pass) when the reference was not built."""
    from oracle import qkref
    cores = os.cpu_count() or 1
    legs = [(0, 0, 100.0, 100.0), (1, 0, 100.0, 100.0), (2, 0, 100.0, 130.0), (6, 1, 100.0, 100.0),
            (8, 0, 105.0, 100.0)]
    if qkref.available():
        total = 0.0
        for _ in range(repeats):
            for t, r, K, B in legs:
                cfg = qkref.config(S0=100.0, v0=0.04, r=0.03, q=0.0, opt_type=t, opt_right=r, K=K, B=B, model=1,
                                   scheme=2, kappa=2.0, theta=0.04, sigma=0.3, rho=-0.7, lambda_j=0.1, mu_j=-0.05,
                                   sigma_j=0.10, T=1.0, dt_in=1.0 / N_STEPS, n_paths=sample_paths, seed=42,
                                   max_cpu_ram_mb=64000)
                t0 = time.perf_counter()
                qkref.price(cfg, 8)
                total += time.perf_counter() - t0
        kind = "reference"
        sample = (f"{sample_paths} paths x {N_STEPS} steps, 5 reference runs (one per payoff leg, FP64, "
                  f"OpenMP over the host shim)")
    else:
        import quantkos_b200 as qk
        from oracle import qkoracle
        k = workload_contract(qk, 0, qk.FP64, sample_paths)
        t0 = time.perf_counter()
        for _ in range(repeats):
            qkoracle.price(k)
        total = time.perf_counter() - t0
        kind = "port"
        sample = f"{sample_paths} paths x {N_STEPS} steps, C restatement, all legs in one pass, FP64"
    value = repeats * sample_paths * N_STEPS / total
    return {"value": value, "unit": METRIC, "cores": cores, "kind": kind, "sample": sample, "seconds": total}


def run_reference_arm(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    for _ in range(args.warmup):
        cpu_reference_rate(args.cpu_sample_paths)
    r = cpu_reference_rate(args.cpu_sample_paths, repeats=args.steps)
    ms_per_step = 1e3 * r["seconds"] / args.steps
    line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample_paths": args.cpu_sample_paths, "n_steps": N_STEPS,
                       "note": "bounded sample of the workload per step"},
            "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": r["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- our arm
# ----------------------------------------------------------------------------- other workloads
def _timed(torch, ext, fn, steps: int, flush=None) -> list[float]:
    """Device-time (CUDA events on the engine stream) of `steps` calls of fn, L2 flushed between."""
    out = []
    for i in range(steps):
        if flush is not None:
            flush.fill_(float(i))
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(ext)
        fn()
        b.record(ext)
        torch.cuda.synchronize()
        out.append(a.elapsed_time(b))
    return out


def _shape_summary(tuned) -> list[dict]:
    return [{k: r[k] for k in ("precision", "model", "scheme", "tiles_per_warp", "guided_tail", "paths_per_lane")}
            for r in tuned]


def _max_mhz() -> float:
    pk = ROOT / "MEASURED_PEAKS.json"
    return json.loads(pk.read_text()).get("sm_max_mhz", 1965.0) if pk.exists() else 1965.0


def measure_batch_mix(qk, W, h, torch, ext, flush, subset: int | None = None, autotune: bool = True) -> dict:
    """The 4096-contract mixed workload with all seven Greeks (49,152 pricing tasks):
    one timed pricing by the batched FP32 engine (one persistent launch per kernel kind)
    and one by the plain FP64 drop-in (one contract per launch sequence), on all the
    contracts or the first `subset`, on the same Philox draws.  Reports contracts/s of
    both, their ratio at equal standard error, the share of FP32 prices within 3 SE
    of the FP64 ones, and the FP32-minus-FP64 Greeks in units of a conservative
    finite-difference SE bound."""
    g = W.batch_greeks()
    full = W.mixed_batch()
    n_cmp = len(full) if subset is None else min(subset, len(full))
    tuned = h.autotune(full[:256], g, reps=1) if autotune else []  # launch shapes per kind (untimed)
    cmp32 = full[:n_cmp]
    cmp64 = W.mixed_batch(n_cmp, precision=qk.FP64)
    qk.price_batch(cmp32[:64], g, h)
    qk.price_plain(cmp64[0], g, h)
    res32: list = []
    res64: list = []
    sampler = ClockSampler(0)
    with sampler:
        t_full = _timed(torch, ext, lambda: res32.__init__(qk.price_batch(full, g, h)), 1, flush)[0]
        tf = h.last_timing()
        if n_cmp < len(full):
            t_cmp32 = _timed(torch, ext, lambda: res32.__init__(qk.price_batch(cmp32, g, h)), 1, flush)[0]
        else:
            t_cmp32 = t_full

        def plain_all():
            res64.clear()
            for c in cmp64:
                res64.append(qk.price_plain(c, g, h))

        t_plain = _timed(torch, ext, plain_all, 1, flush)[0]
    res32 = res32[:n_cmp]
    se_ratio = statistics.mean(a["legs"][0]["std_error"] / b["legs"][0]["std_error"]
                               for a, b in zip(res32, res64) if b["legs"][0]["std_error"] > 0)
    dev = [abs(a["legs"][0]["price"] - b["legs"][0]["price"]) / b["legs"][0]["std_error"]
           for a, b in zip(res32, res64) if b["legs"][0]["std_error"] > 0]
    within = sum(d <= 3.0 for d in dev) / len(dev)
    # Heston contracts follow the same paths in both precisions (the difference is rounding);
    # under Bates the FP32 jump decision reads other bits than the FP64 one, so jump times
    # differ and the two estimates are partly independent: compared in combined SE
    comb = {"heston": [], "bates": []}
    for c, a, b in zip(cmp64, res32, res64):
        la, lb = a["legs"][0], b["legs"][0]
        s = math.hypot(la["std_error"], lb["std_error"])
        if s > 0:
            comb["bates" if c.model == qk.BATES else "heston"].append(abs(la["price"] - lb["price"]) / s)
    all_comb = comb["heston"] + comb["bates"]

    # Greeks: same draws on both sides, so the difference is precision, not sampling;
    # in units of sd(X - Y) <= sd(X) + sd(Y) with every bumped price at the base SE
    def se_bound(c, se, f):
        hs = c.S0 * g.bump_S_rel
        hv = c.v0 * g.bump_vol if g.vega_mode == 1 else g.bump_vol
        return {"delta": se / hs, "gamma": 4 * se / hs ** 2, "vega": se / hv, "vomma": 4 * se / hv ** 2,
                "vanna": se / (hs * hv), "rho": se / g.bump_r_abs, "theta": 2 * se / g.bump_T_abs}[f]

    greek_err = {}
    for f in ("delta", "gamma", "vega", "vomma", "vanna", "rho", "theta"):
        rel, in_se = [], []
        for c, a, b in zip(cmp64, res32, res64):
            la, lb = a["legs"][0], b["legs"][0]
            d = abs(la[f] - lb[f])
            rel.append(d / max(abs(lb[f]), 1e-12))
            bound = se_bound(c, lb["std_error"], f)
            if bound > 0:
                in_se.append(d / bound)
        greek_err[f] = {"median_rel": statistics.median(rel), "median_in_se_bound": statistics.median(in_se),
                        "max_in_se_bound": max(in_se)}
    ps = W.path_steps(full, g)
    batched_cps = n_cmp / (t_cmp32 * 1e-3)
    plain_cps = n_cmp / (t_plain * 1e-3)
    return {"workload": "mixed_4096_contracts_all_greeks_seed123", "contracts": len(full), "pricing_tasks": 12 * len(full),
            "path_steps": ps, "batched_ms": t_full, "contracts_per_s": len(full) / (t_full * 1e-3),
            "path_steps_per_s": ps / (t_full * 1e-3), "gpu_launches": tf["launches"],
            "compared_contracts": n_cmp, "plain_fp64_ms": t_plain,
            "batched_fp32_contracts_per_s": batched_cps, "plain_fp64_contracts_per_s": plain_cps,
            "mean_se_ratio_batched_over_plain": se_ratio,
            # contracts/s ratio at equal SE: the batched engine would need (SE ratio)^2 the paths
            "speedup_vs_plain_fp64_at_equal_se": batched_cps / plain_cps / (se_ratio * se_ratio),
            "prices_within_3se_of_fp64": within, "max_price_diff_in_fp64_se": max(dev),
            "prices_within_3_combined_se": sum(d <= 3.0 for d in all_comb) / len(all_comb),
            "max_price_diff_in_combined_se": {k: max(v) if v else None for k, v in comb.items()},
            "greeks_fp32_minus_fp64": greek_err, "autotune": _shape_summary(tuned),
            "clocks": sampler.summary(_max_mhz())}


def measure_serving(qk, W, h, torch, ext, flush, rate: float, n_requests: int, plain_sample: int = 0,
                    lanes: int = 0, wave_ms: float = 0.0, plain_fp64: bool = False) -> dict:
    """A Poisson stream of `n_requests` pricing requests at `rate` per second (30% American
    puts by LSM) submitted in real time to the continuous-batching server started on h;
    latency is submit to completion.  Optionally the plain FP64 one-contract-per-launch
    method and the batched engine on the first `plain_sample` requests, for throughput
    at equal standard error."""
    import ctypes as C

    from quantkos_b200 import _lib as L
    import threading

    arrivals, contracts = W.serving_stream(n_requests, rate_per_s=rate)
    srv = qk.Server(h, 0, 512, lanes, wave_ms, plain_fp64=plain_fp64)
    # warm the server that is measured: its lanes' device arenas grow to the sizes the
    # stream's largest requests need (one at a time, so every lane takes some), untimed;
    # the statistics below cover the stream's own tickets only
    by_cost = sorted(range(len(contracts)), key=lambda i: -contracts[i].n_paths * contracts[i].n_steps)
    big = [contracts[i] for i in by_cost[:32]]
    for tk in [srv.submit(c) for c in big]:  # all at once: the lanes share them
        srv.poll(tk, 600_000)
    warm = big + big + contracts[:32]
    for c in warm[len(big):]:  # then one at a time
        srv.poll(srv.submit(c), 600_000)
    tickets = []
    sampler = ClockSampler(0)
    t0 = time.perf_counter()

    def producer():
        for t_arr, c in zip(arrivals, contracts):
            now = time.perf_counter() - t0
            if t_arr > now:
                time.sleep(t_arr - now)
            tickets.append(srv.submit(c))

    with sampler:
        th = threading.Thread(target=producer)
        th.start()
        th.join()
        for tk in tickets:
            while srv.poll(tk, 1000) is None:
                pass
    recs = [r for r in srv.records() if r["ticket"] > len(warm)]
    reserved_mib = srv.stats()["reserved_mib"]
    srv.stop()
    lat = sorted(r["latency_ms"] for r in recs)
    pct = lambda q: lat[min(len(lat) - 1, int(q * (len(lat) - 1) + 0.5))]  # noqa: E731
    span = max(r["submit_s"] + r["latency_ms"] * 1e-3 for r in recs) - min(r["submit_s"] for r in recs)
    per_wave = {r["wave"]: r["wave_ms"] for r in recs}  # one wall time per wave
    st = {"p50_ms": pct(0.5), "p99_ms": pct(0.99), "p999_ms": pct(0.999), "max_ms": lat[-1],
          "contracts_per_s": len(recs) / span, "path_steps_per_s": W.path_steps(contracts) / span,
          "batches": len(per_wave), "rejected": 0, "busy_s": sum(per_wave.values()) * 1e-3}
    offered = W.path_steps(contracts)
    # the ceiling: the batched engine pricing every request of the stream in one call
    qk.price_batch(contracts[:64], None, h)
    t_all = _timed(torch, ext, lambda: qk.price_batch(contracts, None, h), 1, flush)[0]
    rec = {"workload": f"serving_{n_requests}_requests_poisson_{rate:g}_per_s_30pct_american",
           "method": "plain_fp64_one_contract_per_launch" if plain_fp64 else "batched_fp32_engine",
           "rate_per_s": rate, "requests": n_requests, "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
           "p999_ms": st["p999_ms"], "max_ms": st["max_ms"], "contracts_per_s": st["contracts_per_s"],
           "path_steps_per_s": st["path_steps_per_s"], "offered_path_steps_per_s": offered / arrivals[-1],
           "batches": st["batches"], "rejected": st["rejected"], "busy_s": st["busy_s"],
           "lanes": lanes or 4, "wave_ms": wave_ms or 2.5, "reserved_mib": reserved_mib,
           "warmup_requests": len(warm),
           "batch_all_contracts_per_s": n_requests / (t_all * 1e-3),
           "batch_all_path_steps_per_s": offered / (t_all * 1e-3),
           "served_over_batch_all": st["contracts_per_s"] / (n_requests / (t_all * 1e-3)),
           "clocks": sampler.summary(_max_mhz())}
    if plain_sample:
        sample = contracts[:plain_sample]
        sample64 = []
        for c in sample:
            c64 = L.Contract()
            C.memmove(C.byref(c64), C.byref(c), C.sizeof(L.Contract))
            c64.precision = qk.FP64
            sample64.append(c64)
        qk.price_plain(sample64[0], None, h)
        plain_res = []

        def plain_all():
            plain_res.clear()
            for c in sample64:
                plain_res.append(qk.price_plain(c, None, h))

        t_plain = _timed(torch, ext, plain_all, 1, flush)[0]
        batch_res = qk.price_batch(sample, None, h)
        t_batch = _timed(torch, ext, lambda: qk.price_batch(sample, None, h), 1, flush)[0]
        rec.update(sample=len(sample), sample_plain_fp64_contracts_per_s=len(sample) / (t_plain * 1e-3),
                   sample_batched_contracts_per_s=len(sample) / (t_batch * 1e-3),
                   sample_mean_se_ratio_batched_over_plain=statistics.mean(
                       a["legs"][0]["std_error"] / b["legs"][0]["std_error"]
                       for a, b in zip(batch_res, plain_res) if b["legs"][0]["std_error"] > 0))
    return rec


def run_other_workload(args) -> None:
    import ctypes as C

    import torch

    import quantkos_b200 as qk
    from quantkos_b200 import _lib as L
    from quantkos_b200 import workloads as W

    torch.cuda.set_device(0)
    h = qk.Handle(0)
    ext = torch.cuda.ExternalStream(h.stream())
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    line: dict = {"metric": METRIC, "unit": METRIC, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                  "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "data": "synthetic"}
    sampler = ClockSampler(0)
    if args.workload == "plain":
        c = W.plain_heston_euler()
        for _ in range(args.warmup):
            qk.price_plain(c, None, h)
        launches = 0
        with sampler:
            ts = _timed(torch, ext, lambda: qk.price_plain(c, None, h), args.steps, flush)
        r = qk.price_plain(c, None, h)["legs"][0]
        ps = c.n_paths * c.n_steps
        line.update(value=ps / (statistics.mean(ts) * 1e-3), ms_per_step=statistics.mean(ts), dtype="f64",
                    config={"workload": "heston_euler_european_call_1048576x252_fp64_plain", "price": r["price"],
                            "std_error": r["std_error"]},
                    gpu_launches=args.steps * h.last_timing()["launches"])
    elif args.workload == "kinds":
        # every FP32 kernel kind on one large contract (16.8M x 252, one European leg, the
        # headline market; Bates jumps as in the headline) at the handle's default shape:
        # path-kernel time against each kind's SFU bound (Euler and Milstein: Box-Muller
        # lg2, sqrt, sin, cos + sqrt(v), ex2 = 6 ops per path-step; QE: 12)
        sfu_ops = h.measure_sfu()
        issue_ops = 8.0 * sfu_ops  # lane operations per second the SMs can issue (128 vs 16 per cycle)
        kinds, total = [], 0.0
        with sampler:
            for model in (qk.HESTON, qk.BATES):
                for scheme, sname in ((qk.EULER, "euler"), (qk.IMPLICIT_MILSTEIN, "milstein"), (qk.ANDERSEN_QE, "qe")):
                    n_sfu, n_issue = algorithmic_ops(sname, model == qk.BATES)
                    c = qk.make_contract(S0=100.0, v0=0.04, r=0.03, q=0.0, model=model, scheme=scheme, kappa=2.0,
                                         theta=0.04, sigma=0.3, rho=-0.7,
                                         lambda_j=0.1 if model == qk.BATES else 0.0, mu_j=-0.05, sigma_j=0.10,
                                         T=1.0, n_steps=N_STEPS, n_paths=N_PATHS, seed=42, precision=qk.FP32,
                                         payoffs=[qk.payoff(qk.EUROPEAN, qk.CALL, 100.0)])
                    prep = qk.PreparedBatch([c], None, h)
                    ms = []
                    for i in range(max(args.warmup, 3) + args.steps):
                        flush.fill_(float(i))
                        torch.cuda.synchronize()
                        prep.run()
                        prep.fetch()
                        if i >= max(args.warmup, 3):
                            ms.append(h.last_timing()["paths_ms"])
                    k_ms = statistics.mean(ms)
                    ps = N_PATHS * N_STEPS / (k_ms * 1e-3)
                    total += k_ms
                    sfu_frac = ps / (sfu_ops / n_sfu)
                    issue_frac = ps / (issue_ops / n_issue)
                    kinds.append({"model": "bates" if model == qk.BATES else "heston", "scheme": sname,
                                  "kernel_ms": k_ms, "gpath_steps_per_s": ps / 1e9, "sfu_ops_per_step": n_sfu,
                                  "issue_ops_per_step": n_issue, "frac_of_sfu_bound": sfu_frac,
                                  "frac_of_issue_bound": issue_frac, "frac": max(sfu_frac, issue_frac),
                                  "bound": "sfu" if sfu_frac >= issue_frac else "issue"})
        line.update(value=6 * N_PATHS * N_STEPS / (total * 1e-3), ms_per_step=total / 6, dtype="f32",
                    config={"workload": f"fp32_kernel_kinds_european_{N_PATHS}x{N_STEPS}", "kinds": kinds,
                            "sfu_ops_per_s": sfu_ops, "issue_lane_ops_per_s": issue_ops,
                            "algorithmic_ops": {"issue": ISSUE_OPS, "sfu": SFU_OPS}},
                    gpu_launches=None)
    elif args.workload == "published_asian":
        # the reference's one published benchmark (benchmarks/configs/
        # bench_asian_option_price_no_greeks.yaml): Heston QE, arithmetic Asian call,
        # 5,000,000 paths x 365 steps; its parameters and published price come from the
        # committed fixture of the reference's test values.  Timed like the headline:
        # resident descriptors (graph replay) and end to end from host structs, FP32.
        fx = json.loads((ROOT / "tests" / "golden" / "reference_tests.json").read_text())["asian_benchmark"]
        pp = fx["params"]
        c = qk.make_contract(S0=pp["S0"], v0=pp["v0"], r=pp["r"], q=pp["q"], scheme=qk.ANDERSEN_QE, kappa=pp["kappa"],
                             theta=pp["theta"], sigma=pp["sigma"], rho=pp["rho"], T=pp["T"], n_steps=pp["n_steps"],
                             n_paths=pp["n_paths"], seed=88471920573105, precision=qk.FP32,
                             payoffs=[qk.payoff(qk.ASIAN, qk.CALL, pp["K"])])
        tuned = [] if args.no_autotune else h.autotune([c], None, reps=1)
        prep = qk.PreparedBatch([c], None, h)
        for _ in range(max(args.warmup, 3)):
            prep.run()
            prep.fetch()
        with sampler:
            ts = _timed(torch, ext, lambda: (prep.run(), prep.fetch()), args.steps, flush)
            te = _timed(torch, ext, lambda: qk.price_batch([c], None, h), args.steps, flush)
        leg = qk.price_batch([c], None, h)[0]["legs"][0]
        ps = float(pp["n_paths"]) * pp["n_steps"]
        ms, ms_e = statistics.mean(ts), statistics.mean(te)
        line.update(value=ps / (ms * 1e-3), ms_per_step=ms, dtype="f32",
                    config={"workload": "published_asian_heston_qe_5000000x365_fp32", "price": leg["price"],
                            "std_error": leg["std_error"], "published_price": fx["price"],
                            "published_std_error": fx["std_error"],
                            "diff_in_combined_se": (leg["price"] - fx["price"]) / math.hypot(leg["std_error"],
                                                                                           fx["std_error"]),
                            "contracts_per_s": 1e3 / ms, "e2e_ms": ms_e, "e2e_path_steps_per_s": ps / (ms_e * 1e-3),
                            "autotune": _shape_summary(tuned),
                            # the reference's published timings of this run (its README), other hardware
                            "published_reference": {"path_steps_per_s": 1.870e10, "seconds": 0.0976,
                                                    "build": "CUDA FP32 fast-math",
                                                    "hardware": "RTX 3060 Laptop GPU (sm_86)"}},
                    gpu_launches=None)
    elif args.workload == "lsm":
        pk_file = ROOT / "MEASURED_PEAKS.json"
        measured = json.loads(pk_file.read_text()).get("hbm_gbs") if pk_file.exists() else None
        hbm_peak = (measured, "measured copy bandwidth (MEASURED_PEAKS.json)") if measured else \
            (6650.0, "fallback 6.65 TB/s (no measured peak file)")
        c32 = W.american_lsm(precision=qk.FP32)
        c64 = W.american_lsm(precision=qk.FP64)
        for _ in range(args.warmup):
            qk.price_batch([c32], None, h)
        with sampler:
            ts = _timed(torch, ext, lambda: qk.price_batch([c32], None, h), args.steps, flush)
        t = h.last_timing()
        r32 = qk.price_batch([c32], None, h)[0]["legs"][0]
        qk.price_plain(c64, None, h)
        t64 = _timed(torch, ext, lambda: qk.price_plain(c64, None, h), 1, flush)[0]
        r64 = qk.price_plain(c64, None, h)["legs"][0]
        ps = c32.n_paths * c32.n_steps
        # backward sweep: algorithmic 16 B per path per date (S, v slab read + cash flow read/write, FP32)
        sweep_bytes = 16.0 * c32.n_paths * 50
        ms = statistics.mean(ts)
        line.update(value=ps / (ms * 1e-3), ms_per_step=ms, dtype="f32",
                    config={"workload": "american_put_lsm_heston_qe_4194304x250_50dates_polysv", "price": r32["price"],
                            "std_error": r32["std_error"], "price_fp64": r64["price"], "std_error_fp64": r64["std_error"],
                            "fp64_plain_ms": t64, "speedup_vs_fp64_plain": t64 / ms},
                    roofline={"bound": "hbm", "achieved": sweep_bytes / (t["reduce_ms"] * 1e-3) / 1e9,
                              "peak": hbm_peak[0], "peak_source": hbm_peak[1],
                              "unit": "GB/s", "kernel": "LSM backward sweep (all dates)",
                              "sweep_ms": t["reduce_ms"], "forward_ms": t["device_ms"] - t["reduce_ms"]},
                    gpu_launches=args.steps * t["launches"])
        line["roofline"]["frac"] = line["roofline"]["achieved"] / line["roofline"]["peak"]
        # the forward kernel (Heston QE paths, FP32, writing the 50 exercise-date slabs):
        # SFU-bound like the path kernels, 12 SFU operations per path-step
        sfu_ops = h.measure_sfu()
        fwd_ms = line["roofline"]["forward_ms"]
        line["forward"] = {"kernel": "slab_paths_two_kernel<float, Heston, QE>", "ms": fwd_ms,
                           "path_steps_per_s": ps / (fwd_ms * 1e-3), "bound": "sfu",
                           "frac_of_sfu_bound": ps / (fwd_ms * 1e-3) / (sfu_ops / SFU_PER_STEP),
                           "slab_bytes_written": 8.0 * c32.n_paths * 50,
                           "slab_write_gbs": 8.0 * c32.n_paths * 50 / (fwd_ms * 1e-3) / 1e9}
    elif args.workload == "attribution":
        # Where the 4096-contract mix loses against its kinds' standalone rates: the mix
        # timed whole; each kernel kind's share of the mix (its contracts, all Greeks)
        # timed alone; and each kind's standalone rate on one 16.8M x 252 European
        # contract.  whole vs sum of shares = what running the kinds in one call costs
        # or saves; shares vs standalone rates = small contracts, legs and tails.
        g = W.batch_greeks()
        full = W.mixed_batch()
        tuned = [] if args.no_autotune else h.autotune(full[:256], g, reps=1)
        qk.price_batch(full[:64], g, h)
        with sampler:
            t_whole = _timed(torch, ext, lambda: qk.price_batch(full, g, h), 1, flush)[0]
            tw = h.last_timing()
            shares = []
            for model in (qk.HESTON, qk.BATES):
                for scheme, sname in ((qk.EULER, "euler"), (qk.IMPLICIT_MILSTEIN, "milstein"), (qk.ANDERSEN_QE, "qe")):
                    sub = [c for c in full if c.model == model and c.scheme == scheme]
                    t_sub = _timed(torch, ext, lambda: qk.price_batch(sub, g, h), 1, flush)[0]
                    big = qk.make_contract(S0=100.0, v0=0.04, r=0.03, model=model, scheme=scheme, kappa=2.0,
                                           theta=0.04, sigma=0.3, rho=-0.7,
                                           lambda_j=0.1 if model == qk.BATES else 0.0, mu_j=-0.05, sigma_j=0.10,
                                           T=1.0, n_steps=N_STEPS, n_paths=N_PATHS, seed=42, precision=qk.FP32,
                                           payoffs=[qk.payoff(qk.EUROPEAN, qk.CALL, 100.0)])
                    qk.price_batch([big], None, h)
                    t_big = _timed(torch, ext, lambda: qk.price_batch([big], None, h), 1, flush)[0]
                    ps_sub = W.path_steps(sub, g)
                    rate_big = N_PATHS * N_STEPS / (t_big * 1e-3)
                    shares.append({"model": "bates" if model == qk.BATES else "heston", "scheme": sname,
                                   "contracts": len(sub), "path_steps": ps_sub, "ms": t_sub,
                                   "path_steps_per_s": ps_sub / (t_sub * 1e-3),
                                   "standalone_path_steps_per_s": rate_big,
                                   "share_over_standalone": ps_sub / (t_sub * 1e-3) / rate_big,
                                   "ideal_ms": ps_sub / rate_big * 1e3})
        ps = W.path_steps(full, g)
        sum_ms = sum(s["ms"] for s in shares)
        ideal_ms = sum(s["ideal_ms"] for s in shares)
        line.update(metric="path-steps/s", value=ps / (t_whole * 1e-3), ms_per_step=t_whole, dtype="f32",
                    config={"workload": "mixed_4096_contracts_all_greeks_seed123_attribution", "whole_ms": t_whole,
                            "whole_paths_ms": tw["paths_ms"], "whole_merge_ms": tw["reduce_ms"],
                            "sum_of_kind_shares_ms": sum_ms, "ideal_at_standalone_rates_ms": ideal_ms,
                            "whole_over_ideal": t_whole / ideal_ms, "kinds": shares,
                            "autotune": _shape_summary(tuned)},
                    gpu_launches=tw["launches"])
    elif args.workload == "batch":
        rec = measure_batch_mix(qk, W, h, torch, ext, flush, subset=args.subset, autotune=not args.no_autotune)
        ms = rec["batched_ms"]
        line.update(metric="contracts/s", unit="contracts/s", value=rec["contracts_per_s"], ms_per_step=ms,
                    dtype="f32", config=rec, gpu_launches=rec["gpu_launches"])
        sampler = None
    else:  # serve
        _, contracts = W.serving_stream(256)
        tuned = [] if args.no_autotune else h.autotune(contracts[:256], None, reps=1)
        rec = measure_serving(qk, W, h, torch, ext, flush, rate=args.rate, n_requests=args.requests,
                              plain_sample=args.subset, lanes=args.lanes, wave_ms=args.wave_ms,
                              plain_fp64=args.serve_plain)
        rec["autotune"] = _shape_summary(tuned)
        line.update(metric="contracts/s", unit="contracts/s", value=rec["contracts_per_s"], dtype="f32",
                    ms_per_step=None, config=rec, gpu_launches=None)
        sampler = None
    pk = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    line["clocks"] = sampler.summary(pk.get("sm_max_mhz", 1965.0)) if sampler else line["config"].pop("clocks")
    print(json.dumps(line), flush=True)
    h.close()


def main() -> None:
    args = parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
        return
    if args.workload != "bates5":
        run_other_workload(args)
        return

    import torch
    import torch.distributed as dist

    import quantkos_b200 as qk

    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local_rank))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    h = qk.Handle(local_rank)
    ext = torch.cuda.ExternalStream(h.stream())
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    contract = workload_contract(qk, rank, n_paths=args.paths)
    path_steps = float(args.paths) * N_STEPS

    # ---- launch shape: the engine's autotuner on the workload itself (untimed)
    tuned = None
    if args.shape:
        tpw, tail, lanes = (int(x) for x in args.shape.split(","))
        h.tune_set(contract.precision, contract.model, contract.scheme, tpw, bool(tail), lanes)
        tuned = {"tiles_per_warp": tpw, "guided_tail": tail, "paths_per_lane": lanes, "set_by": "--shape"}
    elif not args.no_autotune:
        rep = h.autotune([contract], None, reps=1)[0]
        tuned = {"tiles_per_warp": rep["tiles_per_warp"], "guided_tail": rep["guided_tail"],
                 "paths_per_lane": rep["paths_per_lane"], "block_size": rep["block_size"],
                 "best_ms": rep["best_ms"], "default_ms": rep["default_ms"]}

    # ---- value: descriptors resident in HBM, K device-timed pricings
    prep = qk.PreparedBatch([contract], None, h)
    for _ in range(max(args.warmup, 3)):
        prep.run()
        prep.fetch()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    kernel_ms, launches = [], 0
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local_rank)
    with sampler:
        for i in range(args.steps):
            flush.fill_(float(i))  # L2 flush (256 MiB > 126 MB L2) outside the timed events
            torch.cuda.synchronize()
            starts[i].record(ext)
            prep.run()
            ends[i].record(ext)
            res = prep.fetch()
            t = h.last_timing()
            kernel_ms.append(t["paths_ms"])
            launches += t["launches"]
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = max_over_ranks(sum(step_ms))
    ms_per_step = total_ms / args.steps
    value = world * path_steps / (ms_per_step * 1e-3)

    # ---- e2e: the public call with host buffers (plan + H2D descriptors + kernels + D2H results)
    for _ in range(2):
        qk.price_batch([contract], None, h)
    e_s = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e_e = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    h2d = d2h = 0
    torch.cuda.synchronize()
    barrier()
    for i in range(args.steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        e_s[i].record(ext)
        qk.price_batch([contract], None, h)
        e_e[i].record(ext)
        t = h.last_timing()
        h2d, d2h = t["h2d_bytes"], t["d2h_bytes"]
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(sum(s.elapsed_time(e) for s, e in zip(e_s, e_e))) / args.steps
    e2e_value = world * path_steps / (e2e_ms * 1e-3)

    # ---- roofline of the dominant kernel (the fused path kernel)
    sfu_ops = h.measure_sfu()
    peak_ps = sfu_ops / SFU_PER_STEP
    kern_ms = statistics.mean(kernel_ms)
    achieved_ps = path_steps / (kern_ms * 1e-3)
    # DRAM bytes of one path-kernel launch: ncu (dram__bytes_read.sum + dram__bytes_write.sum)
    # on the 1,048,576-path case at the autotuned shape measured 2.09 MB, i.e. 0.0079 B per
    # path-step (tile records plus write-back of the L2-flush buffer), scaled here to the
    # launch's path-steps.  Algorithmic DRAM bytes of the kernel: 0.
    traffic = DRAM_BYTES_PER_PATH_STEP * path_steps

    # ---- the fused Heston-QE European kernel alone (same market, no jumps, one leg)
    hqe = None
    if not args.no_plain:
        hc = qk.make_contract(S0=100.0, v0=0.04, r=0.03, q=0.0, model=qk.HESTON, scheme=qk.ANDERSEN_QE, kappa=2.0,
                              theta=0.04, sigma=0.3, rho=-0.7, psi_c=1.5, T=1.0, n_steps=N_STEPS,
                              n_paths=args.paths, seed=42, stream=rank, precision=qk.FP32,
                              payoffs=[qk.payoff(qk.EUROPEAN, qk.CALL, 100.0)])
        hp = qk.PreparedBatch([hc], None, h)
        hms = []
        for i in range(3 + 5):
            flush.fill_(float(i))
            torch.cuda.synchronize()
            hp.run()
            hp.fetch()
            if i >= 3:
                hms.append(h.last_timing()["paths_ms"])
        h_ps = path_steps / (statistics.mean(hms) * 1e-3)
        hqe = {"workload": f"heston_qe_european_call_{args.paths}x{N_STEPS}_fp32", "kernel_ms": statistics.mean(hms),
               "achieved": h_ps / 1e9, "peak": sfu_ops / SFU_PER_STEP / 1e9, "unit": "Gpath-steps/s",
               "frac": h_ps / (sfu_ops / SFU_PER_STEP)}

    # ---- the same workload with antithetic pairs: throughput and standard error per leg
    anti = None
    if not args.no_plain:
        ac = workload_contract(qk, rank, n_paths=args.paths)
        ac.antithetic = 1
        ap = qk.PreparedBatch([ac], None, h)
        ams, r_anti = [], None
        for i in range(3 + 5):
            flush.fill_(float(i))
            torch.cuda.synchronize()
            ap.run()
            r_anti = ap.fetch()
            if i >= 3:
                ams.append(h.last_timing()["device_ms"])
        a_ms = statistics.mean(ams)
        ratio = [ra["std_error"] / rp["std_error"] for ra, rp in zip(r_anti[0]["legs"], res[0]["legs"])]
        anti = {"ms": a_ms, "value": path_steps / (a_ms * 1e-3), "unit": METRIC,
                "se_ratio_vs_independent": ratio,
                "equal_se_speedup": [ms_per_step / (a_ms * q * q) for q in ratio],
                "price": [leg["price"] for leg in r_anti[0]["legs"]]}

    # ---- plain FP64 drop-in on the same workload (equal paths => equal standard error)
    plain = None
    if not args.no_plain:
        c64 = workload_contract(qk, rank, qk.FP64, args.paths)
        qk.price_plain(c64, None, h)
        r64 = qk.price_plain(c64, None, h)
        t64 = h.last_timing()
        plain = {"ms": t64["device_ms"], "value": path_steps / (t64["device_ms"] * 1e-3),
                 "speedup_of_value": value / world / (path_steps / (t64["device_ms"] * 1e-3)),
                 "std_error_fp64": [leg["std_error"] for leg in r64["legs"]],
                 "std_error_fp32": [leg["std_error"] for leg in res[0]["legs"]],
                 "price_fp64": [leg["price"] for leg in r64["legs"]],
                 "price_fp32": [leg["price"] for leg in res[0]["legs"]],
                 # the FP32 batched price minus the FP64 drop-in price, in units of the FP64 standard error
                 "fp32_minus_fp64_in_se": [(a["price"] - b["price"]) / b["std_error"] if b["std_error"] > 0 else 0.0
                                           for a, b in zip(res[0]["legs"], r64["legs"])]}

    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    clocks = sampler.summary(peaks.get("sm_max_mhz", 1965.0))

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        try:
            cpu = {k: v for k, v in cpu_reference_rate(args.cpu_baseline_paths).items() if k != "seconds"}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": METRIC, "cores": os.cpu_count(), "kind": "unavailable", "sample": str(e)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD if args.paths == N_PATHS else f"{WORKLOAD} (reduced to {args.paths} paths)",
                       "n_paths": args.paths, "n_steps": N_STEPS, "payoff_legs": 5,
                       "parallelism": f"contract-per-gpu x{world}", "l2": "flushed between timed steps (256 MiB write)",
                       "contracts_per_s": world / (ms_per_step * 1e-3)},
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_ms},
            "roofline": {"bound": "sfu", "achieved": achieved_ps / 1e9, "peak": peak_ps / 1e9,
                         "unit": "Gpath-steps/s", "frac": achieved_ps / peak_ps, "traffic": traffic,
                         "kernel": "price_tiles_kernel<float>", "kernel_ms": kern_ms,
                         "peak_source": f"measured SFU rate {sfu_ops / 1e12:.3f} Tops/s (qk_measure_sfu); "
                                        f"{SFU_PER_STEP:.0f} SFU ops per path-step (algorithmic)"},
            "cpu_baseline": cpu,
            "heston_qe_european": hqe,
            "antithetic": anti,
            "autotune": tuned,
            "plain_fp64": plain,
            "clocks": clocks,
            "gpu_launches": launches,
        }
        if world == 1 and not args.no_extra:
            # the other north-star workloads, each with its own clock record: the 4096-contract
            # mix with all Greeks against the plain FP64 drop-in, and the serving stream at
            # 2,000 requests/s (over capacity) and at 1,000 requests/s (under it)
            from quantkos_b200 import workloads as W
            line["batch_4096"] = measure_batch_mix(qk, W, h, torch, ext, flush,
                                                   subset=args.batch_compare, autotune=not args.no_autotune)
            line["serve"] = measure_serving(qk, W, h, torch, ext, flush, rate=2000.0, n_requests=20_000)
            line["serve_sub_capacity"] = measure_serving(qk, W, h, torch, ext, flush, rate=1000.0,
                                                         n_requests=10_000)
            # both methods behind the same server on one stream, at a rate the plain FP64
            # method sustains: latency at equal load
            keys = ("p50_ms", "p99_ms", "p999_ms", "max_ms", "contracts_per_s", "clocks")
            vs = {}
            for name, plain in (("batched", False), ("plain_fp64", True)):
                r = measure_serving(qk, W, h, torch, ext, flush, rate=200.0, n_requests=3_000, plain_fp64=plain)
                vs[name] = {k: r[k] for k in keys}
            line["serve_vs_plain"] = {"workload": "serving_3000_requests_poisson_200_per_s_30pct_american", **vs}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    h.close()


if __name__ == "__main__":
    main()
