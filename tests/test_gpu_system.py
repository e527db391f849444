"""GPU: the system around the kernels — config-driven runs (MCDispatcher, .paths
files, payoff percentiles, the CLI), the continuous-batching server, and the
mixed batched workload against closed forms."""
import math
import os
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tests.helpers import load

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent

YAML = """
Market:
  Price: 100.0
  Variance: 0.04
  r: 0.05
  q: 0.02
Options:
  OptionType: {otype}
  OptionRight: {right}
  StrikePrice: 100.
  BarrierPrice: 120.
Model:
  Heston:
    k: 2.0
    theta: 0.04
    sigma: 0.3
    rho: -0.7
Numerics:
  Scheme: AndersonQE
Time:
  T_End: 1.0
  Inp_DT: 0.0078125
MC:
  Normalize_prices: true
  N_Paths: 20000
  RNG_Seed: 12345
  analyze_risk_neutral_payoff_distribution: {dist}
  compute_delta_et_gamma: {greeks}
  Precision: {prec}
  Engine: {engine}
Output:
  out_dir: "{out_dir}"
  Name_Paths_Out_File: "{paths}"
  Format: BIN
"""


def _cfg(qk, tmp_path, otype="European", right="Call", dist="false", greeks="false", prec="FP64", engine="plain",
         paths=""):
    return qk.Parser.parse_string(YAML.format(otype=otype, right=right, dist=dist, greeks=greeks, prec=prec,
                                              engine=engine, out_dir=str(tmp_path), paths=paths))


def test_dispatcher_matches_contract_path(qk, handle, oracle, tmp_path):
    cfg = _cfg(qk, tmp_path, greeks="true")
    res = qk.MCDispatcher(cfg, handle).launch_montecarlo()
    k, g = cfg.to_contract()
    o = oracle.price(k, g)["legs"][0]
    assert res.OptionPrice.option_price == pytest.approx(o["price"], rel=1e-9)
    assert res.Greeks.delta == pytest.approx(o["delta"], rel=1e-6)
    assert res.Greeks.gamma == pytest.approx(o["gamma"], rel=1e-5, abs=1e-9)


def test_paths_file_roundtrip(qk, handle, oracle, tmp_path):
    """BinWriter / BinReader (include/IO/IOBinary.hpp:72-378): 40-byte header, row-major payload of
    normalised prices; reading column j at t = (j+1) dt returns scaled prices (BinaryFormatTest)."""
    cfg = _cfg(qk, tmp_path, paths="run.paths")
    cfg.n_paths = 300
    qk.MCDispatcher(cfg, handle).launch_montecarlo()
    f = tmp_path / "run.paths"
    data = f.read_bytes()
    key, version, prec, n, steps = struct.unpack_from("<8siiii", data, 0)
    dt, scale = struct.unpack_from("<dd", data, 24)
    assert key == b"QUANTKOS" and version == 1 and prec == 8 and n == 300 and steps == 128
    assert dt == pytest.approx(1.0 / 128) and scale == 100.0
    payload = np.frombuffer(data, dtype=np.float64, offset=40).reshape(n, steps)
    k, _ = cfg.to_contract()
    S, _ = oracle.paths(k, 0, 300)
    np.testing.assert_allclose(payload * scale, S, rtol=1e-12)
    # strided column read at t = 0.7 (BinReader::read_prices_at_target_time)
    j = int(round(0.7 / dt)) - 1
    np.testing.assert_allclose(payload[:, j] * scale, S[:, j], rtol=1e-12)


def test_paths_file_fp32_no_noise(qk, handle, tmp_path):
    """NoNoiseTest through the .paths writer: every path at T equals S0 e^{(r-q)T} (FP32: 5e-3)."""
    y = YAML.format(otype="European", right="Call", dist="false", greeks="false", prec="FP32", engine="batch",
                    out_dir=str(tmp_path), paths="nn.paths")
    y = y.replace("Variance: 0.04", "Variance: 0.0").replace("k: 2.0", "k: 0.0").replace("theta: 0.04", "theta: 0.0")
    y = y.replace("sigma: 0.3", "sigma: 0.0").replace("rho: -0.7", "rho: 0.0")
    cfg = qk.Parser.parse_string(y)
    cfg.n_paths = 100
    qk.MCDispatcher(cfg, handle).launch_montecarlo()
    data = (tmp_path / "nn.paths").read_bytes()
    assert struct.unpack_from("<i", data, 12)[0] == 4
    payload = np.frombuffer(data, dtype=np.float32, offset=40).reshape(100, 128)
    assert np.all(np.abs(payload[:, -1] * 100.0 - 100.0 * math.exp(0.03)) < 5e-3)


def test_payoff_percentiles(qk, handle, oracle, tmp_path):
    """OptionPricer::analyze_risk_neutral_discounted_payoff_distribution (OptionPricer.hpp:340-360)."""
    cfg = _cfg(qk, tmp_path, otype="Asian", dist="true")
    res = qk.MCDispatcher(cfg, handle).launch_montecarlo()
    k, _ = cfg.to_contract()
    pay = np.sort(oracle.payoffs(k))
    eff = math.exp(-0.05 * 1.0) * 100.0
    N = len(pay)
    fr = [0.01, 0.05, 0.10, 0.20, 0.30, 0.40, 0.50, 0.60, 0.70, 0.80, 0.90, 0.95, 0.99]
    want = [pay[0] * eff] + [pay[int(N * f)] * eff for f in fr] + [pay[-1] * eff]
    got = list(res.OptionPrice.percentiles.values())
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12)


def test_cli_runs_a_config(qk, handle, tmp_path):
    y = YAML.format(otype="BarrierUpAndOut", right="Call", dist="false", greeks="true", prec="FP32", engine="batch",
                    out_dir=str(tmp_path), paths="")
    p = tmp_path / "cfg.yaml"
    p.write_text(y)
    exe = ROOT / "quantkos_b200" / "quantkos"
    out = subprocess.run([str(exe), str(p)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert "Estimated Option Price" in out.stdout and "Delta" in out.stdout
    bad = subprocess.run([str(exe), str(tmp_path / "missing.yaml")], capture_output=True, text=True, timeout=60)
    assert bad.returncode == 1 and "File not found" in bad.stderr


def test_server_result_alone_equals_in_the_mix(qk, handle):
    """Continuous batching: a request priced alone and the same request admitted together with
    others (arriving while work is on the GPU) give identical results."""
    from quantkos_b200 import workloads as W
    _, contracts = W.serving_stream(96, seed=11)
    contracts = [c for c in contracts]
    for c in contracts:  # keep the test short
        c.n_paths = min(c.n_paths, 200_000)
    probe = contracts[17]
    alone = qk.price_batch([probe], None, handle)[0]["legs"][0]
    with qk.Server(handle, 0, 16) as srv:
        tickets = [srv.submit(c) for c in contracts[:40]]
        t_probe = srv.submit(probe)
        tickets += [srv.submit(c) for c in contracts[40:]]
        got = None
        while got is None:
            got = srv.poll(t_probe, 1000)
        for t in tickets:
            while srv.poll(t, 1000) is None:
                pass
        st = srv.stats()
    leg = got["legs"][0]
    assert leg["price"] == pytest.approx(alone["price"], rel=1e-12)
    assert leg["std_error"] == pytest.approx(alone["std_error"], rel=1e-9)
    assert st["completed"] == 97 and st["rejected"] == 0 and st["batches"] >= 2
    assert st["p50_ms"] > 0 and st["p99_ms"] >= st["p50_ms"]


def test_server_lanes_take_the_handles_launch_shapes(qk, handle):
    """qk_serve_start gives its lanes the launch shapes of the handle it starts from: a request
    served alone equals, bit for bit, qk_price_batch on that handle with the same shapes, while
    the default shapes merge the moments in other groupings (last-bit differences)."""
    legs = [qk.payoff(qk.EUROPEAN, qk.CALL, 100.0), qk.payoff(qk.ASIAN, qk.CALL, 100.0),
            qk.payoff(qk.BARRIER_UP_OUT, qk.CALL, 100.0, 130.0), qk.payoff(qk.LOOKBACK_FLOATING, qk.PUT, 100.0),
            qk.payoff(qk.BINARY_CASH, qk.CALL, 105.0)]
    key = lambda r: [(g["price"], g["std_error"]) for g in r["legs"]]
    # one path per lane (the default is two): tiles then group the paths differently; the
    # compensated merge often gives the same bits anyway, so take a contract (seed) whose
    # merged moments do differ in the last bits, or the check below could not tell
    for seed in range(5, 25):
        c = qk.make_contract(model=qk.BATES, scheme=qk.ANDERSEN_QE, lambda_j=0.1, mu_j=-0.05, sigma_j=0.1,
                             n_steps=64, n_paths=300_000, seed=seed, precision=qk.FP32, payoffs=legs)
        default = key(qk.price_batch([c], None, handle)[0])
        handle.tune_set(qk.FP32, qk.BATES, qk.ANDERSEN_QE, 4, False, 1)
        tuned = key(qk.price_batch([c], None, handle)[0])
        handle.tune_reset()
        if tuned != default:
            break
    handle.tune_set(qk.FP32, qk.BATES, qk.ANDERSEN_QE, 4, False, 1)
    try:
        assert key(qk.price_batch([c], None, handle)[0]) == tuned
        with qk.Server(handle, 0, 4) as srv:
            t = srv.submit(c)
            got = None
            while got is None:
                got = srv.poll(t, 1000)
    finally:
        handle.tune_reset()
    assert key(got) == tuned
    assert tuned != default
    for (p1, s1), (p0, s0) in zip(tuned, default):
        assert p1 == pytest.approx(p0, rel=1e-12, abs=1e-15) and s1 == pytest.approx(s0, rel=1e-9)


def test_server_admission_rejects_oversized(qk, handle):
    from quantkos_b200 import workloads as W
    big = W.american_lsm(n_paths=4_000_000)
    with qk.Server(handle, 64, 8) as srv:  # 64 MiB budget: the LSM slabs do not fit
        with pytest.raises(RuntimeError, match="admission budget"):
            srv.submit(big)
        small = qk.make_contract(n_paths=10_000, n_steps=10)
        t = srv.submit(small)
        while srv.poll(t, 1000) is None:
            pass
        assert srv.stats()["rejected"] == 1


def test_server_records_account_for_every_request(qk, handle):
    """qk_serve_records: one record per completed request, each ticket once; a wave's records
    agree on its lane, size and wall time and their number is the wave's size; admission wait
    plus the wave's wall time make up the latency; the percentiles of qk_serve_stats_get are
    those of the records' latencies."""
    from quantkos_b200 import workloads as W
    _, contracts = W.serving_stream(120, seed=5)
    for c in contracts:
        c.n_paths = min(c.n_paths, 100_000)
    with qk.Server(handle, 4096, 16, lanes=2, wave_ms=2.0, reserve_mib=-1) as srv:
        tickets = [srv.submit(c) for c in contracts]
        for tk in tickets:
            while srv.poll(tk, 1000) is None:
                pass
        recs = srv.records()
        st = srv.stats()
    assert sorted(r["ticket"] for r in recs) == sorted(tickets)
    waves = {}
    for r in recs:
        waves.setdefault(r["wave"], []).append(r)
        assert 0 <= r["lane"] < 2 and r["wave_requests"] >= 1
        assert r["admit_ms"] >= 0.0 and r["wave_ms"] > 0.0 and r["est_ms"] > 0.0
        assert r["latency_ms"] == pytest.approx(r["admit_ms"] + r["wave_ms"], rel=1e-6, abs=1e-3)
    for w, rs in waves.items():
        assert len(rs) == rs[0]["wave_requests"]
        assert len({(r["lane"], r["wave_ms"], r["wave_est_ms"]) for r in rs}) == 1
        assert rs[0]["wave_est_ms"] == pytest.approx(sum(r["est_ms"] for r in rs), rel=1e-9)
    assert st["completed"] == len(tickets) and st["batches"] == len(waves)
    lat = sorted(r["latency_ms"] for r in recs)
    assert st["max_ms"] == lat[-1]
    assert st["p50_ms"] == lat[int(0.5 * (len(lat) - 1) + 0.5)]


def test_server_plain_fp64_mode_equals_price_plain(qk, handle):
    """plain_fp64 = 1: every request is priced alone by the plain FP64 method behind the same
    lanes; each result equals qk_price_plain on that contract bit for bit, one wave per request."""
    from quantkos_b200 import workloads as W
    _, contracts = W.serving_stream(24, seed=17)
    for c in contracts:
        c.n_paths = min(c.n_paths, 40_000)
    with qk.Server(handle, 4096, 16, lanes=2, reserve_mib=-1, plain_fp64=True) as srv:
        tickets = [srv.submit(c) for c in contracts]
        got = []
        for tk in tickets:
            r = None
            while r is None:
                r = srv.poll(tk, 1000)
            got.append(r)
        recs = srv.records()
    assert all(r["wave_requests"] == 1 for r in recs) and len(recs) == len(contracts)
    for c, g in zip(contracts, got):
        want = qk.price_plain(c, None, handle)
        for a, b in zip(g["legs"], want["legs"]):
            assert a["price"] == b["price"] and a["std_error"] == b["std_error"]


def test_server_reserves_pool_memory(qk, handle):
    """The server maps its reservation into the device pool at the start (0 = the budget, -1 =
    none, else the MiB given), holds it while it runs and gives it back at the stop; an
    explicit reservation that cannot fit fails with QK_ERR_CAPACITY and leaves nothing held.
    Read from the pool's own counters (memory it has mapped), since a reservation may reuse
    blocks the pool already held."""
    from cuda.bindings import runtime as rt
    from quantkos_b200 import _lib as L

    def pool_reserved() -> int:
        err, pool = rt.cudaDeviceGetDefaultMemPool(0)
        assert err == rt.cudaError_t.cudaSuccess
        err, v = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent)
        assert err == rt.cudaError_t.cudaSuccess
        return int(v)

    small = qk.make_contract(n_paths=10_000, n_steps=10)
    for reserve, want in ((0, 2048), (-1, 0), (512, 512)):
        r0 = pool_reserved()
        with qk.Server(handle, 2048, 8, reserve_mib=reserve) as srv:
            assert srv.stats()["reserved_mib"] == want
            assert pool_reserved() >= want << 20
            t = srv.submit(small)
            while srv.poll(t, 1000) is None:
                pass
        assert pool_reserved() <= r0 + (256 << 20)  # the reservation went back to the device
    r0 = pool_reserved()
    with pytest.raises(RuntimeError) as err:
        qk.Server(handle, 2048, 8, reserve_mib=1 << 30)  # 1 PiB
    assert err.value.status == L.QK_ERR_CAPACITY
    assert pool_reserved() <= r0 + (256 << 20)
    with pytest.raises(ValueError):
        qk.Server(handle, 2048, 8, reserve_mib=-2)


def test_mixed_batch_sample_vs_closed_forms(qk, handle, oracle):
    """European legs of the seeded mixed batch within 3 SE (+ discretisation allowance for Euler)
    of the Gil-Pelaez price, priced together in one batch with all Greeks."""
    from quantkos_b200 import workloads as W
    batch = W.mixed_batch(256)
    res = qk.price_batch(batch, W.batch_greeks(), handle)
    checked = fails = 0
    for c, r in zip(batch, res):
        leg = r["legs"][0]
        if c.payoffs[0].type != qk.EUROPEAN or c.scheme == qk.EULER:
            continue
        exact = oracle.exact_call(2 if c.model == qk.BATES else 1, c, 200.0 if c.model == qk.HESTON else 0.0)
        if c.payoffs[0].right == qk.PUT:  # put-call parity
            exact += c.payoffs[0].strike * math.exp(-c.r * c.T) - c.S0 * math.exp(-c.q * c.T)
        checked += 1
        if abs(leg["price"] - exact) > 3.0 * leg["std_error"] + 2e-3 * exact:
            fails += 1
    assert checked >= 20
    assert fails <= max(1, checked // 50), (fails, checked)


def test_config0_plain_fp64_vs_closed_form(qk, handle, oracle):
    """Plain method on the plain-method case (Heston Euler, 1,048,576 x 252, FP64) within 3 SE of
    the Gil-Pelaez price (the allowance covers the Euler bias at dt = 1/252, measured here against a
    1008-step run)."""
    from quantkos_b200 import workloads as W
    c = W.plain_heston_euler()
    r = qk.price_plain(c, None, handle)["legs"][0]
    exact = oracle.exact_call(1, c, 200.0)
    fine = qk.make_contract(**{f: getattr(c, f) for f in ("S0", "v0", "r", "q", "kappa", "theta", "sigma", "rho")},
                            scheme=qk.EULER, T=1.0, n_steps=1008, n_paths=1_048_576, seed=42, precision=qk.FP64,
                            payoffs=[qk.payoff(0, 0, 100.0)])
    rf = qk.price_plain(fine, None, handle)["legs"][0]
    bias = abs(r["price"] - rf["price"])
    assert abs(r["price"] - exact) <= 3.0 * r["std_error"] + 2.0 * bias + 1e-3, (r, exact, rf)
    assert abs(rf["price"] - exact) <= 3.0 * rf["std_error"] + 1e-3


def test_prepared_batch_graph_replay(qk, handle):
    """The prepared set replays its captured launch sequence: every replay equals the one-shot
    batched call bit for bit, uploads nothing, and another pricing call drops the prepared set."""
    from quantkos_b200 import workloads as W
    batch = W.mixed_batch(24, seed=5)
    for c in batch:
        c.n_paths = min(c.n_paths, 100_000)
    g = W.batch_greeks()
    want = qk.price_batch(batch, g, handle)
    prep = qk.PreparedBatch(batch, g, handle)
    for _ in range(2):
        prep.run()
        got = prep.fetch()
        for a, b in zip(got, want):
            assert a["legs"] == b["legs"]
        t = handle.last_timing()
        assert t["h2d_bytes"] == 0 and t["launches"] >= 2 and t["paths_ms"] > 0.0
        assert t["device_ms"] >= t["paths_ms"]
    qk.price_batch(batch[:1], None, handle)
    with pytest.raises(RuntimeError, match="qk_batch_prepare"):
        prep.run()


def test_autotuner_keeps_prices_and_reports_every_kind(qk, handle):
    """The autotuner times every candidate shape per kernel kind and keeps the fastest; a shape
    changes which paths share a tile record, never which paths are simulated, so prices agree to
    the rounding of the moment merge."""
    from quantkos_b200 import workloads as W
    batch = [c for c in W.mixed_batch(48, seed=9)]
    for c in batch:
        c.n_paths = min(c.n_paths, 200_000)
    before = qk.price_batch(batch, None, handle)
    report = handle.autotune(batch, None, reps=1)
    kinds = {(c.precision, c.model, c.scheme) for c in batch}
    assert {(r["precision"], r["model"], r["scheme"]) for r in report} == kinds
    for r in report:
        assert r["tiles_per_warp"] in (4, 8, 12, 24, 48) and r["guided_tail"] in (0, 1)
        assert r["paths_per_lane"] in (1, 2)
        assert 0.0 < r["best_ms"] <= r["default_ms"]
    after = qk.price_batch(batch, None, handle)
    for a, b in zip(before, after):
        assert a["legs"][0]["price"] == pytest.approx(b["legs"][0]["price"], rel=1e-12, abs=1e-15)
        assert a["legs"][0]["std_error"] == pytest.approx(b["legs"][0]["std_error"], rel=1e-9)
    with pytest.raises(ValueError):
        handle.tune_set(1, 0, 3, 12, True)
    handle.tune_reset()  # back to the defaults for the tests that follow


def test_paths_file_batching_keeps_the_file(qk, handle, tmp_path):
    """MC.Batch_Size / MC.Max_VRAM_MB size the stored path batches of the .paths output with the
    reference's rule (fixed, all, or from the device budget); the file is the same whatever the
    batching, since every path's draws depend only on its index."""
    blobs = []
    for bs, vram in ((-1, 256), (64, 256), (0, 1)):
        name = f"b{bs + 1}_{vram}.paths"
        cfg = _cfg(qk, tmp_path, paths=name)
        cfg.n_paths = 300
        cfg.batch_size = bs
        cfg.max_vram_mb = vram
        qk.MCDispatcher(cfg, handle).launch_montecarlo()
        blobs.append((tmp_path / name).read_bytes())
    assert blobs[0] == blobs[1] == blobs[2]


def test_server_cancels_waiting_requests(qk, handle):
    """A request still waiting for admission can be withdrawn: its poll reports the cancellation,
    the requests around it complete, an admitted or finished request is not cancelled, and an
    unknown ticket is an error."""
    from quantkos_b200 import _lib as L
    from quantkos_b200 import workloads as W
    long_job = W.bates_qe_five_payoffs(n_paths=16_777_216)  # keeps both lanes busy for tens of ms
    small = qk.make_contract(n_paths=10_000, n_steps=10)
    with qk.Server(handle, 0, 1, lanes=2) as srv:  # one request per wave, two lanes
        t_busy = [srv.submit(long_job) for _ in range(2)]
        t_keep = srv.submit(small)
        t_drop = srv.submit(small)
        assert srv.cancel(t_drop)
        with pytest.raises(RuntimeError) as err:
            while srv.poll(t_drop, 1000) is None:
                pass
        assert err.value.status == L.QK_ERR_CANCELLED
        for t in t_busy + [t_keep]:
            while srv.poll(t, 1000) is None:
                pass
        assert not srv.cancel(t_keep)
        with pytest.raises(RuntimeError, match="unknown ticket"):
            srv.cancel(10_000)
