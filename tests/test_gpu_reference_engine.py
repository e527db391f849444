"""GPU: the engine against the reference's own engine (oracle/_ref), each side with
its own random numbers, within 3 combined standard errors.

The cases are those of test_reference_engine.py (tests/refcases.py): every payoff
type and right under three (model, scheme) pairs; all seven Greeks by
replication; the reference-mode American put (Laguerre basis, every step an
exercise date) against ForwardBackwardMCRunner.  The engine prices them with the
plain FP64 method and with the batched FP32 engine; the reference runs its FP64
build on the host cores with a pinned thread count.
"""
import pytest

import refcases as RC

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pinned_ref(ref):
    ref.set_threads(RC.REF_THREADS)
    return ref


@pytest.mark.parametrize("model,scheme", RC.PRICE_KINDS)
def test_engine_prices_every_payoff_vs_reference_engine(qk, handle, pinned_ref, model, scheme):
    L = qk.lib
    ks64 = [RC.price_case(qk.make_contract, L, model, scheme, t, right) for t in range(10) for right in (0, 1)]
    ks32 = [RC.price_case(qk.make_contract, L, model, scheme, t, right, precision=L.FP32)
            for t in range(10) for right in (0, 1)]
    plain = [qk.price_plain(k, None, handle)["legs"][0] for k in ks64]
    batch = [r["legs"][0] for r in qk.price_batch(ks32, None, handle)]
    for i, k in enumerate(ks64):
        t, right = k.payoffs[0].type, k.payoffs[0].right
        r = pinned_ref.price(pinned_ref.from_contract(k, seed=RC.ref_price_seed(t, right)))
        for name, e in (("plain FP64", plain[i]), ("batched FP32", batch[i])):
            z = RC.z_score(e["price"], r["price"], e["std_error"], r["std_error"])
            assert z <= RC.K_SE, (name, model, scheme, t, right, e, r)
            assert abs(e["std_error"] / r["std_error"] - 1.0) < 0.25


@pytest.mark.parametrize("case", RC.GREEK_CASES)
def test_engine_greeks_vs_reference_engine(qk, handle, pinned_ref, case):
    L = qk.lib
    b = RC.GREEK_BUMPS
    g = qk.make_greeks(L.GREEK_ALL, vega_mode=0, bump_S_rel=b["bump_S_rel"], bump_vol=b["bump_vol"],
                       bump_r_abs=b["bump_r_abs"], bump_T_abs=b["bump_T_abs"])
    cols = ("price",) + RC.GREEK_NAMES
    reps = range(RC.GREEK_REPS)
    r_rows = []
    for rep in reps:
        k = RC.greek_case(qk.make_contract, L, *case, rep)
        r = pinned_ref.price(RC.ref_greek_config(pinned_ref, k, rep))
        r_rows.append([r[c] for c in cols])
    mr, sr = RC.replicated(r_rows)
    for prec in (L.FP64, L.FP32):
        ks = [RC.greek_case(qk.make_contract, L, *case, rep, precision=prec) for rep in reps]
        rows = [[res["legs"][0][c] for c in cols] for res in qk.price_batch(ks, g, handle)]
        me, se = RC.replicated(rows)
        for j, c in enumerate(cols):
            z = RC.z_score(me[j], mr[j], se[j], sr[j])
            assert z <= RC.K_SE, (case, prec, c, me[j], se[j], mr[j], sr[j])


@pytest.mark.parametrize("case", RC.AMERICAN_CASES)
def test_engine_american_reference_mode_vs_reference_engine(qk, handle, pinned_ref, case):
    L = qk.lib
    k64 = RC.american_case(qk.make_contract, L, *case)
    k32 = RC.american_case(qk.make_contract, L, *case, precision=L.FP32)
    r = pinned_ref.price(pinned_ref.from_contract(k64, seed=4242))
    for name, e in (("plain FP64", qk.price_plain(k64, None, handle)["legs"][0]),
                    ("batched FP32", qk.price_batch([k32], None, handle)[0]["legs"][0])):
        assert RC.z_score(e["price"], r["price"], e["std_error"], r["std_error"]) <= RC.K_SE, (name, case, e, r)
        assert abs(e["std_error"] / r["std_error"] - 1.0) < 0.1
        assert abs(e["prob_itm"] - r["prob_itm"]) < 0.01
