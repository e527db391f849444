"""GPU: the allocation-free entry point qk_price_noalloc.

It exists for callers that must not allocate device memory while pricing (a host
application that owns all GPU memory through its own pool, or a latency-critical
caller that cannot pay for cudaMalloc/cudaFree between requests).  It uses one
fixed device array for all its scratch.  This file is collected last on purpose:
the checks below must hold in a fresh process and after every other test, and a
failure here must not hide any other test's result.

Checked through the C ABI: two calls in a row give the same prices as the
regular batched entry point on the same contract (relative 1e-12: same kernel,
same paths, only the tile merge order may differ), the shared array carries no
state from one call into the next, and requests beyond the fixed size are
rejected with a clear error; and once the first call on the device (its set-up)
has run, a further call leaves the device's free memory unchanged.
"""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def _call(qk, contract):
    out = qk.lib.Result()
    st = qk.lib.lib().qk_price_noalloc(C.byref(contract), None, C.byref(out))
    return st, out


def test_noalloc_matches_batched_entry_point_twice(qk, handle):
    legs = [qk.payoff(qk.EUROPEAN, qk.CALL, 100.0), qk.payoff(qk.ASIAN, qk.CALL, 100.0),
            qk.payoff(qk.BARRIER_UP_OUT, qk.CALL, 100.0, 130.0), qk.payoff(qk.LOOKBACK_FLOATING, qk.PUT, 100.0),
            qk.payoff(qk.BINARY_CASH, qk.CALL, 105.0)]
    for precision in (qk.FP32, qk.FP64):
        k = qk.make_contract(model=qk.BATES, scheme=qk.ANDERSEN_QE, lambda_j=0.1, mu_j=-0.05, sigma_j=0.1,
                             n_paths=1_000_003, n_steps=100, seed=1234, precision=precision, payoffs=legs)
        want = qk.price_batch([k], None, handle)[0]["legs"]
        for _ in range(2):
            st, out = _call(qk, k)
            assert st == qk.lib.QK_OK, qk.lib.lib().qk_last_error()
            assert out.n_payoffs == 5 and out.n_paths == 1_000_003
            for i, w in enumerate(want):
                assert out.p[i].price == pytest.approx(w["price"], rel=1e-12)
                assert out.p[i].std_error == pytest.approx(w["std_error"], rel=1e-9)
                assert out.p[i].prob_itm == pytest.approx(w["prob_itm"], abs=1e-12)


def test_noalloc_carries_no_state_between_calls(qk, handle):
    small = qk.make_contract(n_paths=5_000, n_steps=20, seed=7, precision=qk.FP64)
    big = qk.make_contract(n_paths=3_000_000, n_steps=20, seed=8, precision=qk.FP64)
    st, a = _call(qk, small)
    assert st == qk.lib.QK_OK
    st, _ = _call(qk, big)
    assert st == qk.lib.QK_OK
    st, b = _call(qk, small)
    assert st == qk.lib.QK_OK
    assert a.p[0].price == b.p[0].price and a.p[0].std_error == b.p[0].std_error


def test_noalloc_rejects_oversized_requests(qk, handle):
    legs = [qk.payoff(qk.EUROPEAN, qk.CALL, 100.0 + i) for i in range(8)]
    k = qk.make_contract(n_paths=40_000_000, n_steps=4, payoffs=legs)  # 19532 tiles x 8 legs > 131072
    st, _ = _call(qk, k)
    assert st == qk.lib.QK_ERR_CAPACITY
    assert b"131072" in qk.lib.lib().qk_last_error()
    k = qk.make_contract(payoffs=[qk.payoff(qk.AMERICAN, qk.PUT, 100.0)])
    st, _ = _call(qk, k)
    assert st == qk.lib.QK_ERR_UNSUPPORTED


def test_noalloc_call_after_setup_allocates_no_device_memory(qk, handle):
    """The property the entry point exists for: once the first call on the device
    (its set-up) has run, another call leaves the device's free memory unchanged."""
    import torch

    torch.cuda.mem_get_info(0)  # torch's own CUDA state is set up before measuring
    k = qk.make_contract(model=qk.HESTON, scheme=qk.ANDERSEN_QE, n_paths=2_000_000, n_steps=32, seed=99,
                         precision=qk.FP32, payoffs=[qk.payoff(qk.EUROPEAN, qk.CALL, 100.0),
                                                     qk.payoff(qk.ASIAN, qk.PUT, 95.0)])
    st, first = _call(qk, k)  # set-up: loads the kernels and reserves the array on this device
    assert st == qk.lib.QK_OK, qk.lib.lib().qk_last_error()
    free_before, _ = torch.cuda.mem_get_info(0)
    st, second = _call(qk, k)
    free_after, _ = torch.cuda.mem_get_info(0)
    assert st == qk.lib.QK_OK, qk.lib.lib().qk_last_error()
    assert free_after == free_before
    assert second.p[0].price == first.p[0].price and second.p[1].price == first.p[1].price
