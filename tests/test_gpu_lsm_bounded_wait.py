"""GPU: the bounded grid-wide wait of the persistent Longstaff-Schwartz launch.

The backward induction of an American job is one cooperative launch whose blocks
wait for each exercise date's coefficients.  Here one block is told (test hook
qk_debug_lsm_withhold_block) to leave before it arrives, so nothing ever publishes
the next date: every other block's wait must run out after about a second, the call
must return QK_ERR_TIMEOUT, and the same handle must price correctly afterwards.
No device fault is involved: the failure is an argument the host passes.
"""
import ctypes as C
import time

import pytest

pytestmark = pytest.mark.gpu


def _american(qk, precision):
    return qk.make_contract(model=qk.HESTON, scheme=qk.ANDERSEN_QE, n_paths=300_000, n_steps=40, T=1.0, seed=5,
                            precision=precision, payoffs=[qk.payoff(qk.AMERICAN, qk.PUT, 100.0)],
                            lsm_basis=qk.LSM_POLY_SV, lsm_dates=10)


@pytest.mark.parametrize("precision", ["FP32", "FP64"])
def test_withheld_block_times_out_and_handle_recovers(qk, precision):
    prec = getattr(qk, precision)
    k = _american(qk, prec)
    with qk.Handle(0) as h:
        want = qk.price_batch([k], None, h)[0]["legs"][0]
        assert qk.lib.lib().qk_debug_lsm_withhold_block(h.ptr, 0) == qk.lib.QK_OK
        t0 = time.perf_counter()
        with pytest.raises(qk.QuantKosError) as err:
            qk.price_batch([k], None, h)
        waited = time.perf_counter() - t0
        assert err.value.status == qk.lib.QK_ERR_TIMEOUT
        assert b"bounded wait" in qk.lib.lib().qk_last_error()
        assert 0.2 < waited < 30.0
        assert qk.lib.lib().qk_debug_lsm_withhold_block(h.ptr, -1) == qk.lib.QK_OK
        got = qk.price_batch([k], None, h)[0]["legs"][0]
        assert got["price"] == want["price"] and got["std_error"] == want["std_error"]
        # forward pricing on the same device is unaffected
        e = qk.price_batch([qk.make_contract(n_paths=50_000, n_steps=16, precision=prec)], None, h)[0]
        assert e["legs"][0]["price"] > 0.0
