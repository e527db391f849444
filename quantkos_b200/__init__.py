"""B200-native Monte Carlo hot path of QuantKos (Heston/Bates, Euler/Milstein/QE,
exotic payoffs, Longstaff-Schwartz, finite-difference Greeks) behind a C ABI.

The first call into the engine loads the in-tree CUDA library
(``libquantkos_b200.so``); there is no CPU fallback: if the library is missing that
call raises ImportError.
"""
from . import _lib as lib  # noqa: F401
from ._lib import (ANDERSEN_QE, AMERICAN, ASIAN, BARRIER_DOWN_IN, BARRIER_DOWN_OUT, BARRIER_UP_IN,  # noqa: F401
                   BARRIER_UP_OUT, BATES, BINARY_ASSET, BINARY_CASH, CALL, EULER, EUROPEAN, FP32, FP64,
                   GREEK_ALL, GREEK_DELTA_GAMMA, GREEK_RHO, GREEK_THETA, GREEK_VANNA, GREEK_VEGA_VOMMA, HESTON,
                   IMPLICIT_MILSTEIN, LOOKBACK_FIXED, LOOKBACK_FLOATING, LSM_LAGUERRE3, LSM_POLY_SV, PUT)
from .engine import (Handle, MCDispatcher, MCGreeks, MCOpPrices, MCResults, Parser, PreparedBatch,  # noqa: F401
                     QuantKosError, QuantKosInvalidArgument, Server, UInputs, default_handle, make_contract,
                     make_greeks, n_steps_for, paths, payoff, price_batch, price_noalloc, price_plain, step_trace)


def load_native():
    """dlopen the CUDA library now (raises ImportError when it is not built)."""
    return lib.lib()

__version__ = "1.0.0"
