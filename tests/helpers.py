"""Shared helpers for the parity tests."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"

# Per-step parity tolerances (relative): FP64 1e-12, FP32 1e-5.
TOL_STEP_FP64 = 1e-12
TOL_STEP_FP32 = 1e-5


def load(name: str):
    return json.loads((GOLDEN / name).read_text())


def step_err(S, v, S_ref, v_ref, v_in) -> float:
    """Relative spot error; variance error relative to the variance level the step
    works with (max of input, output, 1e-8), since v' can be a cancellation of
    O(v) terms."""
    return max(abs(S - S_ref) / abs(S_ref), abs(v - v_ref) / max(abs(v_ref), abs(v_in), 1e-8))


def case_contract(make_contract, c: dict):
    return make_contract(S0=c["S"], v0=c["v"], r=c["r"], q=c["q"], model=c["model"], scheme=c["scheme"],
                         kappa=c["kappa"], theta=c["theta"], sigma=c["sigma"], rho=c["rho"],
                         lambda_j=c["lambda_j"], mu_j=c["mu_j"], sigma_j=c["sigma_j"], T=c["dt"], n_steps=1,
                         normalize=False)


def within_se(a: float, b: float, se_a: float, se_b: float, k: float = 3.0) -> bool:
    """|a - b| <= k * combined standard error."""
    return abs(a - b) <= k * float(np.hypot(se_a, se_b))
