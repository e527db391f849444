"""GPU: the C++ names of the reference's building blocks (include/quantkos_b200.hpp)
compiled into a program and run.

tests/cpp/boundary_names.cpp composes them as the reference's runners do
(execute_mc_framework + MSolver::execute_batch + OptionPricer for a forward option with
all Greeks; LSMEngine's statics for the reference-mode backward induction;
SDEScheme::evolve_step with a generator object) and checks each against the fused
engine; its PayoffTracker values on a fixed barrier-crossing sequence are checked here
against the oracle's payoff (pinned to the reference's PayoffTracker)."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


def test_cpp_building_blocks_against_fused_engine(qk, handle, oracle, tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    exe = tmp_path / "boundary_names"
    lib_dir = ROOT / "quantkos_b200"
    subprocess.run([gxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}",
                    str(ROOT / "tests" / "cpp" / "boundary_names.cpp"), f"-L{lib_dir}", "-lquantkos_b200",
                    f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True, capture_output=True, text=True)
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    lines = run.stdout.splitlines()
    fails = [ln for ln in lines if ln.startswith("FAIL")]
    assert run.returncode == 0 and not fails, run.stdout + run.stderr
    checks = [ln for ln in lines if ln.startswith("ok ")]
    assert len(checks) >= 18
    seq = np.array([float(x) for x in next(ln for ln in lines if ln.startswith("sequence")).split()[1:]])
    payoffs = [ln.split() for ln in lines if ln.startswith("payoff ")]
    assert len(payoffs) == 20
    for _, t, r, val in payoffs:
        t, r = int(t), int(r)
        B = 0.93 if t in (3, 5) else 1.08
        want = oracle.payoff_path(t, r, seq, 1.0, 1.02, B)
        assert float(val) == pytest.approx(want, rel=1e-12, abs=1e-15), (t, r)
