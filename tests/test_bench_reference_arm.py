"""bench.py's reference arm — the reference's own pricing code on the host cores, timed
for the same metric and workload as the GPU arm — needs no GPU, so its one-line JSON
contract is checked here: the keys a reader of the line relies on, and that under
torchrun only rank 0 prints it."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _run(extra_env=None):
    env = dict(os.environ, **(extra_env or {}))
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0",
           "--cpu-sample-paths", "2048"]
    return subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)


def test_reference_arm_prints_the_contract_line():
    out = _run()
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "path-steps/s" and line["unit"] == "path-steps/s" and line["value"] > 0
    for key in ("n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling", "vs_baseline", "dtype",
                "data", "config"):
        assert key in line, key
    assert line["config"]["workload"] == "bates_qe_5payoff_16777216x252_fp32"
    base = line["cpu_baseline"]
    assert base["kind"] in ("reference", "port") and base["cores"] >= 1 and base["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "path-steps/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_runs_on_rank_zero_only():
    out = _run({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == ""
