"""The sharded pricer over a real NCCL process group on the GPU.

One GPU is available to these tests, so the group has one rank: that exercises the
NCCL initialisation, the default pricer's binding to the rank's GPU (LOCAL_RANK) and
the gather of the results, not the partitioning across ranks, which the gloo tests
with two ranks cover on the CPU.  The rank runs in a child process with a bounded
process-group timeout, so that the test process keeps no process group.
"""
from __future__ import annotations

import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

CHILD = r"""
import os, sys
from datetime import timedelta
sys.path.insert(0, os.environ["QK_ROOT"])
import torch
import torch.distributed as dist
torch.cuda.set_device(int(os.environ["LOCAL_RANK"]))
dist.init_process_group("nccl", timeout=timedelta(seconds=60), device_id=torch.device("cuda", 0))
import quantkos_b200 as qk
from quantkos_b200 import workloads as W
from quantkos_b200.distributed import local_device, price_sharded, rank_handle
cs = W.mixed_batch(24, seed=9)
for c in cs:
    c.n_paths = min(c.n_paths, 50_000)
g = W.batch_greeks()
res = price_sharded(cs, g)
assert local_device() == 0 and rank_handle().device == 0
ref = qk.price_batch(cs, g, qk.Handle(0))
keys = ("price", "std_error", "delta", "gamma", "vega", "rho", "theta")
for a, b in zip(res, ref):
    for la, lb in zip(a["legs"], b["legs"]):
        for k in keys:
            assert la[k] == lb[k], (k, la[k], lb[k])
dist.destroy_process_group()
print("sharded ok", len(res))
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_price_sharded_over_nccl_one_rank():
    """price_sharded with its default pricer under an NCCL group of one rank: the handle is
    bound to LOCAL_RANK's GPU and the gathered results, Greeks included, equal the batched
    engine's on the same contracts bit for bit."""
    env = dict(os.environ, QK_ROOT=str(ROOT), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()),
               RANK="0", WORLD_SIZE="1", LOCAL_RANK="0", NCCL_NVLS_ENABLE="0")
    proc = subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0, proc.stdout[-2000:] + proc.stderr[-4000:]
    assert "sharded ok 24" in proc.stdout
