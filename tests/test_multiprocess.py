"""CPU, world size 2 over gloo: contract sharding and the result gather.

Each rank prices its shard with the oracle as a stand-in pricer (no GPU); the
gathered results must equal a single-process pricing of the whole list bit for
bit, because every path's draws depend only on (seed, stream, path, step)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from quantkos_b200.distributed import shard_contracts


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _contracts():
    from quantkos_b200 import _lib as L
    from quantkos_b200.engine import make_contract, payoff
    out = []
    for i in range(9):
        out.append(make_contract(model=i % 2, scheme=i % 3, lambda_j=0.3 if i % 2 else 0.0, mu_j=-0.1, sigma_j=0.1,
                                 n_paths=1000 + 500 * i, n_steps=8 + i, seed=77, stream=i, precision=L.FP64,
                                 payoffs=[payoff(i % 4, i % 2, 95.0 + i, 120.0)]))
    return out


def _oracle_pricer(cs, g):
    from oracle import qkoracle
    return [qkoracle.price(c, g) for c in cs]


def _worker(rank, world, port, q):
    import torch.distributed as dist

    from quantkos_b200.distributed import price_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = price_sharded(_contracts(), None, None, _oracle_pricer)
        if rank == 0:
            q.put([r["legs"][0]["price"] for r in res])
    finally:
        dist.destroy_process_group()


def test_shards_balance_and_cover():
    cs = _contracts()
    shards = shard_contracts(cs, 2)
    assert sorted(shards[0] + shards[1]) == list(range(len(cs)))
    loads = [sum(c.n_paths * c.n_steps for i, c in enumerate(cs) if i in s) for s in shards]
    assert max(loads) / min(loads) < 1.3
    assert shard_contracts(cs, 2) == shards  # deterministic


def test_sharded_pricing_equals_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=240)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    want = [r["legs"][0]["price"] for r in _oracle_pricer(_contracts(), None)]
    assert got == want


def test_failed_rank_surfaces_as_error():
    """A rank that raises before the gather makes the other rank's gather fail with an
    error within the process-group timeout (no hang)."""
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert procs[1].exitcode != 0  # the failing rank
    assert procs[0].exitcode is not None  # the survivor finished (with an error), it did not hang


def _failing_worker(rank, world, port):
    from datetime import timedelta

    import torch.distributed as dist

    from quantkos_b200.distributed import price_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=10))

    def pricer(cs, g):
        if rank == 1:
            raise RuntimeError("injected pricing failure on rank 1")
        return _oracle_pricer(cs, g)

    try:
        price_sharded(_contracts(), None, None, pricer)
    except Exception:
        os._exit(3 if rank == 1 else 4)
    os._exit(0)


class _FakeHandle:
    def __init__(self, device):
        self.device = device


def _binding_worker(rank, world, port, q):
    """Default pricer of price_sharded under one-process-per-GPU launch: the engine
    entry point is replaced by a recorder, the handle factory by a fake, so the
    test sees which device each rank's handle was built for without a GPU."""
    import torch.distributed as dist

    import quantkos_b200.engine as engine
    from quantkos_b200.distributed import price_sharded, rank_handle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["LOCAL_RANK"] = str(rank)
    seen = []

    def recording_price_batch(cs, g, handle):
        seen.append(handle.device)
        return _oracle_pricer(cs, g)

    engine.price_batch = recording_price_batch
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = price_sharded(_contracts(), None, None, None, _FakeHandle)
        again = rank_handle(None, _FakeHandle)  # cached: the same handle on a second call
        price_sharded(_contracts(), None, None, None, _FakeHandle)
        payload = {"rank": rank, "devices": seen, "cached": rank_handle(None, _FakeHandle) is again}
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(payload, gathered, dst=0)
        if rank == 0:
            q.put((gathered, [r["legs"][0]["price"] for r in res]))
    finally:
        dist.destroy_process_group()


def test_default_pricer_binds_each_rank_to_its_local_gpu():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_binding_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, prices = q.get(timeout=240)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for entry in gathered:
        assert entry["devices"] and all(d == entry["rank"] for d in entry["devices"])
        assert entry["cached"]
    assert prices == [r["legs"][0]["price"] for r in _oracle_pricer(_contracts(), None)]
