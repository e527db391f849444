"""Multi-GPU pricing: one process per GPU, contracts sharded across ranks.

Paths within a contract and contracts within a batch are independent, and every
path's random numbers are keyed by (seed, stream, path, step) only, so a
contract's price does not depend on which GPU prices it.  The data path needs no
collective: each rank prices its shard with the batched engine on its own GPU;
the only exchange is the per-contract results (a few hundred bytes each),
gathered once.

Sharding is greedy longest-processing-time on the path-step cost of each
contract (with its Greek bumps), deterministic for a given contract list.
"""
from __future__ import annotations

import heapq
import os
from typing import Callable, Sequence


def contract_cost(c, n_tasks: int = 1) -> float:
    return float(c.n_paths) * float(c.n_steps) * float(n_tasks) * (1.25 if c.model == 1 else 1.0)


def shard_contracts(contracts: Sequence, world: int, n_tasks: int = 1) -> list[list[int]]:
    """Indices of the contracts each rank prices (LPT on path-step cost; ties by index)."""
    order = sorted(range(len(contracts)), key=lambda i: (-contract_cost(contracts[i], n_tasks), i))
    heap = [(0.0, r) for r in range(world)]
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + contract_cost(contracts[i], n_tasks), r))
    for s in shards:
        s.sort()
    return shards


def local_device() -> int:
    """The GPU this process prices on: LOCAL_RANK when launched one process per GPU
    (torchrun sets it), else torch's current CUDA device, else 0."""
    lr = os.environ.get("LOCAL_RANK")
    if lr is not None and lr.strip():
        return int(lr)
    try:
        import torch
        if torch.cuda.is_available():
            return int(torch.cuda.current_device())
    except Exception:
        pass
    return 0


_rank_handles: dict = {}


def rank_handle(device: int | None = None, factory: Callable | None = None):
    """One engine handle per (process, device), created on first use and reused by
    later sharded pricings.  `factory(device)` builds it (default: engine.Handle)."""
    dev = local_device() if device is None else int(device)
    key = (dev, factory)
    h = _rank_handles.get(key)
    if h is None:
        if factory is None:
            from .engine import Handle
            factory = Handle
        h = factory(dev)
        _rank_handles[key] = h
    return h


def price_sharded(contracts: Sequence, greeks=None, group=None,
                  pricer: Callable | None = None, handle_factory: Callable | None = None) -> list[dict] | None:
    """Price `contracts` across the ranks of `group` (torch.distributed, any backend).

    Every rank passes the same contract list.  Rank r prices shard r with `pricer`
    (default: the batched engine on this rank's GPU, `local_device()`, through a
    handle that `handle_factory(device)` builds once per process) and rank 0 returns
    the results in the original order; other ranks return None."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    n_tasks = 1
    if greeks is not None and greeks.mask:
        from .workloads import path_steps
        n_tasks = int(round(path_steps([contracts[0]], greeks) / path_steps([contracts[0]])))
    shards = shard_contracts(contracts, world, n_tasks)
    mine = shards[rank]
    if pricer is None:
        handle = rank_handle(None, handle_factory)

        def pricer(cs, g):
            from .engine import price_batch
            return price_batch(cs, g, handle)
    results = pricer([contracts[i] for i in mine], greeks) if mine else []
    gathered: list = [None] * world if rank == 0 else None
    dist.gather_object(list(zip(mine, results)), gathered, dst=0, group=group)
    if rank != 0:
        return None
    out: list = [None] * len(contracts)
    for part in gathered:
        for i, r in part:
            out[i] = r
    return out
