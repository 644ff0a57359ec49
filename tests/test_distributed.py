"""The multi-process path on CPU: instance sharding, result gathering and max-over-ranks timing
with two gloo ranks (the data path has no collective; ranks only exchange small outputs)."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out) -> None:
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from oracle.shim import SpatialDiscretizationModule
        from pyeulerale_b200 import grid as G
        from pyeulerale_b200.batch import gather, max_over_ranks, shard

        items = list(range(5))  # five instances of different sizes and flows
        mine = shard(items, rank, world)
        ora = SpatialDiscretizationModule()
        local = []
        for i in mine:
            X = G.naca_ogrid(9 + i, 11 + 2 * i, 0.12, 1.0, 20.0, 0.05)
            M, N = X.shape[1] - 1, X.shape[2] - 1
            U = G.perturbed_states(M, N, 0.3 + 0.05 * i, 1.0 - i, 0.01,
                                   np.random.default_rng(i))
            ora.aoa[...] = 1.0 - i
            R = np.asfortranarray(np.zeros((4, M, N), dtype=complex))
            ora.compute_odes(0.3 + 0.05 * i, np.asfortranarray(X, dtype=complex),
                             np.zeros_like(X, dtype=complex), np.asfortranarray(U, dtype=complex), R)
            local.append((i, float(np.max(np.abs(R)))))
        allres = gather(local)
        t = max_over_ranks(1.0 + rank)
        out.put((rank, mine, allres, t))
    finally:
        dist.destroy_process_group()


def test_two_rank_shard_gather_and_timing():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    (r0, mine0, all0, t0), (r1, mine1, all1, t1) = results
    assert mine0 + mine1 == list(range(5)) and abs(len(mine0) - len(mine1)) <= 1
    assert all0 == all1 and [i for i, _ in all0] == list(range(5))
    assert t0 == t1 == 2.0


@pytest.mark.parametrize("world", [1, 3, 4, 8])
def test_shard_covers_in_order(world):
    from pyeulerale_b200.batch import shard

    items = list(range(48))
    parts = [shard(items, r, world) for r in range(world)]
    assert sum(parts, []) == items
    assert max(map(len, parts)) - min(map(len, parts)) <= 1
