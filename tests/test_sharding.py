"""Sharding of independent instances over ranks: the LPT partition and the result gather over a
world_size-2 gloo process group on CPU (the multi-rank path of the batched bench workload)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from featb200 import sharding


def test_lpt_partition_covers_and_balances():
    rng = np.random.default_rng(3)
    levels = rng.integers(5, 10, size=256)
    costs = [(2 ** int(l) + 1) ** 2 for l in levels]
    for world in (1, 2, 3, 4, 8):
        parts = sharding.lpt_partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        ld = sharding.loads(costs, parts)
        # LPT bound: max load <= (4/3 - 1/(3m)) OPT, OPT >= max(mean, largest)
        opt_lb = max(sum(costs) / world, max(costs))
        assert max(ld) <= (4.0 / 3.0 - 1.0 / (3 * world)) * opt_lb + 1e-9
        assert parts == sharding.lpt_partition(costs, world)   # deterministic


def test_lpt_edge_cases():
    assert sharding.lpt_partition([], 3) == [[], [], []]
    assert sharding.lpt_partition([5.0], 2) == [[0], []]
    assert sharding.lpt_partition([1.0, 1.0, 1.0, 1.0], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        sharding.lpt_partition([1.0], 0)
    with pytest.raises(ValueError):
        sharding.shard([1.0], 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, costs, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = sharding.shard(costs, rank, world)
        vals = [float(i) * 10.0 + rank * 0.0 for i in mine]   # stand-in per-instance result
        allv = sharding.gather_results(dist, rank, world, mine, vals, len(costs))
        q.put((rank, mine, allv))
    finally:
        dist.destroy_process_group()


def test_gather_two_ranks_gloo():
    costs = [float((2 ** l + 1) ** 2) for l in (5, 9, 7, 6, 8, 9, 5, 5, 7)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    owned = sorted(res[0][1] + res[1][1])
    assert owned == list(range(len(costs)))
    assert set(res[0][1]).isdisjoint(res[1][1])
    for _, _, allv in res:
        assert allv == [float(i) * 10.0 for i in range(len(costs))]
