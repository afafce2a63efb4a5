"""Multi-process host logic on CPU: two gloo ranks place, time and gather independent units.

The GPU step itself never exchanges data between ranks (a snapshot does not shard); these
tests cover the placement of whole units on ranks, the max-over-ranks job time and the
gathering of per-unit scalars, with world_size 2 on the gloo backend.
"""

import os
import socket

import pytest
import torch.multiprocessing as mp

import sharding


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_assign_units_covers_and_balances():
    # 48 units of the batched workload: four box sizes, 47 radii each (44 for 64^3)
    sizes = [64, 96, 128, 192] * 12
    costs = [sharding.unit_cost(n, 44 if n == 64 else 47) for n in sizes]
    for world in (1, 2, 3, 4, 8):
        parts = sharding.assign_units(costs, world)
        flat = sorted(u for p in parts for u in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[u] for u in p) for p in parts]
        # LPT is within 4/3 of the optimum; the optimum is at least the mean
        assert max(loads) <= 4.0 / 3.0 * max(sum(costs) / world, max(costs)) + 1e-6
    with pytest.raises(ValueError):
        sharding.assign_units(costs, 0)


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}")
    try:
        costs = [sharding.unit_cost(n, 40) for n in (64, 96, 128, 192, 64, 96)]
        mine = sharding.assign_units(costs, world)[rank]
        # each unit's "result": two FP64 scalars derived from the unit index
        local = {u: [u * 0.5, float(u) ** 2] for u in mine}
        t = sharding.max_over_ranks(10.0 + rank)
        got = sharding.gather_scalars(local, len(costs))
        q.put((rank, t, got))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_time_and_gather():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        rank, t, got = q.get(timeout=120)
        res[rank] = (t, got)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][0] == 11.0 and res[1][0] == 11.0
    assert res[1][1] is None
    assert res[0][1] == [[u * 0.5, float(u) ** 2] for u in range(6)]


def test_gather_rejects_duplicates_and_gaps_single_process():
    assert sharding.gather_scalars({0: [1.0], 1: [2.0]}, 2) == [[1.0], [2.0]]
    with pytest.raises(ValueError):
        sharding.gather_scalars({0: [1.0]}, 2)
