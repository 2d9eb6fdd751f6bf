"""Multi-rank host logic on CPU (gloo, world size 2): the collision partition and max-over-ranks timing."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from octo_b200.parallel import collision_cost, partition_collisions


def test_partition_is_balanced_and_complete():
    costs = [collision_cost(n, n // 2, s, g) for n, s, g in
             [(64000, 5, 64), (2560000, 31, 256), (300000, 15, 128), (1000000, 9, 96), (80000, 27, 64),
              (1500000, 13, 128), (700000, 21, 256), (120000, 7, 96)]]
    for world in (1, 2, 4, 8):
        parts = partition_collisions(costs, world)
        assert sorted(k for p in parts for k in p) == list(range(len(costs)))
        loads = [sum(costs[k] for k in p) for p in parts]
        assert max(loads) <= max(costs) + sum(costs) / world + 1e-9  # LPT bound
    assert partition_collisions(costs, 2) == partition_collisions(costs, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from octo_b200.parallel import max_over_ranks, partition_collisions
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = max_over_ranks(1.0 + rank)
        mine = partition_collisions([5, 1, 4, 2, 3], world)[rank]
        q.put((rank, t, mine))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_partition_with_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2.0, 2.0]
    assert sorted(res[0][2] + res[1][2]) == [0, 1, 2, 3, 4]
