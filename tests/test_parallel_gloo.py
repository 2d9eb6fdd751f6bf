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


# Scan cases small enough for the CPU oracle: (n1, n2, slices1, slices2, grid, aspect, seed)
SCAN_CASES = [(3000, 2000, 3, 4, 32, 1.0, 11), (5000, 3000, 5, 3, 32, 4.0, 12), (2000, 4000, 4, 4, 32, 11.0, 13),
              (4000, 1500, 2, 5, 32, 25.0, 14), (2500, 2500, 3, 3, 32, 2.0, 15)]


def _scan_case(k):
    """One case's collide on the CPU oracle (deterministic); its luminosity and a digest of both beams."""
    import hashlib
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    from oracle import oracle as orc
    n1, n2, s1, s2, g, aspect, seed = SCAN_CASES[k]
    sy = 8.5e-6
    e = orc.beam_gaussian(n1, seed=seed, rng_id=1, beta=(0.55, 0.056, 12.7), sigma=(aspect * sy, sy, 7e-3))
    p = orc.beam_gaussian(n2, seed=seed, rng_id=2, beta=(0.8, 0.072, 90.9), sigma=(aspect * sy, sy, 6e-2))
    o = orc.Oracle(orc.OracleOptions(grid=(g, g), nslices1=s1, nslices2=s2))
    lum = o.collide(e, p, orc.beam_params(-1.0, orc.EMASS_EV, 10e9, 1.7e11), orc.beam_params(1.0, orc.PMASS_EV, 275e9, 6.9e10))
    return lum, hashlib.sha256(e.tobytes() + p.tobytes()).hexdigest()


def _scan_costs():
    return [collision_cost(n1, n2, max(s1, s2), g) for n1, n2, s1, s2, g, _, _ in SCAN_CASES]


def _scan_worker(rank, world, port, q):
    import torch.distributed as dist
    from octo_b200.parallel import partition_collisions, scan_partitioned
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = partition_collisions(_scan_costs(), world)[rank]
        merged = scan_partitioned(_scan_costs(), _scan_case)
        q.put((rank, mine, merged))
    finally:
        dist.destroy_process_group()


def test_partitioned_scan_equals_the_single_rank_scan():
    """Two gloo ranks run their shares of a scan of independent collides (the oracle on the CPU): the merged
    luminosities and final beams equal the single-rank scan's bit for bit, and each case ran once."""
    from octo_b200.parallel import scan_partitioned
    single = scan_partitioned(_scan_costs(), _scan_case)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_scan_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(res[0][1] + res[1][1]) == list(range(len(SCAN_CASES)))  # a partition: every case exactly once
    assert res[0][1] and res[1][1]
    for _, _, merged in res:
        assert merged == single
