"""Multi-GPU plumbing: one process per GPU.

A single collision does not shard (its 2S-1 wavefronts form one dependent chain), so the
benchmark runs independent replicas; independent collisions (the batched scan of many
collisions of uneven sizes) are partitioned across ranks with a size-balanced greedy
assignment and need no data-path collective.  Timing is the max over ranks."""
from __future__ import annotations

from typing import List, Sequence


def partition_collisions(costs: Sequence[float], world: int) -> List[List[int]]:
    """Longest-processing-time greedy: assign collisions (by decreasing cost) to the least
    loaded rank.  Deterministic: ties go to the lowest rank, equal costs keep index order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    load = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += float(costs[k])
    for p in parts:
        p.sort()
    return parts


def collision_cost(n1: int, n2: int, nslices: int, grid: int) -> float:
    """Relative cost of one collide: particle visits (S*(N1+N2)) plus S^2 field solves on a grid^2 mesh."""
    return float(nslices) * (n1 + n2) + 4.0 * nslices * nslices * grid * grid


def max_over_ranks(value: float, group=None) -> float:
    """All-reduce MAX of a per-rank float (a step time); identity without a process group."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def scan_partitioned(costs: Sequence[float], run_case, group=None):
    """Run a scan of independent collisions across the ranks of `group` (the default process group, or one
    rank when torch.distributed is not initialised): each rank runs its partition_collisions share with
    run_case(index) -> result, and every rank gets back the merged {index: result} of all ranks.  No
    data-path collective: the only exchange is this final gather of the (small, picklable) results."""
    import torch.distributed as dist
    distributed = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank(group) if distributed else 0
    world = dist.get_world_size(group) if distributed else 1
    mine = partition_collisions(costs, world)[rank]
    local = {k: run_case(k) for k in mine}
    if not distributed:
        return local
    parts = [None] * world
    dist.all_gather_object(parts, local, group=group)
    merged = {}
    for p in parts:
        merged.update(p)
    return merged
