"""Multi-process helpers: one process per GPU, torch.distributed for the plumbing.

The single long pair does not shard (its wavefront is one chain of strips), so
N GPUs run N replicas: every rank times its own run and the job reports the
slowest rank (`max_over_ranks`) with the work of all ranks
(`replica_throughput`).  Batches shard naturally: pairs are independent, so a
batch splits by cell count, longest pair first, onto the least-loaded rank
(`lpt_shards`), each rank aligns its share with no collective during compute,
and the per-pair results are gathered back into the batch's order
(`gather_in_order`).  The same functions run under NCCL (device "cuda") and
under gloo on the CPU (device "cpu")."""
from __future__ import annotations

import heapq
from typing import List, Sequence


def max_over_ranks(ms: float, device: str = "cuda") -> float:
    """The largest `ms` over all ranks (a single process returns it unchanged)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(ms)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, units_per_rank: float, steps: int, max_ms: float) -> float:
    """Whole-job rate of `world` replicas that each processed `units_per_rank`
    per step for `steps` steps, timed as the slowest rank's `max_ms`."""
    return world * units_per_rank * steps / (max_ms * 1e-3)


def lpt_shards(weights: Sequence[float], world: int) -> List[List[int]]:
    """Indices of `weights` split over `world` ranks: heaviest first onto the
    least-loaded rank (ties: lower rank, then lower index).  Each shard keeps
    ascending index order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    heap = [(0.0, r) for r in range(world)]
    shards: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(weights[i]), r))
    return [sorted(s) for s in shards]


def gather_in_order(local: Sequence, shard: Sequence[int], n: int) -> list:
    """Every rank's per-pair results (local[k] belongs to pair shard[k]) in the
    batch's order, on every rank (all_gather_object)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        parts = [(list(shard), list(local))]
    else:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, (list(shard), list(local)))
    out = [None] * n
    for idx, vals in parts:
        if len(idx) != len(vals):
            raise ValueError("a rank's shard and results differ in length")
        for i, v in zip(idx, vals):
            if out[i] is not None:
                raise ValueError(f"pair {i} returned by two ranks")
            out[i] = v
    missing = [i for i, v in enumerate(out) if v is None]
    if missing:
        raise ValueError(f"pairs without a result: {missing[:8]}")
    return out
