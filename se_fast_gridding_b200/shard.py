"""Independent systems across ranks (one process per GPU).

A single SE system does not shard cheaply (a P-1 halo exchange and a
distributed FFT would be needed) and the largest configuration fits one B200,
so multi-GPU runs split *batches* of independent systems: each rank solves
its share with one BatchSolver and the results are gathered on the host.
There is no data-path collective; the only exchange is the host-side gather
of per-system outputs and timings.
"""
from __future__ import annotations

import math
from typing import Callable, Sequence


def system_cost(s) -> float:
    """Relative work of one system: spread + interpolation (N P^3) and the
    FFTs (M^3 log M)."""
    return float(s.N) * s.P ** 3 + float(s.M) ** 3 * math.log2(max(s.M, 2))


def partition(items: Sequence, world: int, cost: Callable = system_cost) -> list[list[int]]:
    """Greedy longest-first assignment of items to `world` ranks by cost.
    Deterministic: ties break by index, so every rank computes the same
    assignment without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(items)), key=lambda i: (-cost(items[i]), i))
    load = [0.0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += cost(items[i])
    return [sorted(s) for s in shards]


def admit(items: Sequence, budget_bytes: int, footprint: Callable) -> tuple[list[int], list[int]]:
    """Split items (in order) into those that fit a device-memory budget and
    the rest."""
    taken, rest, used = [], [], 0
    for i, it in enumerate(items):
        b = footprint(it)
        if used + b <= budget_bytes:
            taken.append(i)
            used += b
        else:
            rest.append(i)
    return taken, rest


def gather_outputs(local_idx: Sequence[int], local_out: Sequence, nsys: int, group=None):
    """Collect per-system outputs from every rank into global order on all
    ranks (host objects through torch.distributed's object collectives)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    pieces = [None] * world
    dist.all_gather_object(pieces, list(zip(local_idx, local_out)), group=group)
    out = [None] * nsys
    for part in pieces:
        for i, o in part:
            out[i] = o
    return out


def max_over_ranks(value: float, group=None) -> float:
    """The largest of a host float across ranks (timings are max-over-ranks)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
