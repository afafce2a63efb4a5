"""Host-side plumbing for running independent reionization units on several ranks.

A unit is one snapshot of one box.  A single box does not shard (the whole grid fits one
B200 and slab exchange is not used), so multi-GPU work is independent units placed whole on
ranks (one process per GPU, torch.distributed over NCCL on a GPU box, gloo in the CPU tests):

* ``assign_units`` balances units over ranks by their cost (N^3 times the filtered grids
  over all radii), longest first onto the least loaded rank;
* ``max_over_ranks`` gives the job time (the slowest rank);
* ``gather_scalars`` collects each unit's FP64 scalars on rank 0 in unit order.

No grid data crosses ranks.
"""

from __future__ import annotations

import heapq


def unit_cost(n: int, radii: int, shells: int = 0) -> float:
    """Relative cost of one unit: cells times (radius passes + shell passes + 1)."""
    return float(n) ** 3 * (radii + shells + 1)


def assign_units(costs: list[float], world: int) -> list[list[int]]:
    """Longest-processing-time-first placement: returns, per rank, the unit indices in
    ascending order.  Every unit lands on exactly one rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for u in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        load, r = heapq.heappop(heap)
        out[r].append(u)
        heapq.heappush(heap, (load + costs[u], r))
    return [sorted(x) for x in out]


def max_over_ranks(value: float, group=None) -> float:
    """The maximum of ``value`` over the ranks of ``group`` (the value itself without one)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_scalars(local: dict[int, list[float]], n_units: int, group=None):
    """Rank 0 receives [n_units] lists of scalars (each unit's, in unit order); other ranks
    receive None.  Every unit must be reported by exactly one rank."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        parts = [local]
    else:
        parts = [None] * dist.get_world_size(group)
        dist.all_gather_object(parts, local, group=group)
        if dist.get_rank(group) != 0:
            return None
    out: list = [None] * n_units
    for part in parts:
        for u, vals in part.items():
            if out[u] is not None:
                raise ValueError(f"unit {u} reported twice")
            out[u] = list(vals)
    missing = [u for u, v in enumerate(out) if v is None]
    if missing:
        raise ValueError(f"units {missing} were not reported")
    return out
