"""Host-side helpers for running lattices on several GPUs, one process per GPU.

The single-lattice step does not shard across GPUs here; what does shard is an *ensemble* of
independent lattices: each rank advances its own subset in one batch and no data crosses GPUs.
``lpt_assign`` balances the subsets (greedy longest-processing-time on the per-member cost, e.g. cells
x steps x bytes per cell update), and ``max_over_ranks`` is the timing reduction every multi-rank
measurement uses (the job takes as long as its slowest rank).
"""
from __future__ import annotations

from typing import Sequence


def lpt_assign(costs: Sequence[float], n_ranks: int) -> list[list[int]]:
    """Greedy LPT: members in decreasing cost order, each to the currently least-loaded rank.

    Returns one list of member indices per rank (each list ascending).  Deterministic: ties go to the
    lower member index and the lower rank.  The makespan is within 4/3 of the optimum (Graham 1969).
    """
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    loads = [0.0] * n_ranks
    parts: list[list[int]] = [[] for _ in range(n_ranks)]
    for k in order:
        r = min(range(n_ranks), key=lambda j: (loads[j], j))
        parts[r].append(k)
        loads[r] += float(costs[k])
    return [sorted(p) for p in parts]


def rank_loads(costs: Sequence[float], parts: Sequence[Sequence[int]]) -> list[float]:
    return [float(sum(costs[k] for k in p)) for p in parts]


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar over the default process group (identity without one).

    ``device``: where the reduction tensor lives — a CUDA device for NCCL, None (CPU) for gloo.
    """
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
