"""Ensembles over several GPUs: one process per GPU, members sharded.

The members of an ensemble are independent basins, so a multi-GPU run needs
no data-path exchange: every rank advances its own share of the members in
one batch context (``efdc_xm.BatchSolver``), and only per-member results and
timings meet at the end.  The share is balanced by wet-cell count (the cost of
a member is proportional to its cells x iterations, and the cells are known
up front): longest-processing-time greedy, largest member first to the least
loaded rank.

The collectives go through ``torch.distributed`` (NCCL on GPUs, gloo on CPU);
the calls are the same on every rank and in the same order.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def partition(sizes: Sequence[int], nranks: int) -> list[list[int]]:
    """Split member indices over `nranks` ranks, balancing the sum of sizes.

    Deterministic (ties go to the lower rank, members in index order within a
    rank).  Every member appears on exactly one rank."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k))
    heap = [(0, r) for r in range(nranks)]
    parts: list[list[int]] = [[] for _ in range(nranks)]
    for k in order:
        load, r = heapq.heappop(heap)
        parts[r].append(k)
        heapq.heappush(heap, (load + int(sizes[k]), r))
    return [sorted(p) for p in parts]


def imbalance(sizes: Sequence[int], parts: list[list[int]]) -> float:
    """Largest rank load over the mean load (1.0 = perfect balance)."""
    loads = [sum(int(sizes[k]) for k in p) for p in parts]
    mean = sum(loads) / max(len(loads), 1)
    return max(loads) / mean if mean > 0 else 1.0


def _reduce(values, op, device):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return tuple(float(v) for v in values)
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return tuple(float(x) for x in t.cpu())


def max_over_ranks(values, device="cpu"):
    """Element-wise maximum over ranks (the slowest rank's times)."""
    import torch.distributed as dist
    return _reduce(values, dist.ReduceOp.MAX if dist.is_available() else None, device)


def sum_over_ranks(values, device="cpu"):
    """Element-wise sum over ranks (whole-job work)."""
    import torch.distributed as dist
    return _reduce(values, dist.ReduceOp.SUM if dist.is_available() else None, device)


def gather_members(local: dict, nmembers: int) -> list:
    """Collect {member index: result} from every rank into one list indexed by
    member (on every rank).  Missing or duplicated members are an error."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, local)
    else:
        parts = [local]
    out = [None] * nmembers
    seen = set()
    for p in parts:
        for k, v in p.items():
            if k in seen or not 0 <= k < nmembers:
                raise RuntimeError(f"member {k} reported twice or out of range")
            seen.add(k)
            out[k] = v
    if len(seen) != nmembers:
        raise RuntimeError(f"{nmembers - len(seen)} members missing from the gather")
    return out
