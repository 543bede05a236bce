"""Multi-GPU by replicas: independent transforms are dealt to ranks (one process per GPU), and
no collective touches the data path. Only the timing uses a collective (max over ranks).

The work of one transform at bandwidth B is dominated by the discrete Wigner transform,
~8 B^2 (4B^2-1)/3 FP64 flops, plus 5 passes of 16 (2B)^3 bytes over HBM; ``transform_cost``
weighs both with measured B200 peaks so that ranks receive equal device time.
"""
from __future__ import annotations

import heapq

HBM_BYTES_PER_S = 6551.7e9      # measured copy bandwidth
FP64_FLOPS_PER_S = 37.0e12      # measured FP64 MMA peak


def transform_cost(B: int) -> float:
    """Roofline seconds of one DSOFT (or iDSOFT) at bandwidth B."""
    N = 2 * B
    flops = 8.0 * B * B * (4 * B * B - 1) / 3
    bytes_ = 5 * 16.0 * N ** 3
    return flops / FP64_FLOPS_PER_S + bytes_ / HBM_BYTES_PER_S


def shard(bandwidths: list[int], world: int) -> list[list[int]]:
    """Indices of the transforms each rank runs: longest-processing-time-first assignment of the
    costs to `world` ranks. Deterministic, so every rank computes the same plan."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(bandwidths)), key=lambda i: (-transform_cost(bandwidths[i]), i))
    heap = [(0.0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + transform_cost(bandwidths[i]), r))
    for lst in out:
        lst.sort()
    return out


def imbalance(bandwidths: list[int], plan: list[list[int]]) -> float:
    """max rank load / mean rank load (1.0 = perfect)."""
    loads = [sum(transform_cost(bandwidths[i]) for i in lst) for lst in plan]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank timing over the default process group (identity without one)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
