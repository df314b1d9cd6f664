"""Replica bookkeeping across ranks (one process per GPU, no data exchange).

Independent AMR solves do not shard across GPUs: each rank runs its own hierarchies
and ranks meet only to combine timings. Whole-job throughput is the cell-updates of
all ranks over the slowest rank's device time, as the benchmark contract asks.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def assign(n_items: int, rank: int, world: int) -> List[int]:
    """Items (requests, replicas) run by `rank`: round-robin, so every rank gets work."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank %d of %d" % (rank, world))
    return list(range(rank, n_items, world))


def combine(ms: float, cells: float, dist=None, device: str = "cpu") -> Tuple[float, float]:
    """(max over ranks of ms, sum over ranks of cells); identity without a process group.

    `dist` is torch.distributed (gloo on CPU tensors, nccl on CUDA tensors)."""
    if dist is None:
        return ms, cells
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([cells], dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), float(c.item())


def percentiles(values: Sequence[float], qs=(50, 99)) -> List[float]:
    """Nearest-rank percentiles of a sample (empty sample: NaN)."""
    v = sorted(values)
    out = []
    for q in qs:
        if not v:
            out.append(float("nan"))
            continue
        k = max(0, min(len(v) - 1, int(-(-q * len(v) // 100)) - 1))
        out.append(v[k])
    return out
