"""Replica aggregation for N > 1 processes (one per GPU).

The path does not shard for a single GPU's workload: a GA generation (or an
independent search replicate, like GARLI's MPI job farm) runs whole on each
GPU, with no data-path collective.  The only cross-rank steps are the barrier
around the timed region and these reductions: the job's time is the slowest
rank's, its work the sum over ranks.
"""
from __future__ import annotations

import torch


def aggregate(dist, ms: float, work: list[float]) -> tuple[float, list[float]]:
    """(max over ranks of ms, per-item sums over ranks of work); identity without a process group."""
    if dist is None:
        return float(ms), [float(x) for x in work]
    t = torch.tensor([ms], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    u = torch.tensor(list(work), dtype=torch.float64)
    dist.all_reduce(u)
    return float(t.item()), [float(x) for x in u]
