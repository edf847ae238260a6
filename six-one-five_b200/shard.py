"""Multi-GPU replicas: how ranks split a B range and how their results merge.

The search has no exchange step: units are independent and the xor table is
read-only, so each rank (one process per GPU) takes its own contiguous B band,
holds its own copy of the table and runs with no collective on the data path.
Only the host-side merge below talks between ranks: the slowest rank's device
time (MAX) and the sums of the counters.
"""
from __future__ import annotations

import math
from typing import Dict, Tuple


def rank_band(lo: int, width: int, rank: int) -> Tuple[int, int]:
    """Rank `rank`'s half-open band [lo + rank*width, lo + (rank+1)*width)."""
    return lo + rank * width, lo + (rank + 1) * width


def table_N(lo: int, width: int, world: int) -> int:
    """One table serves every rank: N = ceil(B_max / 42) over the whole range
    (every 42-term c of a unit with B <= B_max satisfies c <= (B-1)/42)."""
    return math.ceil((lo + world * width) / 42)


def merge(dist, device, time_ms: float, counts: Dict[str, int]) -> Tuple[float, Dict[str, int]]:
    """MAX of the ranks' device times and SUM of their counters (any backend:
    nccl on GPUs, gloo on CPU).  Without a process group returns the inputs."""
    if dist is None:
        return time_ms, dict(counts)
    import torch
    t = torch.tensor([time_ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    keys = sorted(counts)
    c = torch.tensor([int(counts[k]) for k in keys], dtype=torch.int64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), {k: int(v) for k, v in zip(keys, c.tolist())}
