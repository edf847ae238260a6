"""Multi-GPU: how ranks split the work and how their results merge.

Replicas (the default): units are independent and the xor table is
read-only, so each rank (one process per GPU) takes its own contiguous B band,
holds its own copy of the table and runs with no collective on the data path.
Only the host-side merge talks between ranks: the slowest rank's device time
(MAX) and the sums of the counters.

Shard split (a table too large for one GPU): each rank holds a contiguous
range of the pair-space shards and runs the SAME units; a probe whose key
belongs to another rank's shard finds nothing here.  Each rank repeats the
peel and the gate (its counters are the whole search's) and probes only its
own keys, so no key crosses NVLink: the union of the ranks' raw hits is the
whole set's.  The merge takes the slowest time, checks that the counters
agree, and gathers the hits.
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


def shard_range(rank: int, world: int, shards: int) -> Tuple[int, int]:
    """Rank `rank`'s contiguous shards [lo, hi) of `shards` (world <= shards)."""
    return shards * rank // world, shards * (rank + 1) // world


def merge_split(dist, device, time_ms: float, counts: Dict[str, int], hits):
    """Shard-split merge: MAX time, the (equal) counters of every rank, and
    the union of the ranks' hits (a numpy structured array) on every rank."""
    if dist is None:
        return time_ms, dict(counts), hits
    import numpy as np
    import torch
    t = torch.tensor([time_ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    keys = sorted(counts)
    c = torch.tensor([int(counts[k]) for k in keys], dtype=torch.int64, device=device)
    lo, hi = c.clone(), c.clone()
    dist.all_reduce(lo, op=dist.ReduceOp.MIN)
    dist.all_reduce(hi, op=dist.ReduceOp.MAX)
    if not torch.equal(lo, hi):
        raise RuntimeError("shard-split ranks disagree on the counters of the same units")
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, hits)
    return float(t.item()), {k: int(v) for k, v in zip(keys, c.tolist())}, np.concatenate(parts)
