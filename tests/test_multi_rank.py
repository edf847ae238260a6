"""Replicas over two ranks (CPU, gloo): the band split and the merge.

Each rank takes its own B band (shard.rank_band), derives its units with the
engine's host rule, counts its grid points with the oracle, and the ranks
merge with shard.merge (MAX of times, SUM of counters).  The merged counts
must equal one process doing the union band; bands must not overlap or leave
gaps; every rank uses the same table N.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


LO, WIDTH = 20000, 300


def counts_for(lo, hi):
    """Stage-1 class-5 units of B in [lo, hi) and their oracle counters."""
    import orc
    import workloads as W
    units = W.cls5_units(lo, hi - 1)
    arr = orc.units_array([orc.pack_unit(B, u) for B, u in units])
    t = orc.Table.build_pairs(300, 16)
    _, (calls, gated, probes) = orc.cls5_run(t, arr, len(units), threads=2)
    return {"units": len(units), "calls": calls, "gated": gated, "probes": probes}


def worker(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "six-one-five_b200"), os.path.join(root, "oracle")]
    import datetime

    import torch.distributed as dist

    import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        lo, hi = shard.rank_band(LO, WIDTH, rank)
        c = counts_for(lo, hi)
        t, tot = shard.merge(dist, "cpu", 10.0 + rank, c)
        N = shard.table_N(LO, WIDTH, world)
        out.put((rank, lo, hi, t, tot, N))
    except Exception as e:       # report instead of leaving the parent waiting
        out.put((rank, "error", repr(e), 0, {}, 0))
        raise
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_ranks_merge_equals_one_process():
    import shard
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(world)]
    assert not [r for r in res if r[1] == "error"], res
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    # bands tile [LO, LO + world*WIDTH) with no overlap and no gap
    assert [r[1:3] for r in res] == [(LO, LO + WIDTH), (LO + WIDTH, LO + 2 * WIDTH)]
    # every rank sees the slowest rank's time and the same sums and N
    assert all(r[3] == 11.0 for r in res)
    assert res[0][4] == res[1][4]
    assert {r[5] for r in res} == {shard.table_N(LO, WIDTH, world)}
    assert res[0][4] == counts_for(LO, LO + world * WIDTH)
    # without a process group merge is the identity
    assert shard.merge(None, "cpu", 3.0, {"a": 1}) == (3.0, {"a": 1})


# ---- shard split: every rank runs the same units on its own range of shards ----
S_SPLIT, N_SPLIT = 4, 700


def split_worker(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "six-one-five_b200"), os.path.join(root, "oracle")]
    import datetime

    import torch.distributed as dist

    import orc
    import shard
    import workloads as W
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        lo, hi = shard.shard_range(rank, world, S_SPLIT)
        parts = [orc.Table.build_pairs_shard(N_SPLIT, 10, S_SPLIT, s) if lo <= s < hi else None
                 for s in range(S_SPLIT)]
        mine = orc.Table.shard_set(parts)
        units = W.cls5_units(29001, 29400)
        arr = orc.units_array([orc.pack_unit(B, u) for B, u in units])
        hits, (calls, gated, probes) = orc.cls5_run(mine, arr, len(units), threads=2)
        t, tot, allh = shard.merge_split(dist, "cpu", 5.0 + rank,
                                         {"calls": calls, "gated": gated, "probes": probes}, hits)
        out.put((rank, (lo, hi), t, tot,
                 sorted((int(h["unit"]), int(h["d"]), int(h["e"]), int(h["fp"])) for h in allh)))
    except Exception as e:
        out.put((rank, "error", repr(e), {}, []))
        raise
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_shard_split_union_equals_whole_set():
    import orc
    import workloads as W
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=split_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert all(r[1] != "error" for r in res), res
    assert [r[1] for r in res] == [(0, 2), (2, 4)]
    whole = orc.Table.shard_set([orc.Table.build_pairs_shard(N_SPLIT, 10, S_SPLIT, s)
                                 for s in range(S_SPLIT)])
    units = W.cls5_units(29001, 29400)
    arr = orc.units_array([orc.pack_unit(B, u) for B, u in units])
    hits, (calls, gated, probes) = orc.cls5_run(whole, arr, len(units), threads=2)
    want = sorted((int(h["unit"]), int(h["d"]), int(h["e"]), int(h["fp"])) for h in hits)
    assert want, "r = 10 leaves raw hits to split"
    for rank, rng, t, tot, allh in res:
        assert t == 6.0
        assert tot == {"calls": calls, "gated": gated, "probes": probes}
        assert allh == want
