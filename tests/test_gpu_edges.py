"""Edge cases of the class-5 path on the device against the CPU oracle (GPU):
an empty batch, units the reference drops, units outside the engine's range,
and units at the top of that range (B up to 40,000,000, B^6 ~ 2^151.5)."""
import numpy as np
import pytest

import orc
import s615
import workloads as W

pytestmark = pytest.mark.gpu

N1 = 715
B_TOP = 40_000_000          # the engine's largest class-5 B (host_math.cpp kMaxB)


def sorted_hits(h):
    a = np.stack([h["unit"].astype(np.uint64), h["d"].astype(np.uint64), h["e"].astype(np.uint64),
                  h["fp"]], axis=1)
    if a.size == 0:
        return a.reshape(0, 4)
    return a[np.lexsort(a.T[::-1])]


@pytest.fixture(scope="module")
def table(engine, oracle_table):
    t, path = oracle_table(N1, 16)
    tid = engine.load_table(path, N1)
    yield t, tid
    engine.free_table(tid)


def test_empty_batch(engine, table):
    _, tid = table
    arr, _ = W.unit_array([], [], N1)
    hits, ctr = engine.cls5_run(tid, arr, 0)
    assert len(hits) == 0 and (ctr.calls, ctr.gated, ctr.probes, ctr.pos) == (0, 0, 0, 0)
    hits, ctr = engine.run(tid, arr, 0)
    assert len(hits) == 0 and (ctr.calls, ctr.probes) == (0, 0)


def test_units_the_reference_drops(engine, table):
    # u >= B makes base <= 0: pack_unit5 drops the unit (fourcore_cls5_gpu_v4.cu:
    # 169-184), so a batch of such units searches nothing
    t, tid = table
    units = [(1003, 1008), (29999, 30000), (29999, 30006)]
    arr, n = W.unit_array(units, [], N1)
    hits, ctr = engine.cls5_run(tid, arr, n)
    assert len(hits) == 0 and (ctr.calls, ctr.probes) == (0, 0)
    assert all(orc.pack_unit(B, u) is None for B, u in units)


def test_units_outside_the_range_are_refused(engine, table):
    _, tid = table
    for units in ([(B_TOP + 1, 6)], [(1, 6)]):
        arr, n = W.unit_array(units, [], N1)
        with pytest.raises(s615.S615Error) as ei:
            engine.cls5_run(tid, arr, n)
        assert ei.value.status == -3          # S615_E_FORMAT


def top_units(k, seed):
    """k truncated Stage-1 units of B in (B_TOP - 2000, B_TOP]: the unit's own base
    B^6 - u^6 and one of its own e / d residues, with the grid cut at a random e and
    d of that residue (an oracle-sized grid over the largest terms the engine takes)."""
    rng = np.random.RandomState(seed)
    out = []
    B = B_TOP + 1
    while len(out) < k:
        B -= 2
        if not W.eligible(B):
            continue
        us = s615.unit_candidates(B, 5)
        if not us:
            continue
        u = int(us[rng.randint(len(us))])
        U = orc.pack_unit(B, u)
        if U is None:
            continue
        er, dr = int(U.res[0]), int(U.res[U.nres1])
        fe, fd = (B - 1) // 14, (B - 1) // 21
        # the top rows (largest e) and a band of the first columns, or the reverse
        e = fe - (fe - er) % 729 - 729 * int(rng.randint(0, 40))
        d = dr + 64 * int(rng.randint(200, 2000))
        if len(out) % 2:
            e, d = er + 729 * int(rng.randint(100, 400)), fd - (fd - dr) % 64
        out.append((B, u, e, d))
    return out


def test_top_of_range_parity(engine, table):
    t, tid = table
    units = top_units(6, 11)
    arr = (s615.Unit * len(units))()
    ous = []
    for i, (B, u, e, d) in enumerate(units):
        base = B**6 - u**6
        arr[i] = s615.make_plant(base, e, d, lim=N1, u=u, B=B)
        ous.append(orc.plant_unit(base, e, d, lim=N1, B=B, u=u))
    hits, ctr = engine.cls5_run(tid, arr, len(units))
    ohits, (calls, gated, probes) = orc.cls5_run(t, orc.units_array(ous), len(ous))
    assert calls > 0 and probes > 0
    assert (ctr.calls, ctr.gated, ctr.probes) == (calls, gated, probes)
    np.testing.assert_array_equal(sorted_hits(hits), sorted_hits(ohits))


def test_top_of_range_plants(engine, table):
    # planted targets at the largest B, base = (14e)^6 + (21d)^6 + 42^6 (c1^6 + c2^6):
    # one axis near its largest value, the other short (oracle-sized grids); every
    # plant is among the raw hits
    t, tid = table
    plants = W.plants(6, 3, B_TOP - 5000, B_TOP, N1)
    rng = np.random.RandomState(4)
    for j, p in enumerate(plants):
        fe, fd = (p.B - 1) // 14, (p.B - 1) // 21
        if j % 2:
            p.e, p.d = fe - int(rng.randint(0, 5000)), 1 + int(rng.randint(0, 64 * 300))
        else:
            p.e, p.d = 1 + int(rng.randint(0, 729 * 60)), fd - int(rng.randint(0, 5000))
    arr, n = W.unit_array([], plants, N1)
    hits, ctr = engine.cls5_run(tid, arr, n)
    ous = [orc.plant_unit(p.base, p.e, p.d, lim=N1, B=p.B, u=p.u) for p in plants]
    ohits, (calls, gated, probes) = orc.cls5_run(t, orc.units_array(ous), len(ous))
    assert (ctr.calls, ctr.gated, ctr.probes) == (calls, gated, probes)
    np.testing.assert_array_equal(sorted_hits(hits), sorted_hits(ohits))
    for j, p in enumerate(plants):
        sel = (hits["unit"] == j) & (hits["d"] == p.d) & (hits["e"] == p.e)
        assert (hits["fp"][sel] == p.fp).any(), p
