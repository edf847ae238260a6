"""Class 1 (find4, fourcore_find_v4.cu:287-338) on the device against the CPU
oracle (GPU): raw hits, counters, plants, and the mixed queue."""
import numpy as np
import pytest

import orc
import s615
import workloads as W

pytestmark = pytest.mark.gpu

LO, HI = 1000, 200000
N = HI // 42


@pytest.fixture(scope="module")
def cls1_units():
    out = []
    for B in range(LO, HI + 1):
        if W.eligible(B):
            out += [(B, u) for u in s615.unit_candidates(B, 1)]
    assert len(out) > 100
    return out


def unit_arr(units):
    arr = (s615.Unit * len(units))()
    for i, (B, u) in enumerate(units):
        arr[i].cls, arr[i].B, arr[i].u = 1, B, u
    return arr


@pytest.mark.parametrize("r", [16, 48])
def test_cls1_parity(engine, oracle_table, cls1_units, r):
    t, path = oracle_table(N, r)
    tid = engine.load_table(path, N)
    try:
        arr = unit_arr(cls1_units)
        hits, ctr = engine.run(tid, arr, len(cls1_units))
        jobs, nj, origin = orc.jobs_cls1(cls1_units)
        oh, (calls, gated, probes) = orc.run_find4(t, jobs, nj)
        assert (ctr.calls, ctr.gated, ctr.probes, ctr.pos) == (calls, gated, probes, calls)
        mine = sorted((int(h["unit"]), int(h["e"]), int(h["c4"]), int(h["fp"])) for h in hits)
        theirs = sorted((origin[int(h["job"])], int(h["c3"]), int(h["c4"]), int(h["fp"])) for h in oh)
        assert mine == theirs
        assert all(int(h["d"]) == 0 for h in hits)
        assert not [s for s in engine.verify(arr, len(cls1_units), hits, N) if s.kind == 0]
    finally:
        engine.free_table(tid)


def test_cls1_plants_and_mixed_queue(engine, oracle_table, cls1_units):
    _, path = oracle_table(N, 20)
    tid = engine.load_table(path, N)
    try:
        rng = np.random.RandomState(4)
        plants = []
        while len(plants) < 24:
            c = sorted(int(x) for x in rng.choice(np.arange(1, N + 1), 4, replace=False))
            plants.append(c)
        units = list(cls1_units[:40])
        arr = (s615.Unit * (len(units) + len(plants)))()
        for i, (B, u) in enumerate(units):
            arr[i].cls, arr[i].B, arr[i].u = 1, B, u
        for j, c in enumerate(plants):
            arr[len(units) + j] = s615.make_plant1(c, N, B=42 * N + 1)
        n = len(units) + len(plants)
        hits, ctr = engine.run(tid, arr, n)
        got = {(s.unit, tuple(sorted((s.c1, s.c2, s.c3, s.c4))))
               for s in engine.verify(arr, n, hits, N) if s.kind == 1}
        for j, c in enumerate(plants):
            assert (len(units) + j, tuple(c)) in got, c
        # one queue with class-5 and (6,1,7) units == the classes run alone
        u5 = W.cls5_units(54301, 54400)
        a5, n5 = W.unit_array(u5, [], N)
        c7 = s615.candidates617(54347)
        mixed = (s615.Unit * (n + n5 + c7[1]))()
        for i in range(n):
            mixed[i] = arr[i]
        for i in range(n5):
            mixed[n + i] = a5[i]
        for i in range(c7[1]):
            mixed[n + n5 + i] = c7[0][i]
        hm, cm = engine.run(tid, mixed, n + n5 + c7[1])
        parts = [(0, engine.run(tid, arr, n)), (n, engine.run(tid, a5, n5)),
                 (n + n5, engine.run(tid, c7[0], c7[1]))]
        tot = {f: sum(getattr(p[1][1], f) for p in parts) for f in ("calls", "gated", "probes", "pos")}
        assert {f: getattr(cm, f) for f in tot} == tot
        key = lambda h, off: [(int(x["unit"]) + off, int(x["d"]), int(x["e"]), int(x["c4"]), int(x["fp"]))
                              for x in h]
        assert sorted(key(hm, 0)) == sorted(sum((key(p[1][0], p[0]) for p in parts), []))
    finally:
        engine.free_table(tid)
