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


F234 = {2: 14, 3: 21, 4: 7}
MOD234 = {2: 729, 3: 64, 4: 46656}


def iroot6(n):
    if n <= 0:
        return 0
    x = int(round(n ** (1 / 6)))
    while x**6 > n:
        x -= 1
    while (x + 1) ** 6 <= n:
        x += 1
    return x


def find3_window(T, lim):
    """make_cand mode 3 (fourcore_find_v4.cu:411-416): hi = min(iroot6 T, lim),
    lo the least c with 3 c^6 >= T."""
    hi = min(iroot6(T), lim)
    lo = iroot6(-(-T // 3) - 1) + 1
    return (lo, hi) if lo <= hi else (1, 0)


def test_top_of_range_cls234_plants(engine, table):
    # class 2-4 planted targets with f d near B = 40,000,000 (base ~ 2^151.6,
    # T up to 2^119): the oracle's find3 rows over the plant's residue class
    t, tid = table
    rng = np.random.RandomState(21)
    plants = []
    for i, cls in enumerate([2, 3, 4] * 2):
        B = B_TOP - 1 - 2 * i
        f = F234[cls]
        d = (B - 1) // f - int(rng.randint(0, 3 * MOD234[cls]))
        c = sorted(int(x) for x in rng.choice(np.arange(1, N1 + 1), 3, replace=False))
        plants.append(dict(cls=cls, B=B, d=d, c=c, base=(f * d) ** 6 + 42**6 * sum(x**6 for x in c)))
    arr = (s615.Unit * len(plants))()
    jobs, origin = [], []
    for j, p in enumerate(plants):
        arr[j] = s615.make_plant234(p["cls"], p["base"], p["d"], lim=N1, B=p["B"])
        f, mod = F234[p["cls"]], MOD234[p["cls"]]
        d = p["d"] % mod or mod
        while d <= p["d"]:
            R = p["base"] - (f * d) ** 6
            if R > 0:
                assert R % 42**6 == 0
                T = R // 42**6
                lo, hi = find3_window(T, N1)
                if lo <= hi:
                    J = orc.OrcJob3()
                    J.cls, J.lim, J.B, J.u, J.d = p["cls"], N1, p["B"], 0, d
                    J.T[0], J.T[1] = T % 2**64, T >> 64
                    J.lo, J.hi = lo, hi
                    jobs.append(J)
                    origin.append((j, d))
            d += mod
    assert jobs
    hits, ctr = engine.run(tid, arr, len(plants))
    jarr = (orc.OrcJob3 * len(jobs))(*jobs)
    hits3 = (orc.OrcHit3 * (1 << 16))()
    c3 = np.zeros(3, dtype=np.uint64)
    nh = orc.lib().orc_find3_run(t.h, orc.C.cast(jarr, orc.C.c_void_p), len(jobs), 1, 0,
                                 orc.C.cast(hits3, orc.C.c_void_p), 1 << 16, orc._ptr(c3))
    assert (ctr.calls, ctr.gated, ctr.probes) == tuple(int(x) for x in c3)
    mine = sorted((int(h["unit"]), int(h["d"]), int(h["e"]), int(h["fp"])) for h in hits)
    theirs = sorted((origin[hits3[k].job][0], origin[hits3[k].job][1], hits3[k].c3, hits3[k].fp)
                    for k in range(nh))
    assert mine == theirs
    lines = {s615.solution_line(s) for s in engine.verify(arr, len(plants), hits, N1)}
    for j, p in enumerate(plants):
        c1, c2, c3v = p["c"]
        assert f"PLANT cls={p['cls']} unit={j} d={p['d']} c1={c1} c2={c2} c3={c3v}" in lines


def test_top_of_range_jobs(engine, table):
    # reduced-T jobs of class 2-4 Stage-1 units at B ~ 40,000,000: T up to 2^119 and
    # c3 windows up to ~150k wide (lim = (B-1)/42 = 952,380); a spread of each unit's
    # jobs against the oracle's expand_unit + make_cand + k_find3 restatement
    t, tid = table
    picked, opicked = [], []
    for cls in (2, 3, 4):
        B = B_TOP + 1
        while True:
            B -= 2
            if W.eligible(B) and s615.unit_candidates(B, cls):
                break
        u = s615.unit_candidates(B, cls)[0]
        arr, n, fail = s615.expand_unit(B, u, cls)
        oarr, on, ofail = orc.expand_unit(B, u, cls)
        assert (n, fail) == (on, ofail) and n > 0
        for i in range(0, n, max(1, n // 60)):
            assert (arr[i].base[0], arr[i].base[1]) == (oarr[i].T[0], oarr[i].T[1])
            picked.append(arr[i])
            opicked.append(oarr[i])
    jarr = (s615.Unit * len(picked))(*picked)
    oj = (orc.OrcJob * len(opicked))(*opicked)
    hits, ctr = engine.run(tid, jarr, len(picked))
    oh, (calls, gated, probes) = orc.run_jobs(t, oj, len(opicked))
    assert calls > 10**7 and len(oh) > 0          # r = 16: filter false positives
    assert (ctr.calls, ctr.gated, ctr.probes) == (calls, gated, probes)
    mine = sorted((int(h["unit"]), int(h["e"]), int(h["c4"]), int(h["fp"])) for h in hits)
    theirs = sorted((int(h["job"]), int(h["c3"]), int(h["c4"]), int(h["fp"])) for h in oh)
    assert mine == theirs


def test_top_of_range_617_plants(engine):
    # (6,1,7) Branch-A class-5 plants just below the i128 wall (21 d up to
    # B_HARD_MAX = 2,353,973, base up to 2^127): the c4 windows of the large-T
    # rows, and the planted row, against the oracle's k_find4_cls5 restatement
    import test_gpu_617 as T7
    N, r = 600, 16
    rng = np.random.RandomState(17)
    plants = []
    for k in range(12):
        c = sorted(int(x) for x in rng.choice(np.arange(1, N + 1), 4, replace=False))
        d = 2_353_973 // 21 - int(rng.randint(0, 2000))
        plants.append((c, d))
    cands = (orc.OrcCand617 * len(plants))()
    units = (s615.Unit * len(plants))()
    for i, (c, d) in enumerate(plants):
        cands[i], units[i] = T7.plant(c, d, N)
        assert (21 * d) ** 6 < 2**127 and (21 * d) ** 6 > 2**126
    tid = engine.build_table(N, r)
    try:
        hdr, packed = engine.export_table(tid)
        t = orc.Table.from_memory(hdr, packed)
        hits, ctr = engine.run(tid, units, len(plants))
        oh, oc = orc.run617(t, cands, len(plants))
        T7.check_counters(ctr, oc)
        assert T7.mine(hits) == T7.theirs(oh)
        got = {(s.unit, tuple(sorted((s.c1, s.c2, s.c3, s.c4))))
               for s in engine.verify(units, len(plants), hits, N) if s.kind == 1}
        for i, (c, d) in enumerate(plants):
            assert ((i, tuple(c)) in got) == T7.window_reaches(c, N), (i, c, d)
    finally:
        engine.free_table(tid)
