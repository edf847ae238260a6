"""cls2-4 find3 leaf on the device against the CPU oracle (GPU).

The oracle restates expand_unit + make_cand (mode 3) + k_find3
(fourcore_find_v4.cu:165-205,401-425,255-284) with 64-bit cell indices.
"""
import math

import numpy as np
import pytest

import orc
import s615
import workloads as W

pytestmark = pytest.mark.gpu

F = {2: 14, 3: 21, 4: 7}
MOD = {2: 729, 3: 64, 4: 46656}


def iroot6(n):
    if n <= 0:
        return 0
    x = int(round(n ** (1 / 6)))
    while x**6 > n:
        x -= 1
    while (x + 1) ** 6 <= n:
        x += 1
    return x


def window(T, lim):
    """make_cand mode 3 (fourcore_find_v4.cu:411-416)."""
    hi = min(iroot6(T), lim)
    lo = 1
    while lo <= hi and 3 * lo**6 < T:
        lo += 1
    return (1, 0) if lo > hi else (lo, hi)


def stage1(lo, hi, classes):
    out = []
    for B in range(lo, hi + 1):
        if not W.eligible(B):
            continue
        for c in classes:
            for u in s615.unit_candidates(B, c):
                out.append((c, B, u))
    return out


def plant234(rng, cls, B, N):
    """base = (f d)^6 + 42^6 (c1^6 + c2^6 + c3^6), c1 < c2 < c3 <= N."""
    d = int(rng.randint(1, (B - 1) // F[cls] + 1))
    c = sorted(int(x) for x in rng.choice(np.arange(1, N + 1), 3, replace=False))
    base = (F[cls] * d) ** 6 + 42**6 * sum(x**6 for x in c)
    return dict(cls=cls, B=B, d=d, c=c, base=base)


def oracle_jobs(units, plants, N):
    """Oracle find3 jobs for Stage-1 units (orc_expand_cls234) and plants
    (the same window rule over the plant's residue class), with the
    (unit index, d) each job came from."""
    jobs, origin = [], []
    buf = (orc.OrcJob3 * 100000)()
    for ui, (c, B, u) in enumerate(units):
        n = orc.lib().orc_expand_cls234(B, u, c, orc.C.cast(buf, orc.C.c_void_p), 100000)
        for k in range(n):
            if buf[k].lo <= buf[k].hi:
                jobs.append(orc.OrcJob3.from_buffer_copy(buf[k]))
                origin.append((ui, buf[k].d))
    for pj, p in enumerate(plants):
        ui = len(units) + pj
        f, mod = F[p["cls"]], MOD[p["cls"]]
        r0 = p["d"] % mod
        d = r0 if r0 else mod
        while d <= p["d"]:
            R = p["base"] - (f * d) ** 6
            if R > 0:
                assert R % 42**6 == 0
                T = R // 42**6
                lo, hi = window(T, N)
                if lo <= hi:
                    J = orc.OrcJob3()
                    J.cls, J.lim, J.B, J.u, J.d = p["cls"], N, p["B"], 0, d
                    J.T[0], J.T[1] = T % 2**64, T >> 64
                    J.lo, J.hi = lo, hi
                    jobs.append(J)
                    origin.append((ui, d))
            d += mod
    arr = (orc.OrcJob3 * max(len(jobs), 1))()
    for i, J in enumerate(jobs):
        arr[i] = J
    return arr, len(jobs), origin


def unit_array(units, plants, N):
    n = len(units) + len(plants)
    arr = (s615.Unit * max(n, 1))()
    for i, (c, B, u) in enumerate(units):
        arr[i].cls, arr[i].kind, arr[i].B, arr[i].u = c, 0, B, u
    for j, p in enumerate(plants):
        arr[len(units) + j] = s615.make_plant234(p["cls"], p["base"], p["d"], lim=N, B=p["B"])
    return arr, n


@pytest.fixture(scope="module")
def case():
    N = 2000
    units = stage1(400000, 401500, (2, 3, 4))
    assert {c for c, _, _ in units} == {2, 3, 4}
    rng = np.random.RandomState(11)
    plants = [plant234(rng, c, 400003 + 2 * i, N) for i, c in enumerate([2, 3, 4] * 4)]
    return N, units, plants


@pytest.mark.parametrize("r", [16, 20])
def test_cls234_parity_and_plants(engine, oracle_table, case, r):
    N, units, plants = case
    t, path = oracle_table(N, r)
    tid = engine.load_table(path, N)
    try:
        arr, n = unit_array(units, plants, N)
        hits, ctr = engine.run(tid, arr, n)
        jarr, nj, origin = oracle_jobs(units, plants, N)
        hits3 = (orc.OrcHit3 * (1 << 20))()
        c3 = np.zeros(3, dtype=np.uint64)
        nh = orc.lib().orc_find3_run(t.h, orc.C.cast(jarr, orc.C.c_void_p), nj, 1, 0,
                                     orc.C.cast(hits3, orc.C.c_void_p), 1 << 20, orc._ptr(c3))
        calls, gated, probes = (int(x) for x in c3)
        assert (ctr.calls, ctr.gated, ctr.probes) == (calls, gated, probes)
        assert ctr.pos == calls
        mine = sorted((int(h["unit"]), int(h["d"]), int(h["e"]), int(h["fp"])) for h in hits)
        theirs = sorted((origin[hits3[k].job][0], origin[hits3[k].job][1], hits3[k].c3, hits3[k].fp)
                        for k in range(nh))
        assert mine == theirs
        sols = engine.verify(arr, n, hits, N)
        lines = {s615.solution_line(s) for s in sols}
        for j, p in enumerate(plants):
            c1, c2, c3v = p["c"]
            assert (f"PLANT cls={p['cls']} unit={len(units) + j} d={p['d']} "
                    f"c1={c1} c2={c2} c3={c3v}") in lines
        assert not [l for l in lines if l.startswith("SOLUTION")]
    finally:
        engine.free_table(tid)


def test_mixed_batch_equals_per_class_runs(engine, oracle_table, case):
    # one persistent launch over a mixed queue == the classes run separately
    N, units, _ = case
    _, path = oracle_table(N, 16)
    tid = engine.load_table(path, N)
    try:
        cls5 = [(5, B, u) for B, u in W.cls5_units(400000, 401500)]
        mixed = units + cls5
        arr, n = unit_array(mixed, [], N)
        hits, ctr = engine.run(tid, arr, n)
        tot = [0, 0, 0]
        allh = []
        for c in (2, 3, 4, 5):
            idx = [i for i, x in enumerate(mixed) if x[0] == c]
            sub, sn = unit_array([mixed[i] for i in idx], [], N)
            h, cc = engine.run(tid, sub, sn)
            tot = [tot[0] + cc.calls, tot[1] + cc.gated, tot[2] + cc.probes]
            allh += [(idx[int(x["unit"])], int(x["d"]), int(x["e"]), int(x["fp"])) for x in h]
        assert [ctr.calls, ctr.gated, ctr.probes] == tot
        assert sorted((int(x["unit"]), int(x["d"]), int(x["e"]), int(x["fp"])) for x in hits) == sorted(allh)
    finally:
        engine.free_table(tid)
