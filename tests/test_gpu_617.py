"""(6,1,7) Branch-A search (classes 1-5) on the device against the CPU oracle (GPU).

The oracle restates gen_class_cands(cls=5), k_find4_cls5 and verify_hit of
solve_617_v1.cu (:885-906, :563-657, :1040-1110); the device path is the
cls 7 unit of s615_run / s615_verify.  Hits, counters and verified lines must
be equal.
"""
import numpy as np
import pytest

import orc
import s615

pytestmark = pytest.mark.gpu

M42 = 42**6


def eligible617(B):
    """Branch-A B values of the campaign loop (solve_617_v1.cu:1910-1913)."""
    return B >= 11 and B % 2 == 1 and B % 3 != 0 and B % 7 != 0


def band(lo, hi):
    """Oracle candidates of every eligible B in [lo, hi] and the same
    candidates as engine units, index for index."""
    parts = [orc.cands617(B) for B in range(lo, hi + 1) if eligible617(B)]
    cands, n = orc.concat617([p for p in parts if p[1]])
    units, nu = s615.make_units617((cands[i].B, cands[i].u, cands[i].w) for i in range(n))
    assert nu == n
    return cands, units, n


def mine(hits):
    return sorted((int(h["unit"]), int(h["d"]), int(h["e"]), int(h["c4"]), int(h["fp"])) for h in hits)


def theirs(hits):
    return sorted((int(h["cand"]), int(h["e"]), int(h["c"]), int(h["d"]), int(h["fp"])) for h in hits)


def check_counters(ctr, oc, tri=True):
    calls, gated, _, tri_total, tri_skipped = oc
    assert (ctr.probes, ctr.gated, ctr.pos, ctr.calls) == (calls, gated, calls + gated, calls + gated)
    assert (ctr.tri_total, ctr.tri_skipped) == ((tri_total, tri_skipped) if tri else (0, 0))


@pytest.fixture(scope="module")
def band54(engine, oracle_table):
    cands, units, n = band(54301, 54400)
    return cands, units, n, 54400 // 42


@pytest.mark.parametrize("r", [16, 48])
def test_band_parity(engine, oracle_table, band54, r):
    cands, units, n, N = band54
    t, path = oracle_table(N, r)
    tid = engine.load_table(path, N)
    try:
        hits, ctr = engine.run(tid, units, n)
        oh, oc = orc.run617(t, cands, n)
        check_counters(ctr, oc)
        assert ctr.hits == len(oh)
        assert mine(hits) == theirs(oh)
        lines = sorted(s615.solution_line(s) for s in engine.verify(units, n, hits, N))
        assert lines == sorted(orc.verify617(cands, oh, N))
        if r == 48:
            assert any("B=54347 a1=2100 a2=3150 a3=19467 a4=32748 a5=33376 a6=46032 a7=48846"
                       in l for l in lines)
    finally:
        engine.free_table(tid)


@pytest.mark.parametrize("flags", [s615.F_NO_GATE, s615.F_NO_TRI, s615.F_PLAIN])
def test_flags(engine, oracle_table, flags):
    cands, units, n = band(54301, 54340)
    N = 54340 // 42
    t, path = oracle_table(N, 20)
    tid = engine.load_table(path, N)
    try:
        hits, ctr = engine.run(tid, units, n, flags)
        oh, oc = orc.run617(t, cands, n, use_gate=not (flags & s615.F_NO_GATE),
                            use_tri=not (flags & s615.F_NO_TRI))
        check_counters(ctr, oc, tri=not (flags & s615.F_NO_TRI))
        assert mine(hits) == theirs(oh)
    finally:
        engine.free_table(tid)


def test_known_identities(engine, golden):
    # every known identity of this shape with B < 200,000, from its own anchor
    known = golden["known617_cls5"]
    assert len(known) >= 12
    N = max(k["B"] for k in known) // 42
    tid = engine.build_table(N, 48)
    try:
        trip = [(k["B"], k["u"], k["w"]) for k in known]
        units, n = s615.make_units617(trip)
        hits, ctr = engine.run(tid, units, n)
        lines = [s615.solution_line(s) for s in engine.verify(units, n, hits, N)]
        for k in known:
            want = (f"SOLUTION cls=5 B={k['B']} " +
                    " ".join(f"a{i + 1}={x}" for i, x in enumerate(k["terms"])))
            assert len([l for l in lines if l.startswith(want)]) == 1, k["B"]
    finally:
        engine.free_table(tid)


def plant(c, d, N):
    """The plant shape of solve_617_v1.cu:1564-1582: (oracle cand, unit)."""
    base = (21 * d) ** 6 + M42 * sum(x**6 for x in c)
    C = orc.OrcCand617()
    C.base[0], C.base[1] = base % 2**64, base >> 64
    C.B, C.u, C.w, C.lim = 42 * N + 1, 14, 6, N
    C.mod1, C.fmax1, C.nres1 = 64, d, 1
    C.res[0] = d % 64
    return C, s615.make_plant617(base, d, N, B=42 * N + 1)


def window_reaches(c, N):
    s = sorted(c)
    T = sum(x**6 for x in s)
    return 3 * s[3] ** 6 >= T and 3 * s[2] ** 6 >= T - s[3] ** 6 and s[3] <= N


@pytest.mark.parametrize("N,r", [(600, 48), (13000, 16)])
def test_plants(engine, N, r):
    # N = 13,000: c4 windows wider than 2048 (the reference's tile width)
    rng = np.random.RandomState(N)
    plants = []
    while len(plants) < 48:
        c = sorted(int(x) for x in rng.choice(np.arange(1, N + 1), 4, replace=False))
        plants.append((c, int(rng.randint(1, 281))))
    plants.append(([N - 3, N - 2, N - 1, N], 5))
    cands = (orc.OrcCand617 * len(plants))()
    units = (s615.Unit * len(plants))()
    for i, (c, d) in enumerate(plants):
        cands[i], units[i] = plant(c, d, N)
    tid = engine.build_table(N, r)
    try:
        hdr, packed = engine.export_table(tid)
        t = orc.Table.from_memory(hdr, packed)
        hits, ctr = engine.run(tid, units, len(plants))
        oh, oc = orc.run617(t, cands, len(plants))
        check_counters(ctr, oc)
        assert mine(hits) == theirs(oh)
        got = set()
        for s in engine.verify(units, len(plants), hits, N):
            assert s.kind == 1
            got.add((s.unit, tuple(sorted((s.c1, s.c2, s.c3, s.c4)))))
        for i, (c, d) in enumerate(plants):
            assert ((i, tuple(c)) in got) == window_reaches(c, N), (i, c, d)
        assert sum(window_reaches(c, N) for c, _ in plants) >= 30
    finally:
        engine.free_table(tid)


def test_mixed_batch_with_cls5(engine, oracle_table):
    # cls5 (6,1,5) units and cls 7 units in one call == separate calls
    import workloads as W
    cands, u7, n7 = band(54301, 54340)
    cls5 = W.cls5_units(54301, 54400)
    N = 54400 // 42
    _, path = oracle_table(N, 20)
    tid = engine.load_table(path, N)
    try:
        mixed = (s615.Unit * (len(cls5) + n7))()
        for i, (B, u) in enumerate(cls5):
            mixed[i].cls, mixed[i].B, mixed[i].u = 5, B, u
        for j in range(n7):
            mixed[len(cls5) + j] = u7[j]
        hm, cm = engine.run(tid, mixed, len(cls5) + n7)
        u5, n5 = s615.make_units(cls5)
        h5, c5 = engine.run(tid, u5, n5)
        h7, c7 = engine.run(tid, u7, n7)
        for f in ("calls", "gated", "probes", "pos", "hits", "tri_total", "tri_skipped"):
            assert getattr(cm, f) == getattr(c5, f) + getattr(c7, f), f
        h7 = h7.copy()
        h7["unit"] += len(cls5)
        assert mine(hm) == sorted(mine(h5) + mine(h7))
    finally:
        engine.free_table(tid)


def test_bad_units_rejected(engine, oracle_table):
    _, path = oracle_table(300, 16)
    tid = engine.load_table(path, 300)
    try:
        for B, u, w in [(54347, 33377, 32748),      # u not 14u'
                        (54347, 33376, 32749),      # w not 6v'
                        (54347, 14 * 5, 32748),     # u^6 != B^6 (mod 3^6)
                        (2353975, 33376, 32748)]:   # B^6 >= 2^127
            units, n = s615.make_units617([(B, u, w)])
            with pytest.raises(s615.S615Error) as e:
                engine.run(tid, units, n)
            assert e.value.status == -3
    finally:
        engine.free_table(tid)


@pytest.mark.parametrize("lo,hi,r", [(34701, 34800, 48), (38101, 38200, 16), (39701, 39800, 20),
                                      (24301, 24400, 48), (28101, 28200, 16)])
def test_classes_1_to_4_parity(engine, oracle_table, lo, hi, r):
    """(6,1,7) classes 1-4: the native find4 jobs equal the oracle's, and the
    device run over them gives the oracle's hits, counters and lines."""
    N = hi // 42
    t, path = oracle_table(N, r)
    tid = engine.load_table(path, N)
    try:
        for cls in (1, 2, 3, 4):
            parts = [orc.jobs617(B, cls) for B in range(lo, hi + 1) if eligible617(B)]
            oj, n = orc.concat_jobs617([p for p in parts if p[1]])
            units = []
            for B in range(lo, hi + 1):
                if eligible617(B):
                    a, k = s615.jobs617(B, cls)
                    units += [a[i] for i in range(k)]
            assert len(units) == n
            if not n:
                continue
            arr = (s615.Unit * n)(*units)
            hits, ctr = engine.run(tid, arr, n)
            oh, oc = orc.run617_find4(t, oj, n)
            check_counters(ctr, oc)
            assert sorted((int(h["unit"]), int(h["e"]), int(h["c4"]), int(h["fp"])) for h in hits) == \
                sorted((int(h["job"]), int(h["c3"]), int(h["c4"]), int(h["fp"])) for h in oh)
            lines = sorted(s615.solution_line(s) for s in engine.verify(arr, n, hits, N))
            assert lines == sorted(orc.verify617_find4(oj, oh, N))
    finally:
        engine.free_table(tid)
