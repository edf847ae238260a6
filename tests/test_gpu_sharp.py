"""The sharper gate (S615_F_SHARP) on the device (GPU).

It adds sound residue tests (sums of two sixth powers mod 64, 27, 49, 31, 37,
43), so against the default run on the same units: the same in-range and R>0
point counts, fewer probes, raw hits a subset, and exactly the same verified
solutions and recovered plants, for every unit kind.
"""
import numpy as np
import pytest

import orc
import s615
import workloads as W

pytestmark = pytest.mark.gpu


def hit_set(h):
    return {(int(x["unit"]), int(x["d"]), int(x["e"]), int(x["c4"]), int(x["fp"])) for x in h}


def sol_set(sols):
    return {(s.unit, s.kind, s.cls, s.d, s.e, s.c1, s.c2, s.c3, s.c4, tuple(s.a)) for s in sols}


def both(engine, tid, arr, n, N, flags=0):
    h0, c0 = engine.run(tid, arr, n, flags)
    h1, c1 = engine.run(tid, arr, n, flags | s615.F_SHARP)
    return (h0, c0, sol_set(engine.verify(arr, n, h0, N))), (h1, c1, sol_set(engine.verify(arr, n, h1, N)))


@pytest.mark.parametrize("r", [16, 48])
def test_sharp_cls5_config1(engine, oracle_table, r):
    N = 715
    _, path = oracle_table(N, r)
    tid = engine.load_table(path, N)
    try:
        units = W.cls5_units(1000, 30000)
        plants = W.plants(16, 1, 1000, 30000, N)
        arr, n = W.unit_array(units, plants, N)
        (h0, c0, s0), (h1, c1, s1) = both(engine, tid, arr, n, N)
        assert (c1.calls, c1.pos) == (c0.calls, c0.pos)
        assert c1.probes < c0.probes and c1.gated == c1.pos - c1.probes
        assert hit_set(h1) <= hit_set(h0)
        assert s1 == s0 and len([s for s in s1 if s[1] == 1]) >= len(plants)
    finally:
        engine.free_table(tid)


def test_sharp_cls5_band_sample(engine):
    N = 76300
    tid = engine.build_table(N, 48)
    try:
        units = W.cls5_units(3200000, 3200400)
        plants = W.plants(32, 2, 3200000, 3200400, N)
        arr, n = W.unit_array(units, plants, N)
        (h0, c0, s0), (h1, c1, s1) = both(engine, tid, arr, n, N)
        assert c1.pos == c0.pos and c1.probes * 2 < c0.probes
        assert hit_set(h1) <= hit_set(h0)
        assert s1 == s0
        got = {(s[0], s[3], s[4], s[5], s[6]) for s in s1 if s[1] == 1}
        assert all((len(units) + j, p.d, p.e, p.c1, p.c2) in got for j, p in enumerate(plants))
    finally:
        engine.free_table(tid)


def test_sharp_617(engine, oracle_table):
    N = 54400 // 42
    _, path = oracle_table(N, 16)
    tid = engine.load_table(path, N)
    try:
        trip = []
        for B in range(54301, 54401):
            if B % 2 and B % 3 and B % 7:
                arr, k = s615.candidates617(B)
                trip += [(arr[i].B, arr[i].u, arr[i].w) for i in range(k)]
        arr, n = s615.make_units617(trip)
        (h0, c0, s0), (h1, c1, s1) = both(engine, tid, arr, n, N)
        assert (c1.tri_total, c1.tri_skipped, c1.pos) == (c0.tri_total, c0.tri_skipped, c0.pos)
        assert c1.probes < c0.probes
        assert hit_set(h1) <= hit_set(h0) and s1 == s0
        lines = [s615.solution_line(s) for s in engine.verify(arr, n, h1, N)]
        assert any("B=54347 a1=2100 a2=3150 a3=19467 a4=32748 a5=33376 a6=46032 a7=48846" in l
                   for l in lines)
    finally:
        engine.free_table(tid)


def test_sharp_617_plants(engine):
    N = 600
    tid = engine.build_table(N, 48)
    try:
        rng = np.random.RandomState(9)
        units, want = [], []
        while len(units) < 64:
            c = sorted(int(x) for x in rng.choice(np.arange(1, N + 1), 4, replace=False))
            T = sum(x**6 for x in c)
            if 3 * c[3] ** 6 < T or 3 * c[2] ** 6 < T - c[3] ** 6:
                continue
            d = int(rng.randint(1, 281))
            units.append(s615.make_plant617((21 * d) ** 6 + 42**6 * T, d, N, B=42 * N + 1))
            want.append((d, tuple(c)))
        arr = (s615.Unit * len(units))(*units)
        h1, _ = engine.run(tid, arr, len(units), s615.F_SHARP)
        got = {(s.unit, s.d, tuple(sorted((s.c1, s.c2, s.c3, s.c4))))
               for s in engine.verify(arr, len(units), h1, N)}
        assert all((i, d, c) in got for i, (d, c) in enumerate(want))
    finally:
        engine.free_table(tid)


def test_sharp_cls234_and_jobs(engine, oracle_table):
    """Find3 rows (classes 2-4, reduced-T jobs, find2 jobs) take the sharper
    gate too: fewer probes, raw hits a subset, the same verified results."""
    N = 2000
    _, path = oracle_table(N, 16)
    tid = engine.load_table(path, N)
    try:
        units = [(c, B, u) for B in range(400000, 400600) if W.eligible(B)
                 for c in (2, 3, 4) for u in s615.unit_candidates(B, c)]
        p24 = W.plants234(12, 8, 400000, 400600, N)
        arr0, n0 = W.mixed_unit_array(units, [], p24, N)
        rows = [arr0[i] for i in range(n0)]
        rng = np.random.RandomState(3)
        for k in range(30):   # planted jobs: find2, find3 and find4
            m = (2, 3, 4)[k % 3]
            c = sorted(int(x) for x in rng.choice(np.arange(1, N + 1), m, replace=False))
            cls = {2: 5, 3: 2 + (k // 3) % 3, 4: 1}[m]
            rows.append(s615.make_job(cls, 999999 - k, 1, sum(x**6 for x in c), 1, 1, lim=N))
        for c, B, u in [(4, 400003, s615.unit_candidates(400003, 4)[0]),
                        (5, *W.cls5_units(100001, 100100)[0])]:
            a, k, _ = s615.expand_unit(B, u, c)
            rows += [a[i] for i in range(min(k, 4000))]
        arr = (s615.Unit * len(rows))(*rows)
        (h0, c0, s0), (h1, c1, s1) = both(engine, tid, arr, len(rows), N)
        assert (c1.calls, c1.pos) == (c0.calls, c0.pos)
        assert c1.probes < c0.probes / 4
        assert hit_set(h1) <= hit_set(h0) and s1 == s0
        assert sum(1 for x in s0 if x[1] == 1) >= len(p24)                  # plants
        assert sum(1 for x in s0 if x[1] == s615.S615_KIND_JOB) >= 30        # planted jobs
    finally:
        engine.free_table(tid)


def test_sharp_find4_kinds(engine, oracle_table):
    """Class-1 find4 units and plants, and (6,1,7) classes 1-4 jobs with their
    known identities, through the sharp gate: same tri counts and points,
    fewer probes, raw hits a subset, the same verified lines."""
    N = 40000 // 42
    _, path = oracle_table(N, 16)
    tid = engine.load_table(path, N)
    try:
        rows = []
        for B in (24329, 28121, 32105, 33365):                 # class-1 units
            for u in s615.unit_candidates(B, 1):
                U = s615.Unit()
                U.cls, U.B, U.u = 1, B, u
                rows.append(U)
        rng = np.random.RandomState(12)
        for _ in range(16):                                    # class-1 plants
            c = sorted(int(x) for x in rng.choice(np.arange(1, N + 1), 4, replace=False))
            rows.append(s615.make_plant1(c, N, B=42 * N + 1))
        for B, cls in ((34781, 4), (38191, 4), (39779, 3), (34763, 2)):   # (6,1,7) jobs
            a, k = s615.jobs617(B, cls)
            rows += [a[i] for i in range(k)]
        arr = (s615.Unit * len(rows))(*rows)
        (h0, c0, s0), (h1, c1, s1) = both(engine, tid, arr, len(rows), N)
        assert (c1.tri_total, c1.tri_skipped, c1.pos) == (c0.tri_total, c0.tri_skipped, c0.pos)
        assert c1.probes < c0.probes
        assert hit_set(h1) <= hit_set(h0) and s1 == s0
        lines = [s615.solution_line(s) for s in engine.verify(arr, len(rows), h1, N)]
        for B in (34781, 38191, 39779):
            assert any(f"B={B} " in l and l.startswith("SOLUTION") for l in lines), B
        assert sum(l.startswith("PLANT cls=1") for l in lines) >= 16
    finally:
        engine.free_table(tid)
