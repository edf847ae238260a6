"""cls5 peel + gate + probe + verify on the device against the CPU oracle (GPU)."""
import math

import numpy as np
import pytest

import orc
import s615
import workloads as W

pytestmark = pytest.mark.gpu

N1 = 715   # ceil(30000 / 42): config 1's table


def sorted_hits(h):
    a = np.stack([h["unit"].astype(np.uint64), h["d"].astype(np.uint64), h["e"].astype(np.uint64),
                  h["fp"]], axis=1)
    if a.size == 0:
        return a.reshape(0, 4)
    return a[np.lexsort(a.T[::-1])]


def oracle_units(units, plants, N):
    us = []
    for B, u in units:
        U = orc.pack_unit(B, u)
        assert U is not None
        us.append(U)
    for p in plants:
        us.append(orc.plant_unit(p.base, p.e, p.d, lim=N, B=p.B, u=p.u))
    return orc.units_array(us), len(us)


@pytest.fixture(scope="module")
def config1():
    units = W.cls5_units(1000, 30000)
    assert len(units) == 725
    plants = W.plants(8, 0, 1000, 30000, N1)
    return units, plants


@pytest.mark.parametrize("r", [16, 20, 48])
def test_config1_parity(engine, oracle_table, config1, r):
    units, plants = config1
    t, path = oracle_table(N1, r)
    tid = engine.load_table(path, N1)
    try:
        arr, n = W.unit_array(units, plants, N1)
        hits, ctr = engine.cls5_run(tid, arr, n)
        oarr, on = oracle_units(units, plants, N1)
        ohits, (calls, gated, probes) = orc.cls5_run(t, oarr, on)
        assert (ctr.calls, ctr.gated, ctr.probes) == (calls, gated, probes)
        np.testing.assert_array_equal(sorted_hits(hits), sorted_hits(ohits))
        # every plant appears among the raw hits
        for j, p in enumerate(plants):
            sel = (hits["unit"] == len(units) + j) & (hits["d"] == p.d) & (hits["e"] == p.e)
            assert (hits["fp"][sel] == p.fp).any(), p
    finally:
        engine.free_table(tid)


def test_config1_no_gate_parity(engine, oracle_table, config1):
    units, plants = config1
    t, path = oracle_table(N1, 20)
    tid = engine.load_table(path, N1)
    try:
        arr, n = W.unit_array(units[:200], plants, N1)
        hits, ctr = engine.cls5_run(tid, arr, n, flags=s615.F_NO_GATE)
        oarr, on = oracle_units(units[:200], plants, N1)
        ohits, (calls, gated, probes) = orc.cls5_run(t, oarr, on, use_gate=False)
        assert gated == 0 and ctr.gated == 0
        assert (ctr.calls, ctr.probes) == (calls, probes)
        np.testing.assert_array_equal(sorted_hits(hits), sorted_hits(ohits))
    finally:
        engine.free_table(tid)


def test_plain_equals_batched_and_layouts(engine, oracle_table, config1):
    units, plants = config1
    _, path = oracle_table(N1, 16)
    arr, n = W.unit_array(units, plants, N1)
    res = []
    for layout in (s615.LAYOUT_WIDE, s615.LAYOUT_PACKED):
        tid = engine.load_table(path, N1, layout)
        for flags in (0, s615.F_PLAIN):
            hits, ctr = engine.cls5_run(tid, arr, n, flags=flags)
            res.append((sorted_hits(hits), (ctr.calls, ctr.gated, ctr.probes)))
        engine.free_table(tid)
    for h, c in res[1:]:
        np.testing.assert_array_equal(h, res[0][0])
        assert c == res[0][1]


def test_plants_verified_like_oracle(engine, oracle_table, config1):
    units, plants = config1
    t, path = oracle_table(N1, 20)
    tid = engine.load_table(path, N1)
    try:
        arr, n = W.unit_array(units, plants, N1)
        hits, _ = engine.cls5_run(tid, arr, n)
        sols = engine.verify(arr, n, hits, N1)
        lines = sorted(s615.solution_line(s) for s in sols)
        oarr, on = oracle_units(units, plants, N1)
        ohits, _ = orc.cls5_run(t, oarr, on)
        olines = sorted(orc.cls5_verify(oarr, ohits, N1))
        assert lines == olines
        for j, p in enumerate(plants):
            assert f"PLANT unit={len(units) + j} d={p.d} e={p.e} c1={p.c1} c2={p.c2}" in lines
        assert not [l for l in lines if l.startswith("SOLUTION")]
    finally:
        engine.free_table(tid)


def test_hit_overflow_is_reported(engine, oracle_table, config1):
    units, plants = config1
    _, path = oracle_table(N1, 16)
    tid = engine.load_table(path, N1)
    try:
        arr, n = W.unit_array(units, plants, N1)
        with pytest.raises(s615.S615Error) as ei:
            engine.cls5_run(tid, arr, n, hit_cap=2)
        assert ei.value.status == -9
    finally:
        engine.free_table(tid)


def test_band_3p2M_sample_parity(engine, oracle_table):
    # production-shape units (past the i128 wall, 1.8e7 grid points each)
    # against the oracle on a small shared table at r=16
    units = []
    B = 3_200_001
    while len(units) < 6:
        if W.eligible(B):
            us = s615.unit_candidates(B, 5)
            if us:
                units.append((B, us[len(us) // 2]))
        B += 997
    t, path = oracle_table(2000, 16)
    tid = engine.load_table(path, 2000)
    try:
        arr, n = W.unit_array(units, [], 2000)
        hits, ctr = engine.cls5_run(tid, arr, n)
        oarr, on = oracle_units(units, [], 2000)
        ohits, (calls, gated, probes) = orc.cls5_run(t, oarr, on)
        assert (ctr.calls, ctr.gated, ctr.probes) == (calls, gated, probes)
        assert calls > 6 * 10**7
        np.testing.assert_array_equal(sorted_hits(hits), sorted_hits(ohits))
    finally:
        engine.free_table(tid)


def test_band_production_table_parity(engine):
    # the configuration the bench times, against the oracle: 64 evenly spaced
    # Stage-1 units of the B ~ 3.2M band plus 8 plants on a table for
    # N = 76,667 built on the device in its default layout, at r = 20 so that
    # the filter gives raw hits; the table is exported (reference file bytes)
    # and probed by the oracle
    N, r = 76667, 20
    band = W.cls5_units(3_200_000, 3_219_999)
    idx = np.linspace(0, len(band) - 1, 64).astype(int)
    units = [band[i] for i in idx]
    plants = W.plants(8, 7, 3_200_000, 3_219_999, N)
    tid = engine.build_table(N, r)
    try:
        arr, n = W.unit_array(units, plants, N)
        hits, ctr = engine.cls5_run(tid, arr, n)
        hb, pk = engine.export_table(tid)
    finally:
        engine.free_table(tid)
    t = orc.Table.from_memory(hb, pk)
    del pk
    oarr, on = oracle_units(units, plants, N)
    ohits, (calls, gated, probes) = orc.cls5_run(t, oarr, on)
    assert (ctr.calls, ctr.gated, ctr.probes) == (calls, gated, probes)
    assert len(ohits) > len(plants)   # filter false positives at r = 20 (~26 expected), and the plants
    np.testing.assert_array_equal(sorted_hits(hits), sorted_hits(ohits))


def test_l2_window_does_not_change_results(engine, oracle_table, config1):
    # the peel launches mark config 1's table (1.9 MB) persisting in L2 by
    # default; without the window the counters and raw hits are the same
    units, plants = config1
    _, path = oracle_table(N1, 20)
    tid = engine.load_table(path, N1)
    try:
        arr, n = W.unit_array(units, plants, N1)
        h0, c0 = engine.cls5_run(tid, arr, n)
        h1, c1 = engine.cls5_run(tid, arr, n, flags=s615.F_NO_L2_WINDOW)
        assert (c0.calls, c0.gated, c0.probes, c0.hits) == (c1.calls, c1.gated, c1.probes, c1.hits)
        np.testing.assert_array_equal(sorted_hits(h0), sorted_hits(h1))
    finally:
        engine.free_table(tid)


def test_reference_selftest_plants(engine):
    """The reference's GPU self-test recipe (solve_516_v3.cu:1149-1170): 512
    class-5 plants, base = (14e)^6 + (21d)^6 + 42^6 (i^6 + j^6) with e in
    [1, 280], d in [1, 190] and i != j <= 4096, each unit a single residue per
    axis with fmax the planted value; every one must be found and verified."""
    N = 4096
    tid = engine.build_table(N, 48)
    try:
        rng = np.random.RandomState(1149)
        ps = []
        while len(ps) < 512:
            e, d = int(rng.randint(1, 281)), int(rng.randint(1, 191))
            i, j = (int(x) for x in rng.randint(1, N + 1, 2))
            if i != j:
                ps.append(W.Plant(172_049, 6, e, d, min(i, j), max(i, j)))
        arr, n = W.unit_array([], ps, N)
        hits, ctr = engine.cls5_run(tid, arr, n)
        sols = engine.verify(arr, n, hits, N)
        got = {(s.unit, s.d, s.e, s.c1, s.c2) for s in sols if s.kind == 1}
        assert sum((k, p.d, p.e, p.c1, p.c2) in got for k, p in enumerate(ps)) == 512
    finally:
        engine.free_table(tid)
