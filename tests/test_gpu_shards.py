"""Pair-space shard sets on the device (GPU).

A set of S oracle-built shard files loaded on the device must give the
oracle's shard set the same raw hits and counters for every unit kind; a
device-built set must answer every pair key (no false negatives), keep the
FPR of one table, and find the same verified solutions as one table.
"""
import numpy as np
import pytest

import orc
import s615
import workloads as W

pytestmark = pytest.mark.gpu

M64 = 2**64 - 1


def pair_keys(N):
    return np.array(sorted({(i**6 + j**6) & M64 for i in range(1, N + 1) for j in range(i, N + 1)}),
                    dtype=np.uint64)


@pytest.fixture(scope="module")
def oracle_shards(tmp_path_factory):
    d = tmp_path_factory.mktemp("shards")
    cache = {}

    def get(N, r, S):
        if (N, r, S) not in cache:
            parts = [orc.Table.build_pairs_shard(N, r, S, s) for s in range(S)]
            paths = []
            for s, p in enumerate(parts):
                path = str(d / f"xor_N{N}_r{r}_s{s}of{S}.bin")
                p.save(path)
                paths.append(path)
            cache[(N, r, S)] = (orc.Table.shard_set(parts), paths)
        return cache[(N, r, S)]

    return get


@pytest.mark.parametrize("S,r", [(4, 16), (3, 20)])
def test_set_parity_every_unit_kind(engine, oracle_shards, S, r):
    N = 54400 // 42
    ts, paths = oracle_shards(N, r, S)
    tid = engine.load_table_shards(paths, N)
    try:
        info = engine.table_info(tid)
        assert (info.hdr.shard_count, info.hdr.N, info.hdr.n_keys) == (S, N, ts.header.n_keys)
        # class 5
        units = W.cls5_units(54301, 54400)
        arr, n = s615.make_units(units)
        hits, ctr = engine.run(tid, arr, n)
        ou = orc.units_array([orc.pack_unit(B, u) for B, u in units])
        oh, (calls, gated, probes) = orc.cls5_run(ts, ou, len(units))
        assert (ctr.calls, ctr.gated, ctr.probes) == (calls, gated, probes)
        assert sorted((int(h["unit"]), int(h["d"]), int(h["e"]), int(h["fp"])) for h in hits) == \
            sorted((int(h["unit"]), int(h["d"]), int(h["e"]), int(h["fp"])) for h in oh)
        # (6,1,7) class 5
        parts = [orc.cands617(B) for B in (54347, 54349, 54353)]
        cands, nc = orc.concat617([p for p in parts if p[1]])
        u7, n7 = s615.make_units617((cands[i].B, cands[i].u, cands[i].w) for i in range(nc))
        h7, c7 = engine.run(tid, u7, n7)
        oh7, oc7 = orc.run617(ts, cands, nc)
        assert (c7.probes, c7.tri_total) == (oc7[0], oc7[3])
        assert sorted((int(h["unit"]), int(h["e"]), int(h["c4"]), int(h["fp"])) for h in h7) == \
            sorted((int(h["cand"]), int(h["c"]), int(h["d"]), int(h["fp"])) for h in oh7)
        # reduced-T jobs of classes 1-5
        jobs, oj, nj = [], [], 0
        for c, B, u in [(c, B, u) for B in (24329, 28121, 54347) for c in (1, 4, 5)
                        for u in orc.unit_candidates(B, c)]:
            a, k, _ = s615.expand_unit(B, u, c)
            jobs += [a[i] for i in range(k)]
            oj.append(orc.expand_unit(B, u, c))
        jarr = (s615.Unit * len(jobs))(*jobs)
        oarr, nj = orc.concat_jobs([p for p in oj if p[1]])
        hj, cj = engine.run(tid, jarr, nj)
        ohj, ocj = orc.run_jobs(ts, oarr, nj)
        assert (cj.calls, cj.gated, cj.probes) == tuple(ocj)
        assert sorted((int(h["unit"]), int(h["fp"])) for h in hj) == \
            sorted((int(h["job"]), int(h["fp"])) for h in ohj)
    finally:
        engine.free_table(tid)


@pytest.mark.parametrize("S", [2, 3, 8])
def test_device_built_set(engine, tmp_path, S):
    N, r = 1000, 48
    tid = engine.build_table_sharded(N, r, S)
    mono = engine.build_table(N, r)
    try:
        info = engine.table_info(tid)
        assert (info.hdr.shard_count, info.hdr.N, info.hdr.r) == (S, N, r)
        assert info.hdr.n_keys == engine.table_info(mono).hdr.n_keys
        keys = pair_keys(N)
        assert engine.query(tid, keys).all()            # no false negative over all pair keys
        hits = s615.C.c_int(0)
        s615._check(s615.lib().s615_fpr_smoke(engine._ctx, tid, s615.C.byref(hits)), "fpr_smoke")
        assert hits.value <= 16
        # the saved shards are the reference's file format, one file per shard
        paths = []
        for s in range(S):
            path = str(tmp_path / f"s{s}.bin")
            engine.save_table_shard(tid, s, path)
            paths.append(path)
        parts = [orc.Table.load(p, N) for p in paths]
        assert [p.header.shard_index for p in parts] == list(range(S))
        ts = orc.Table.shard_set(parts)
        rng = np.random.RandomState(S)
        rk = np.concatenate([keys[::7], rng.randint(0, 2**63, 1 << 18, dtype=np.int64).astype(np.uint64)])
        assert (engine.query(tid, rk) == ts.query(rk)).all()
        # reloading the files gives the same table
        tid2 = engine.load_table_shards(paths, N)
        assert (engine.query(tid2, rk) == engine.query(tid, rk)).all()
        engine.free_table(tid2)
        with pytest.raises(s615.S615Error) as e:         # one shard alone is not a table
            engine.load_table(paths[0], N)
        assert e.value.status == -3
        with pytest.raises(s615.S615Error):
            engine.load_table_shards(paths[::-1], N)     # shards out of order
    finally:
        engine.free_table(tid)
        engine.free_table(mono)


def test_set_finds_what_one_table_finds(engine):
    # a class-5 band with plants: same verified lines and plants with a set as with one table
    N = 3000
    units = W.cls5_units(120001, 120600)
    plants = W.plants(24, 9, 100000, 126000, N)
    arr, n = W.unit_array(units, plants, N)
    out = []
    for build in (lambda: engine.build_table(N, 48), lambda: engine.build_table_sharded(N, 48, 6)):
        tid = build()
        try:
            hits, ctr = engine.run(tid, arr, n)
            sols = engine.verify(arr, n, hits, N)
            out.append((ctr.probes, sorted(s615.solution_line(s) for s in sols)))
        finally:
            engine.free_table(tid)
    assert out[0] == out[1]
    assert sum(l.startswith("PLANT") for l in out[0][1]) >= len(plants)


def test_cli_shards(tmp_path):
    import os
    import re
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cli = os.path.join(root, "six-one-five_b200", "bin", "s615_cls5")
    buc = tmp_path / "u.buc"
    W.write_buc(str(buc), W.cls5_units(54301, 54400))
    prefix = str(tmp_path / "xor54k")
    done = re.compile(r"---- done cls5-gpu: solutions=(\d+) units=(\d+) calls=(\d+) probes=(\d+)")
    runs = [[], ["--shards", "4", "--save-shards", prefix],
            ["--load-shards", ",".join(f"{prefix}.shard{k}of4" for k in range(4))]]
    outs = []
    for extra in runs:
        p = subprocess.run([cli, "--units", str(buc), "--r", "48"] + extra, capture_output=True,
                           text=True, timeout=600)
        assert p.returncode == 0, p.stderr
        m = done.search(p.stdout)
        assert m, p.stdout
        outs.append((m.groups(), sorted(l for l in p.stdout.splitlines() if l.startswith("SOLUTION"))))
    assert outs[0] == outs[1] == outs[2]
    assert "pair-space shards" in p.stderr


@pytest.mark.parametrize("G", [2, 3, 4])
def test_probe_groups_change_nothing(engine, oracle_shards, G):
    """Probing a set in G passes (one group of shards each) gives the one-pass
    counters and raw hits, for every unit kind in one mixed batch."""
    N = 54400 // 42
    _, paths = oracle_shards(N, 16, 4)
    tid = engine.load_table_shards(paths, N)
    try:
        units = list(s615.make_units(W.cls5_units(54301, 54400))[0])
        c7, n7 = s615.candidates617(54347)
        units += [c7[i] for i in range(n7)]
        for B, u, c in [(24329, orc.unit_candidates(24329, 1)[0], 1), (54301, 5856, 5)]:
            a, k, _ = s615.expand_unit(B, u, c)
            units += [a[i] for i in range(min(k, 3000))]
        arr = (s615.Unit * len(units))(*units)
        key = lambda hs: sorted(tuple(int(h[f]) for f in ("unit", "d", "e", "c4", "fp")) for h in hs)
        fields = ("calls", "gated", "probes", "pos", "hits", "tri_total", "tri_skipped")
        out = []
        for g, flags in ((1, 0), (G, 0), (1, s615.F_SHARP), (G, s615.F_SHARP)):
            engine.set_probe_groups(tid, g)
            h, c = engine.run(tid, arr, len(units), flags)
            out.append((key(h), tuple(getattr(c, f) for f in fields)))
        assert out[0] == out[1] and out[2] == out[3]
        engine.set_probe_groups(tid, G)                   # the plain form, a few units
        hp, cp = engine.run(tid, arr, 40, s615.F_PLAIN)
        engine.set_probe_groups(tid, 1)
        h1, c1 = engine.run(tid, arr, 40, s615.F_PLAIN)
        assert key(hp) == key(h1) and tuple(getattr(cp, f) for f in fields) == \
            tuple(getattr(c1, f) for f in fields)
        with pytest.raises(s615.S615Error):
            engine.set_probe_groups(tid, 5)                # more groups than shards
    finally:
        engine.free_table(tid)
    mono = engine.build_table(300, 16)
    try:
        with pytest.raises(s615.S615Error):
            engine.set_probe_groups(mono, 2)               # a single table has no groups
    finally:
        engine.free_table(mono)


def test_shard_ranges_split_the_set(engine, oracle_shards, tmp_path):
    """The parts two GPUs would hold of one set, run in turn on this GPU: each
    part gives the whole set's counters, and their raw hits together are the
    whole set's; a part answers exactly the keys of its own shards."""
    N = 54400 // 42
    _, paths = oracle_shards(N, 16, 4)
    full = engine.load_table_shards(paths, N)
    parts = [engine.load_table_shards(paths[:2], N), engine.load_table_shards(paths[2:], N)]
    built = engine.build_table_shard_range(N, 48, 4, 1, 3)
    key = lambda hs: sorted(tuple(int(h[f]) for f in ("unit", "d", "e", "c4", "fp")) for h in hs)
    fields = ("calls", "gated", "probes", "pos", "tri_total", "tri_skipped")
    try:
        units = list(s615.make_units(W.cls5_units(54301, 54400))[0])
        c7, n7 = s615.candidates617(54347)
        units += [c7[i] for i in range(n7)]
        arr = (s615.Unit * len(units))(*units)
        hf, cf = engine.run(full, arr, len(units))
        union = []
        for tid, lo in zip(parts, (0, 2)):
            info = engine.table_info(tid)
            assert (info.hdr.shard_count, info.hdr.shard_index) == (4, lo)
            h, c = engine.run(tid, arr, len(units))
            assert tuple(getattr(c, f) for f in fields) == tuple(getattr(cf, f) for f in fields)
            union += key(h)
        assert sorted(union) == key(hf) and len(union) > 0
        keys = pair_keys(N)
        owner = np.array([orc.shard_of(int(k), 4) for k in keys])
        for tid, lo in zip(parts + [built], (0, 2, 1)):
            got = engine.query(tid, keys).astype(bool)
            mine = (owner >= lo) & (owner < lo + 2)
            assert got[mine].all() and not got[~mine].any()
        engine.save_table_shard(built, 2, str(tmp_path / "s2.bin"))
        assert orc.Table.load(str(tmp_path / "s2.bin"), N).header.shard_index == 2
        with pytest.raises(s615.S615Error):
            engine.save_table_shard(built, 0, str(tmp_path / "s0.bin"))   # not held here
    finally:
        for tid in [full, built] + parts:
            engine.free_table(tid)
