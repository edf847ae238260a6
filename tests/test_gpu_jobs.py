"""Reduced-T jobs (fourcore_find_v4 --jobs / --units) on the device (GPU).

The oracle restates expand_unit, make_cand + k_find2 / k_find3 / k_find4 and
run_batch's exact filter with report_solution (fourcore_find_v4.cu:164-205,
401-425, 233-338, 536-560, 427-457).  Job units (kind 2) must give the
oracle's counters, raw hits, exact matches and SOLUTION lines; a Stage-1 unit
and the jobs it expands into must give the same search.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import orc
import s615
import workloads as W

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIND = os.path.join(ROOT, "six-one-five_b200", "bin", "s615_find")


def stage1(lo, hi, classes):
    return [(c, B, u) for B in range(lo, hi + 1) if B % 2 and B % 3 and B % 7
            for c in classes for u in orc.unit_candidates(B, c)]


def expand(units):
    """(engine jobs, oracle jobs, n, origin unit of each job)."""
    mine, parts, origin = [], [], []
    for k, (c, B, u) in enumerate(units):
        a, n, _ = s615.expand_unit(B, u, c)
        mine += [a[i] for i in range(n)]
        parts.append(orc.expand_unit(B, u, c))
        origin += [k] * n
    oarr, n = orc.concat_jobs([p for p in parts if p[1]])
    assert n == len(mine)
    return (s615.Unit * max(n, 1))(*mine), oarr, n, origin


def plants(rng, N, count):
    """Planted jobs in the shape of the reference's GPU selftest (fake B, lim = N)."""
    out = []
    for k in range(count):
        mode = (2, 3, 4)[k % 3]
        c = sorted(int(x) for x in rng.choice(np.arange(1, N + 1), mode, replace=False))
        T = sum(x**6 for x in c)
        cls = {2: 5, 3: 2 + (k // 3) % 3, 4: 1}[mode]
        out.append((s615.make_job(cls, 999999 - k, 1, T, 1, 1 if cls == 5 else 0, lim=N), c))
    return out


def oracle_job(J):
    o = orc.OrcJob()
    o.cls, o.lim, o.B, o.u = J.cls, J.lim or (J.B - 1) // 42, J.B, J.u
    o.free1, o.free2, o.T[0], o.T[1] = J.res_d, J.res_e, J.base[0], J.base[1]
    return o


def mine(hits, arr):
    # find2 rows carry c3 = 1 in e; the oracle's find2 hits carry 0
    return sorted((int(h["unit"]), 0 if arr[int(h["unit"])].cls == 5 else int(h["e"]), int(h["c4"]),
                   int(h["fp"])) for h in hits)


def theirs(hits):
    return sorted((int(h["job"]), int(h["c3"]), int(h["c4"]), int(h["fp"])) for h in hits)


@pytest.fixture(scope="module")
def band():
    units = stage1(24001, 26000, (1, 2, 3, 4, 5))
    assert {c for c, _, _ in units} >= {1, 4, 5}
    arr, oarr, n, _ = expand(units)
    N = 26000 // 42
    P = plants(np.random.RandomState(7), N, 48)
    allj = (s615.Unit * (n + len(P)))()
    oall = (orc.OrcJob * (n + len(P)))()
    for i in range(n):
        allj[i], oall[i] = arr[i], oarr[i]
    for j, (J, _) in enumerate(P):
        allj[n + j], oall[n + j] = J, oracle_job(J)
    return allj, oall, n + len(P), n, P, N


@pytest.mark.parametrize("r", [16, 48])
def test_jobs_parity(engine, oracle_table, band, r):
    arr, oarr, n, n_real, P, N = band
    t, path = oracle_table(N, r)
    tid = engine.load_table(path, N)
    try:
        hits, ctr = engine.run(tid, arr, n)
        oh, (calls, gated, probes) = orc.run_jobs(t, oarr, n)
        assert (ctr.calls, ctr.gated, ctr.probes, ctr.pos) == (calls, gated, probes, calls)
        assert mine(hits, arr) == theirs(oh)
        sols = engine.verify(arr, n, hits, N)
        exact, lines = orc.verify_jobs(oarr, oh, N)
        assert len(sols) == exact
        assert sorted(s615.solution_line(s) for s in sols if s.kind == 0) == sorted(lines)
        got = {(s.unit, s.c1, s.c2, s.c3, s.c4) for s in sols if s.kind == s615.S615_KIND_JOB}
        for j, (J, c) in enumerate(P):   # every plant is an exact match
            c = c + [0] * (4 - len(c))
            assert (n_real + j, *c) in got, (j, J.cls, c)
    finally:
        engine.free_table(tid)


def test_units_equal_their_jobs(engine, oracle_table):
    """A Stage-1 unit and its expanded jobs: same counters and raw hits."""
    N = 2000
    units = stage1(400000, 400600, (2, 3, 4)) + [(1, B, u) for B in (24329, 28121, 32105)
                                                 for u in orc.unit_candidates(B, 1)]
    cls5 = [(5, B, u) for B, u in W.cls5_units(100001, 100400)][:4]
    t, path = oracle_table(N, 16)
    tid = engine.load_table(path, N)
    try:
        for group in (units, cls5):
            uarr = (s615.Unit * len(group))()
            for i, (c, B, u) in enumerate(group):
                uarr[i].cls, uarr[i].B, uarr[i].u = c, B, u
            uh, uc = engine.run(tid, uarr, len(group))
            jarr, _, n, origin = expand(group)
            jh, jc = engine.run(tid, jarr, n)
            assert (jc.calls, jc.gated, jc.probes) == (uc.pos, uc.gated, uc.probes)
            if group is units:
                assert uc.calls == uc.pos
            ukey = sorted((int(h["unit"]), int(h["d"]), int(h["e"]), int(h["c4"]), int(h["fp"]))
                          for h in uh)
            jkey = []
            for h in jh:
                J = jarr[int(h["unit"])]
                c = J.cls
                d = J.res_d
                e = J.res_e if c == 5 else int(h["e"])
                jkey.append((origin[int(h["unit"])], d, e, int(h["c4"]), int(h["fp"])))
            assert ukey == sorted(jkey)
    finally:
        engine.free_table(tid)


def test_jobs_in_a_mixed_batch(engine, oracle_table, band):
    # job rows next to Stage-1 units and (6,1,7) units in one call == separate calls
    arr, _, n, _, _, N = band
    _, path = oracle_table(N, 16)
    tid = engine.load_table(path, N)
    try:
        u5 = W.cls5_units(24001, 26000)
        c7, n7 = s615.candidates617(24329)
        assert n7
        mixed = (s615.Unit * (len(u5) + n + n7))()
        for i, (B, u) in enumerate(u5):
            mixed[i].cls, mixed[i].B, mixed[i].u = 5, B, u
        for i in range(n):
            mixed[len(u5) + i] = arr[i]
        for i in range(n7):
            mixed[len(u5) + n + i] = c7[i]
        hm, cm = engine.run(tid, mixed, len(mixed))
        parts = []
        for lo, k in ((0, len(u5)), (len(u5), n), (len(u5) + n, n7)):
            sub = (s615.Unit * max(k, 1))(*[mixed[lo + i] for i in range(k)])
            h, c = engine.run(tid, sub, k)
            h = h.copy()
            h["unit"] += lo
            parts.append((h, c))
        for f in ("calls", "gated", "probes", "pos", "hits"):
            assert getattr(cm, f) == sum(getattr(c, f) for _, c in parts), f
        key = lambda hs: sorted(tuple(int(h[f]) for f in ("unit", "d", "e", "c4", "fp")) for h in hs)
        assert key(hm) == key(np.concatenate([h for h, _ in parts]))
    finally:
        engine.free_table(tid)


def test_large_batch_threads_equal_chunks(engine, oracle_table, band):
    """A batch of 16,384 units or more is packed and cut into work items on
    several host threads; the same units in chunks below that size take one
    thread each.  Job-row runs, Stage-1 units and (6,1,7) candidates are
    interleaved so that thread ranges start beside every kind of unit."""
    arr, _, n, _, _, N = band
    _, path = oracle_table(N, 16)
    tid = engine.load_table(path, N)
    try:
        u5 = W.cls5_units(24001, 26000)
        c7, n7 = s615.candidates617(24329)
        seq, k = [], 0
        while len(seq) < 60_000:
            run = 1 + (k * 7919) % 3000
            seq += [arr[(k * 131 + i) % n] for i in range(run)]
            B, u = u5[k % len(u5)]
            x = s615.Unit()
            x.cls, x.B, x.u = 5, B, u
            seq.append(x)
            seq.append(c7[k % n7])
            k += 1
        whole = (s615.Unit * len(seq))(*seq)
        hw, cw = engine.run(tid, whole, len(seq))
        parts, tot = [], {f: 0 for f in ("calls", "gated", "probes", "pos", "hits")}
        for lo in range(0, len(seq), 9000):
            m = min(9000, len(seq) - lo)
            sub = (s615.Unit * m)(*seq[lo:lo + m])
            h, c = engine.run(tid, sub, m)
            h = h.copy()
            h["unit"] += lo
            parts.append(h)
            for f in tot:
                tot[f] += getattr(c, f)
        for f in tot:
            assert getattr(cw, f) == tot[f], f
        key = lambda hs: sorted(tuple(int(h[f]) for f in ("unit", "d", "e", "c4", "fp")) for h in hs)
        assert key(hw) == key(np.concatenate(parts))
        assert cw.hits > 0
    finally:
        engine.free_table(tid)


DONE = re.compile(r"---- done: solutions=(\d+) jobs=(\d+) failT=(\d+)( \(\w+ stream\))? ----")


def test_cli_job_files(tmp_path, band):
    arr, oarr, n, n_real, _, N = band
    path_b, path_t = str(tmp_path / "j.bbj"), str(tmp_path / "j.but")
    s615.jobs_write(path_b, arr, n_real)
    s615.jobs_write(path_t, arr, n_real)
    t = orc.Table.build_pairs(N, 16)
    oh, (calls, gated, probes) = orc.run_jobs(t, oarr, n_real)
    exact, lines = orc.verify_jobs(oarr, oh, N)
    gate_re = re.compile(r"\[gate\] batch n=\d+ calls=(\d+) gated=(\d+) probes=(\d+)")
    outs = []
    for path, tail in ((path_b, " (bbj stream)"), (path_t, None)):
        p = subprocess.run([FIND, "--jobs", path, "--r", "16", "--N", str(N), "--batch", "20000"],
                           capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stderr
        m = DONE.search(p.stdout)
        assert m and (int(m.group(1)), int(m.group(2))) == (exact, n_real) and m.group(4) == tail
        g = [tuple(int(x) for x in mm.groups()) for mm in gate_re.finditer(p.stderr)]
        assert tuple(map(sum, zip(*g))) == (calls, gated, probes)
        sols = sorted(l for l in p.stdout.splitlines() if l.startswith("SOLUTION"))
        assert sols == sorted(lines)
        outs.append(sols)
    assert outs[0] == outs[1]


def test_cli_units_stream(tmp_path):
    units = stage1(24001, 24600, (1, 2, 3, 4, 5))
    buc = tmp_path / "u.buc"
    buc.write_text("".join(f"{c} {B} {u}\n" for c, B, u in units))
    p = subprocess.run([FIND, "--units", str(buc), "--quiet"], capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr
    m = DONE.search(p.stdout)
    parts = [orc.expand_unit(B, u, c) for c, B, u in units]
    assert m and m.group(4) == " (units stream)"
    assert (int(m.group(2)), int(m.group(3))) == (sum(x[1] for x in parts), sum(x[2] for x in parts))


def test_cli_selftest_gpu():
    p = subprocess.run([FIND, "--selftest-gpu"], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    for mode in (2, 3, 4):
        assert re.search(rf"find{mode} plant exact_hits=1 ", p.stdout), p.stdout
    assert "[selftest-gpu] PASS (exact=3)" in p.stdout


def test_cli_jobs_on_a_shard_set(tmp_path, band):
    # the same job file against one table and against a 3-shard set: same lines
    arr, _, _, n_real, _, N = band
    path = str(tmp_path / "j.bbj")
    s615.jobs_write(path, arr, n_real)
    gate_re = re.compile(r"\[gate\] batch n=\d+ calls=(\d+) gated=(\d+) probes=(\d+)")
    outs = []
    for extra in ([], ["--shards", "3"]):
        p = subprocess.run([FIND, "--jobs", path, "--r", "16", "--batch", "50000"] + extra,
                           capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stderr
        g = [tuple(int(x) for x in m.groups()) for m in gate_re.finditer(p.stderr)]
        sols = sorted(l for l in p.stdout.splitlines() if l.startswith("SOLUTION"))
        outs.append((DONE.search(p.stdout).groups(), tuple(map(sum, zip(*g))), sols))
    assert outs[0] == outs[1]
