"""Reduced-T jobs on the host: expand_unit and the .but / .bbj job files.

The oracle restates expand_unit (fourcore_find_v4.cu:164-205, with its
compute_T_*_gmp failure count); the file layout is fourcore_job_bin.hpp:16-46
(parsed here with struct, independently of the library) and the text line is
the hunt tool's --expand --emit line (fourcore_hunt_v3.cpp:391).
"""
import os
import struct
import subprocess

import numpy as np
import pytest

import orc
import s615

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIND = os.path.join(ROOT, "six-one-five_b200", "bin", "s615_find")


def as_tuples(arr, n):
    return [(arr[i].cls, arr[i].B, arr[i].u, arr[i].res_d, arr[i].res_e, arr[i].base[0], arr[i].base[1])
            for i in range(n)]


def oracle_tuples(arr, n):
    return [(arr[i].cls, arr[i].B, arr[i].u, arr[i].free1, arr[i].free2, arr[i].T[0], arr[i].T[1])
            for i in range(n)]


@pytest.mark.parametrize("B", [24329, 28121, 100003, 400471, 1000003])
def test_expand_unit_matches_oracle(B):
    seen = 0
    for cls in (1, 2, 3, 4, 5):
        for u in orc.unit_candidates(B, cls)[:2]:
            a, n, fail = s615.expand_unit(B, u, cls)
            oa, on, ofail = orc.expand_unit(B, u, cls)
            assert (n, fail) == (on, ofail), (B, u, cls)
            assert as_tuples(a, n) == oracle_tuples(oa, on), (B, u, cls)
            assert all(a[i].kind == s615.S615_KIND_JOB for i in range(n))
            seen += n
    assert seen


def test_expand_unit_known_sample():
    # the reference's peel2 sample (B=100003, u=17646, d=9, e=44) is one of the unit's jobs
    a, n, _ = s615.expand_unit(100003, 17646, 5)
    T = (100003**6 - 17646**6 - (21 * 9) ** 6 - (14 * 44) ** 6) // 42**6
    assert (9, 44, T % 2**64, T >> 64) in [(a[i].res_d, a[i].res_e, a[i].base[0], a[i].base[1])
                                             for i in range(n)]
    for i in range(0, n, 997):   # every job's T is exact
        d, e = a[i].res_d, a[i].res_e
        R = 100003**6 - 17646**6 - (21 * d) ** 6 - (14 * e) ** 6
        assert R > 0 and R % 42**6 == 0 and R // 42**6 == a[i].base[0] + (a[i].base[1] << 64)


def test_job_files_round_trip(tmp_path):
    a, n, _ = s615.expand_unit(100003, 17646, 5)
    b1, n1, _ = s615.expand_unit(400471, orc.unit_candidates(400471, 4)[0], 4)
    jobs = (s615.Unit * (n + n1))()
    for i in range(n):
        jobs[i] = a[i]
    for i in range(n1):
        jobs[n + i] = b1[i]
    m = n + n1
    for name in ("j.bbj", "j.BBJ", "j.but"):
        path = str(tmp_path / name)
        s615.jobs_write(path, jobs, m)
        got, k, info = s615.jobs_read(path, chunk=4096)
        assert k == m and as_tuples(got, k) == as_tuples(jobs, m)
        assert info.binary == (name != "j.but")
        if info.binary:   # a caller's buffer that fits is filled in place; one too small is not used
            buf = (s615.Unit * (m + 5))()
            got, k, _ = s615.jobs_read(path, out=buf)
            assert got is buf and k == m and as_tuples(buf, k) == as_tuples(jobs, m)
            small = (s615.Unit * (m - 1))()
            got, k, _ = s615.jobs_read(path, out=small)
            assert got is not small and k == m and as_tuples(got, k) == as_tuples(jobs, m)
    raw = open(str(tmp_path / "j.bbj"), "rb").read()
    magic, ver, nj, rec, lo, hi, pad = struct.unpack("<IIQIIII", raw[:32])
    assert (magic, ver, nj, rec, lo, hi) == (0x4A424346, 2, m, 36, 100003, 400471)
    assert len(raw) == 32 + 36 * m
    recs = np.frombuffer(raw[32:], dtype=np.dtype([("cls", "u1"), ("pad", "u1", 3), ("B", "<u4"),
                                                   ("u", "<u4"), ("f1", "<u4"), ("f2", "<u4"),
                                                   ("tlo", "<u8"), ("thi", "<u8")]))
    assert [tuple(int(x) for x in (r["cls"], r["B"], r["u"], r["f1"], r["f2"], r["tlo"], r["thi"]))
            for r in recs] == as_tuples(jobs, m)
    text = open(str(tmp_path / "j.but")).read().splitlines()
    assert text[0] == "%d %d %d %d %d %d %d" % as_tuples(jobs, 1)[0]


def test_job_file_errors(tmp_path):
    bad = tmp_path / "bad.bbj"
    bad.write_bytes(struct.pack("<IIQIIII", 0x4A424346, 1, 1, 36, 0, 0, 0))   # version 1
    with pytest.raises(s615.S615Error) as e:
        s615.jobs_read(str(bad))
    assert e.value.status == -3
    with pytest.raises(s615.S615Error) as e:
        s615.jobs_read(str(tmp_path / "missing.bbj"))
    assert e.value.status == -2
    txt = tmp_path / "t.but"
    txt.write_text("5 100003 17646 9 44 1 0\nnot a job\n2 100139 73365 19 0 7 0\n")
    got, k, info = s615.jobs_read(str(txt))
    assert k == 2 and info.bad_lines == 1
    assert (got[1].cls, got[1].B, got[1].u, got[1].res_d, got[1].base[0]) == (2, 100139, 73365, 19, 7)
    for B, u, cls in [(100003, 17646, 6), (40_000_043, 17646, 5)]:   # no such class; B too large
        with pytest.raises(s615.S615Error) as e:
            s615.expand_unit(B, u, cls)
        assert e.value.status == -1


def test_job_unit_status():
    # kind 2 units: what a run does with each (searched / dropped / rejected)
    T3 = 3**6 + 4**6 + 5**6
    ok = [s615.make_job(5, 999999, 1, 3**6 + 4**6, 1, 1, lim=40),
          s615.make_job(2, 999998, 1, T3, 1, lim=40),
          s615.make_job(1, 999997, 1, T3 + 6**6, lim=40),
          s615.make_job(5, 100003, 17646, 2**127 + 5, 9, 44)]   # find2 takes any T
    dropped = [s615.make_job(3, 100003, 1, 2**121, 1),           # find3 window empty
               s615.make_job(2, 100003, 1, 0, 1),
               s615.make_job(1, 1000003, 1, 2**122, 0)]
    rejected = [s615.make_job(6, 100003, 1, 5, 1),
                s615.make_job(2, 40_000_043, 1, 5, 1)]          # lim beyond the device range
    st = lambda J: s615.lib().s615_unit_status(s615.C.byref(J))
    assert [st(J) for J in ok] == [0] * len(ok)
    assert [st(J) for J in dropped] == [1] * len(dropped)
    assert [st(J) for J in rejected] == [-3] * len(rejected)


def test_cli_emits_the_oracles_jobs(tmp_path):
    if not os.path.exists(FIND):
        pytest.skip("s615_find not built")
    units = [(5, 100003, 17646)] + [(c, B, u) for B in (24329, 28121) for c in (1, 4, 5)
                                    for u in orc.unit_candidates(B, c)]
    buc = tmp_path / "u.buc"
    buc.write_text("".join(f"{c} {B} {u}\n" for c, B, u in units))
    for name in ("o.bbj", "o.but"):
        out = tmp_path / name
        p = subprocess.run([FIND, "--units", str(buc), "--emit-jobs", str(out)], capture_output=True,
                           text=True, timeout=120)
        assert p.returncode == 0, p.stderr
        got, k, _ = s615.jobs_read(str(out))
        parts = [orc.expand_unit(B, u, c) for c, B, u in units]
        want = sum((oracle_tuples(a, n) for a, n, _ in parts), [])
        assert as_tuples(got, k) == want
        assert f"failT={sum(f for _, _, f in parts)}" in p.stderr
    p = subprocess.run([FIND, "--units", str(buc), "--emit-jobs", str(tmp_path / "c.bbj"),
                        "--max-expand", "100"], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0 and s615.jobs_read(str(tmp_path / "c.bbj"))[1] == 100
