"""The (6,1,5) path against the reference's own programs (CPU).

tests/golden/ref615.json holds what the reference's fourcore_hunt_v3,
fourcore_cls5_gpu_v4 and fourcore_find_v4 printed on a B200 (built from the
reference sources by oracle/Makefile `ref`; tests/golden/gen_ref615.py).  Here:

  * the Stage-1 unit files (.buc) and reduced-T job files (.but) the hunt
    tool wrote equal, byte for byte (sha256), the lines formed from the
    engine's rule (s615_unit_candidates, s615_expand_unit) and from the
    oracle's (fourcore_hunt_v3.cpp:371-431);
  * the oracle's restatement of k_cls5_192 gives the reference binary's
    calls= and probes= and its gate percentage on every recorded class-5 run
    (config-1 window at r = 16, 20, 48 with and without the gate, and B ~ 3.2M
    slices), the same unit count and the same SOLUTION lines
    (fourcore_cls5_gpu_v4.cu:353-410, 472-562);
  * the oracle's restatement of run_batch gives fourcore_find_v4's summed
    find3 (classes 2-4) and find4 (class 1) counters, job and failT counts and
    SOLUTION lines, for Stage-1 units (--units) and for reduced-T job files
    (--jobs: the hunt tool's .but, and the engine's .bbj of the same jobs,
    whose bytes the reference read) (fourcore_find_v4.cu:460-562, 1094-1222).

The tables are the oracle's builds of the same (N, r); their bytes must
equal the reference builder's files (the fixture records their sha256).
"""
import hashlib
import json
import math
import os

import pytest

import orc
import s615

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIXTURE = os.path.join(ROOT, "tests", "golden", "ref615.json")


@pytest.fixture(scope="module")
def ref615():
    with open(FIXTURE) as f:
        return json.load(f)


def classes_of(s):
    return [int(c) for c in s.split(",")]


def buc_text(lo, hi, classes, rule):
    """The hunt tool's --emit-units lines: B ascending, classes in the given
    order, u ascending (fourcore_hunt_v3.cpp:371-381)."""
    out = []
    for B in range(lo, hi + 1):
        if B <= 1 or math.gcd(B, 42) != 1:
            continue
        for c in classes:
            out += [f"{c} {B} {u}\n" for u in rule(B, c)]
    return "".join(out)


def sha(text):
    return hashlib.sha256(text.encode()).hexdigest()


def test_stage1_units_equal_the_hunt_tool(ref615):
    assert len(ref615["units"]) >= 5
    for w in ref615["units"]:
        cl = classes_of(w["classes"])
        if w["lines"] > 20000:   # the 3.2M band: the engine's rule only (the oracle's is slower)
            rules = [s615.unit_candidates]
        else:
            rules = [s615.unit_candidates, orc.unit_candidates]
        for rule in rules:
            text = buc_text(w["lo"], w["hi"], cl, rule)
            assert text.count("\n") == w["lines"], (w, rule)
            assert sha(text) == w["sha256"], (w, rule)


def job_lines(jobs, n, fields):
    out = []
    for i in range(n):
        cls, B, u, f1, f2, tlo, thi = fields(jobs[i])
        out.append(f"{cls} {B} {u} {f1} {f2} {tlo} {thi}\n")
    return out


def test_reduced_T_jobs_equal_the_hunt_tool(ref615):
    assert len(ref615["jobs"]) >= 3
    for w in ref615["jobs"]:
        assert w["rc"] == 0
        cl = classes_of(w["classes"])
        units = [(c, B, u) for B in range(w["lo"], w["hi"] + 1) if math.gcd(B, 42) == 1
                 for c in cl for u in s615.unit_candidates(B, c)]
        assert len(units) == w["units"]
        # the unit file the expansion started from
        assert sha("".join(f"{c} {B} {u}\n" for c, B, u in units)) == w["units_sha256"]
        eng_lines, orc_lines, eng_fail, orc_fail = [], [], 0, 0
        for c, B, u in units:
            arr, n, fail = s615.expand_unit(B, u, c)
            eng_fail += fail
            eng_lines += job_lines(arr, n, lambda J: (J.cls, J.B, J.u, J.res_d, J.res_e,
                                                      J.base[0], J.base[1]))
            oarr, on, ofail = orc.expand_unit(B, u, c)
            orc_fail += ofail
            orc_lines += job_lines(oarr, on, lambda J: (J.cls, J.B, J.u, J.free1, J.free2,
                                                        J.T[0], J.T[1]))
        for lines, fail in ((eng_lines, eng_fail), (orc_lines, orc_fail)):
            assert len(lines) == w["lines"]
            assert fail == w["failT"]
            assert sha("".join(lines)) == w["sha256"]


_tables = {}


def table(N, r):
    if (N, r) not in _tables:
        _tables[(N, r)] = orc.Table.build_pairs(N, r)
    return _tables[(N, r)]


def test_oracle_tables_equal_the_reference_builder(ref615, tmp_path):
    for case in ref615["cls5"]:
        path = str(tmp_path / f"t{case['N']}_{case['r']}.bin")
        table(case["N"], case["r"]).save(path)
        with open(path, "rb") as f:
            assert hashlib.sha256(f.read()).hexdigest() == case["table_sha256"], case["tag"]


def test_cls5_counters_equal_the_reference_binary(ref615):
    cases = ref615["cls5"]
    assert len(cases) >= 8 and all("error" not in c for c in cases)
    for case in cases:
        units = [(B, u) for B in range(case["lo"], case["hi"] + 1) if math.gcd(B, 42) == 1
                 for u in orc.unit_candidates(B, 5)]
        assert case["lines"] == len(units) == case["units"], case["tag"]
        arr = orc.units_array([orc.pack_unit(B, u) for B, u in units])
        hits, (calls, gated, probes) = orc.cls5_run(table(case["N"], case["r"]), arr, len(units),
                                                    use_gate=case["gate"])
        assert (calls, probes) == (case["calls"], case["probes"]), (case, calls, probes)
        assert f"{100.0 * gated / calls:.1f}" == case["gate_pct"], case
        lines = orc.cls5_verify(arr, hits, case["N"])
        assert sorted(l for l in lines if l.startswith("SOLUTION")) == sorted(case["solution_lines"])
        assert case["solutions"] == len(case["solution_lines"])


def find_table(N, r):
    """The table a find run probes: the reference builder's bytes for N up to
    5,000; for larger N (class-1 windows) an N = 2,000 table, since the
    counters do not depend on the table and no raw hit is compared there."""
    return table(N, r) if N <= 5000 else table(2000, r)


def test_find_units_counters_equal_the_reference_binary(ref615):
    # classes 2-4 (find3) and class 1 (find4, the reference's repeated c4 tiles
    # restated by ref_tiles: fourcore_find_v4.cu:490-497, 300)
    cases = ref615["find"]
    assert len(cases) >= 5 and all("error" not in c for c in cases)
    assert any(c["classes"] == "1" for c in cases)
    for case in cases:
        cl = classes_of(case["classes"])
        units = [(c, B, u) for B in range(case["lo"], case["hi"] + 1) if math.gcd(B, 42) == 1
                 for c in cl for u in orc.unit_candidates(B, c)]
        assert len(units) == case["units"]
        parts = [orc.expand_unit(B, u, c) for c, B, u in units]
        assert sum(p[2] for p in parts) == case["failT"]
        jobs, n = orc.concat_jobs([p for p in parts if p[1]])
        assert n == case["jobs"]
        hits, ctr = orc.run_jobs(find_table(case["N"], case["r"]), jobs, n, use_gate=case["gate"],
                                 ref_tiles=True)
        want = [sum(m[k] for m in case["modes"].values()) for k in ("calls", "gated", "probes")]
        assert ctr == want, (case["summary"], ctr, want)
        if case["N"] <= 5000:
            exact, lines = orc.verify_jobs(jobs, hits, case["N"])
            assert sorted(l for l in lines if l.startswith("SOLUTION")) == sorted(case["solution_lines"])
        else:
            assert case["solution_lines"] == []


def test_find_job_files_equal_the_reference_binary(ref615, tmp_path):
    # --jobs on the hunt tool's .but file and on the same jobs written as .bbj by
    # the engine (fourcore_find_v4.cu:1094-1126, 1160-1222; fourcore_job_bin.hpp)
    cases = ref615["find_jobs"]
    assert {c["format"] for c in cases} == {"but", "bbj"} and all("error" not in c for c in cases)
    for case in cases:
        cl = classes_of(case["classes"])
        units = [(c, B, u) for B in range(case["lo"], case["hi"] + 1) if math.gcd(B, 42) == 1
                 for c in cl for u in orc.unit_candidates(B, c)]
        parts = [orc.expand_unit(B, u, c) for c, B, u in units]
        jobs, n = orc.concat_jobs([p for p in parts if p[1]])
        assert n == case["jobs"] and case["failT"] == 0
        if case["format"] == "bbj":   # the engine writes the bytes the reference read
            mine, m, _ = s615.expand_units([(c, B, u) for c, B, u in units])
            path = str(tmp_path / "j.bbj")
            s615.jobs_write(path, mine, m)
            with open(path, "rb") as f:
                assert hashlib.sha256(f.read()).hexdigest() == case["file_sha256"]
        N = max((B - 1) // 42 for _, B, _ in units)
        hits, ctr = orc.run_jobs(find_table(N, case["r"]), jobs, n, use_gate=case["gate"],
                                 ref_tiles=True)
        want = [sum(m[k] for m in case["modes"].values()) for k in ("calls", "gated", "probes")]
        assert ctr == want, (case["summary"], ctr, want)
        exact, lines = orc.verify_jobs(jobs, hits, N)
        assert sorted(l for l in lines if l.startswith("SOLUTION")) == sorted(case["solution_lines"])
