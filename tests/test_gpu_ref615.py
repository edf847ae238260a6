"""The engine's (6,1,5) drop-ins against the reference's own programs (GPU).

tests/golden/ref615.json records what fourcore_cls5_gpu_v4 and fourcore_find_v4
(built from the reference sources, run on a B200 by tests/golden/gen_ref615.py)
printed for fixed Stage-1 windows and one shared table file per (N, r).
bin/s615_cls5 and bin/s615_find, given the same units and a table file with
the same bytes (the oracle's build, which equals the reference builder's
file: tests/test_oracle615.py), must print the same summary (time excluded),
packed-unit count, gate percentage, counters and SOLUTION lines; the C ABI
(s615_cls5_run) must give the same counters.
"""
import json
import math
import os
import re
import subprocess

import pytest

import orc
import s615
import workloads as W

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN5 = os.path.join(ROOT, "six-one-five_b200", "bin", "s615_cls5")
BINF = os.path.join(ROOT, "six-one-five_b200", "bin", "s615_find")
DONE5 = re.compile(r"---- done cls5-gpu: solutions=(\d+) units=(\d+) calls=(\d+) probes=(\d+) time=\S+ ----")
PROG5 = re.compile(r"\[cls5-gpu\] units=\d+/\d+ calls=\d+ probes=\d+ gate=([\d.]+)%")
PACKED = re.compile(r"\[cls5-gpu\] packed (\d+)/(\d+) units")
GATE = re.compile(r"\[gate\] batch n=\d+ (?:mode=\d )?calls=(\d+) gated=(\d+) probes=(\d+)")
DONEF = re.compile(r"---- done: solutions=(\d+) jobs=(\d+) failT=(\d+) \(units stream\) ----")


def fixture():
    with open(os.path.join(ROOT, "tests", "golden", "ref615.json")) as f:
        return json.load(f)


def units_of(lo, hi, classes):
    return [(c, B, u) for B in range(lo, hi + 1) if math.gcd(B, 42) == 1
            for c in classes for u in s615.unit_candidates(B, c)]


def write_buc(path, units):
    with open(path, "w") as f:
        f.writelines(f"{c} {B} {u}\n" for c, B, u in units)


CLS5 = [c for c in fixture()["cls5"] if "error" not in c]
FIND = [c for c in fixture()["find"] if "error" not in c and c["classes"] != "1"]
FIND1 = [c for c in fixture()["find"] if "error" not in c and c["classes"] == "1"]
FINDJ = [c for c in fixture().get("find_jobs", []) if "error" not in c]


def cid(c):
    return f"{c['tag']}-r{c['r']}{'' if c['gate'] else '-nogate'}"


@pytest.mark.parametrize("case", CLS5, ids=cid)
def test_cls5_cli_prints_what_the_reference_printed(case, tmp_path, oracle_table):
    units = units_of(case["lo"], case["hi"], [5])
    buc = str(tmp_path / "u.buc")
    write_buc(buc, units)
    _, path = oracle_table(case["N"], case["r"])
    cmd = [BIN5, "--units", buc, "--N", str(case["N"]), "--r", str(case["r"]), "--load-table", path]
    if not case["gate"]:
        cmd.append("--no-gate")
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    d = DONE5.search(p.stdout)
    assert d, p.stdout
    assert tuple(int(x) for x in d.groups()) == (case["solutions"], case["units"], case["calls"],
                                                 case["probes"])
    pk = PACKED.search(p.stderr)
    assert (int(pk.group(1)), int(pk.group(2))) == (case["packed"], case["lines"])
    assert PROG5.findall(p.stderr)[-1] == case["gate_pct"]
    sols = [l for l in p.stdout.splitlines() if l.startswith("SOLUTION")]
    assert sorted(sols) == sorted(case["solution_lines"])


@pytest.mark.parametrize("case", CLS5, ids=cid)
def test_cls5_abi_counters_equal_the_reference(case, engine, oracle_table):
    units = [(B, u) for _, B, u in units_of(case["lo"], case["hi"], [5])]
    _, path = oracle_table(case["N"], case["r"])
    tid = engine.load_table(path, case["N"])
    try:
        arr, n = W.unit_array(units, [], case["N"])
        _, c = engine.cls5_run(tid, arr, n, flags=0 if case["gate"] else s615.F_NO_GATE)
        assert (c.calls, c.probes) == (case["calls"], case["probes"])
        assert f"{100.0 * c.gated / c.calls:.1f}" == case["gate_pct"]
    finally:
        engine.free_table(tid)


@pytest.mark.parametrize("case", FIND, ids=lambda c: f"{c['lo']}-r{c['r']}{'' if c['gate'] else '-nogate'}")
def test_find_cli_prints_what_the_reference_printed(case, tmp_path, oracle_table):
    units = units_of(case["lo"], case["hi"], [int(x) for x in case["classes"].split(",")])
    assert len(units) == case["units"]
    buc = str(tmp_path / "u.buc")
    write_buc(buc, units)
    _, path = oracle_table(case["N"], case["r"])
    cmd = [BINF, "--units", buc, "--r", str(case["r"]), "--N", str(case["N"]), "--load-table", path]
    if not case["gate"]:
        cmd.append("--no-gate")
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    d = DONEF.search(p.stdout)
    assert d, p.stdout
    assert tuple(int(x) for x in d.groups()) == (case["solutions"], case["jobs"], case["failT"])
    got = [0, 0, 0]
    for m in GATE.finditer(p.stderr):
        for k in range(3):
            got[k] += int(m.group(k + 1))
    want = [sum(m[k] for m in case["modes"].values()) for k in ("calls", "gated", "probes")]
    assert got == want, p.stderr[-2000:]
    sols = [l for l in p.stdout.splitlines() if l.startswith("SOLUTION")]
    assert sorted(sols) == sorted(case["solution_lines"])


def gate_sums(stderr):
    got = [0, 0, 0]
    for m in GATE.finditer(stderr):
        for k in range(3):
            got[k] += int(m.group(k + 1))
    return got


@pytest.mark.parametrize("case", FIND1, ids=lambda c: f"cls1-r{c['r']}{'' if c['gate'] else '-nogate'}")
def test_find_cli_class1(case, tmp_path):
    # class-1 units (find4).  The reference's k_find4 y tiles re-walk every
    # c4 >= lo + 2048 (fourcore_find_v4.cu:490-497, 300) and the engine visits
    # each c4 once, so the counters are set against the oracle's one-visit
    # form (its reference-tile form equals the fixture: tests/test_oracle615.py);
    # jobs, failT and SOLUTION lines against the fixture.  The table is built on
    # the device; the counters do not depend on its bytes.
    units = units_of(case["lo"], case["hi"], [1])
    assert len(units) == case["units"]
    buc = str(tmp_path / "u.buc")
    write_buc(buc, units)
    cmd = [BINF, "--units", buc, "--r", str(case["r"])]
    if not case["gate"]:
        cmd.append("--no-gate")
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    d = DONEF.search(p.stdout)
    assert d and tuple(int(x) for x in d.groups()) == (case["solutions"], case["jobs"], case["failT"])
    parts = [orc.expand_unit(B, u, c) for c, B, u in units]
    jobs, n = orc.concat_jobs([q for q in parts if q[1]])
    _, once = orc.run_jobs(orc.Table.build_pairs(2000, case["r"]), jobs, n, use_gate=case["gate"],
                           ref_tiles=False)
    assert gate_sums(p.stderr) == once
    assert [l for l in p.stdout.splitlines() if l.startswith("SOLUTION")] == case["solution_lines"]


DONEJ = re.compile(r"---- done: solutions=(\d+) jobs=(\d+) failT=(\d+)(?: \(bbj stream\))? ----")


@pytest.mark.parametrize("case", FINDJ, ids=lambda c: f"{c['format']}-r{c['r']}{'' if c['gate'] else '-nogate'}")
def test_find_cli_job_files(case, tmp_path, oracle_table):
    # --jobs on the same job file the reference read (.but lines of the hunt
    # tool, or their .bbj form written by s615_jobs_write) and the same table bytes
    units = units_of(case["lo"], case["hi"], [int(x) for x in case["classes"].split(",")])
    jobs, n, _ = s615.expand_units(units)
    path = str(tmp_path / f"j.{case['format']}")
    if case["format"] == "bbj":
        s615.jobs_write(path, jobs, n)
    else:
        with open(path, "w") as f:
            for i in range(n):
                J = jobs[i]
                f.write(f"{J.cls} {J.B} {J.u} {J.res_d} {J.res_e} {J.base[0]} {J.base[1]}\n")
    N = max((B - 1) // 42 for _, B, _ in units)
    _, tpath = oracle_table(N, case["r"])
    cmd = [BINF, "--jobs", path, "--r", str(case["r"]), "--N", str(N), "--load-table", tpath]
    if not case["gate"]:
        cmd.append("--no-gate")
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    d = DONEJ.search(p.stdout)
    assert d and tuple(int(x) for x in d.groups()) == (case["solutions"], case["jobs"], case["failT"])
    want = [sum(m[k] for m in case["modes"].values()) for k in ("calls", "gated", "probes")]
    assert gate_sums(p.stderr) == want
    assert sorted(l for l in p.stdout.splitlines() if l.startswith("SOLUTION")) == \
        sorted(case["solution_lines"])
