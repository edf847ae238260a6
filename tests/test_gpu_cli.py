"""The drop-in command lines on the device (GPU).

bin/s615_617 against what the reference's own solve_617_v1 printed on a B200
for the same arguments (tests/golden/ref617.json, made by
tests/golden/gen_ref617.py), and bin/s615_cls5 against the oracle's counters
for the same units.
"""
import json
import os
import re
import subprocess

import pytest

import orc
import s615
import workloads as W

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN617 = os.path.join(ROOT, "six-one-five_b200", "bin", "s615_617")
BIN5 = os.path.join(ROOT, "six-one-five_b200", "bin", "s615_cls5")
SUMMARY = re.compile(
    r"cls(\d): cands=(\d+) probes=(\S+) kernel=\S+ rate=\S+ probes/s exact=(\d+) fp-false=(\d+) "
    r"gate-kill=([\d.]+)%(?: tri-skip=[\d.]+% \((\d+)/(\d+) c4\))?")


def ref_cases():
    with open(os.path.join(ROOT, "tests", "golden", "ref617.json")) as f:
        return [c for c in json.load(f)["cases"] if "error" not in c]


@pytest.mark.parametrize("case", ref_cases(), ids=lambda c: f"{c['B_lo']}-{c['B_hi']}-r{c['r']}"
                         f"-c{c.get('classes', '5')}"
                         f"{'' if c['gate'] else '-nogate'}{'' if c['tri'] else '-notri'}")
def test_617_cli_prints_what_the_reference_printed(case):
    cmd = [BIN617, str(case["B_lo"]), str(case["B_hi"]), case.get("classes", "5"), "--branch-a-only",
           "--r", str(case["r"]), "--quiet"]
    if not case["gate"]:
        cmd.append("--no-gate")
    if not case["tri"]:
        cmd.append("--no-tri-gate")
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    per = {}
    for m in SUMMARY.finditer(p.stderr):
        c = {"cands": int(m.group(2)), "probes": m.group(3), "exact": int(m.group(4)),
             "fp_false": int(m.group(5)), "gate_kill": m.group(6)}
        if m.group(7):
            c.update(tri_skipped=int(m.group(7)), tri_total=int(m.group(8)))
        per[m.group(1)] = c
    want = case.get("per_class", {"5": {k: case[k] for k in ("cands", "probes", "exact", "fp_false",
                                                              "gate_kill", "tri_skipped", "tri_total")
                                        if k in case}})
    assert per == want, p.stderr
    sols = [l for l in p.stdout.splitlines() if l.startswith("SOLUTION")]
    assert sorted(sols) == sorted(case["solutions"])


def test_617_cli_check_known_and_selftest(tmp_path, golden):
    known = tmp_path / "known.txt"
    known.write_text("# test database\n" + "".join(
        f"{k['B']} = " + " + ".join(str(x) for x in reversed(k["terms"])) + "  | 2nd kind | test\n"
        for k in golden["known617_cls5"]))
    p = subprocess.run([BIN617, "54301", "54400", "5", "--branch-a-only", "--quiet", "--check-known",
                        "--known-file", str(known)], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    assert "expected=1 found=1 missing=0 new-candidates=0 PASS" in p.stderr
    p = subprocess.run([BIN617, "--selftest"], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0 and "[plant] find4 (cls5 shape): 256/256" in p.stderr, p.stderr


def test_cls5_cli_counters_equal_oracle(tmp_path, oracle_table):
    # config-1 units as a .buc file; the done line's calls/probes against the oracle
    N = 715
    t, path = oracle_table(N, 48)
    units = W.cls5_units(1000, 30000)
    buc = tmp_path / "u.buc"
    W.write_buc(str(buc), units)
    p = subprocess.run([BIN5, "--units", str(buc), "--N", str(N), "--load-table", path, "--r", "48"],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    m = re.search(r"---- done cls5-gpu: solutions=(\d+) units=(\d+) calls=(\d+) probes=(\d+)", p.stdout)
    assert m, p.stdout
    arr = orc.units_array([orc.pack_unit(B, u) for B, u in units])
    _, (calls, gated, probes) = orc.cls5_run(t, arr, len(units))
    assert (int(m.group(2)), int(m.group(3)), int(m.group(4))) == (len(units), calls, probes)
    assert int(m.group(1)) == 0 and "SOLUTION" not in p.stdout


def test_cls5_cli_plants_and_serve(tmp_path, oracle_table):
    N = 715
    _, path = oracle_table(N, 48)
    units = W.cls5_units(1000, 30000)
    buc = tmp_path / "u.buc"
    W.write_buc(str(buc), units)
    p = subprocess.run([BIN5, "--units", str(buc), "--N", str(N), "--load-table", path,
                        "--plant", "16:3"], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    assert "[plant] recovered 16/16" in p.stderr
    # the same units streamed through the serving loop, 100 per request
    with open(buc) as f:
        p = subprocess.run([BIN5, "--serve", "--N", str(N), "--load-table", path, "--batch", "100"],
                           stdin=f, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    m = re.search(r"---- done cls5-gpu serve: solutions=(\d+) units=(\d+) requests=(\d+)", p.stdout)
    assert m and int(m.group(2)) == len(units) and int(m.group(3)) == (len(units) + 99) // 100
    assert int(m.group(1)) == 0


def test_cls5_cli_journal_resumes(tmp_path, oracle_table):
    # a run journals its chunks; after a crash (journal cut inside a block) the
    # rerun searches only the units not committed, and every plant is still
    # recovered once (before or after the restart)
    N = 715
    t, path = oracle_table(N, 20)
    units = W.cls5_units(1000, 30000)
    buc = tmp_path / "u.buc"
    W.write_buc(str(buc), units)
    jpath = tmp_path / "run.journal"
    cmd = [BIN5, "--units", str(buc), "--N", str(N), "--load-table", path, "--plant", "8:3",
           "--batch", "200", "--journal", str(jpath)]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    total = len(units) + 8
    assert "[plant] recovered 8/8" in p.stderr
    full = jpath.read_bytes()
    # cut inside the third block: two committed blocks of 200 units survive
    starts = [i for i in range(len(full)) if full.startswith(b"B ", i) and (i == 0 or full[i - 1] == 10)]
    assert len(starts) == (total + 199) // 200
    jpath.write_bytes(full[:starts[2] + (starts[3] - starts[2]) // 2])
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    assert f"[journal] 400 of {total} units already committed; searching {total - 400}" in p.stderr
    assert "[plant] recovered 8/8" in p.stderr
    m = re.search(r"---- done cls5-gpu: solutions=(\d+) units=(\d+) calls=(\d+) probes=(\d+)", p.stdout)
    assert m and int(m.group(1)) == 0 and int(m.group(2)) == total
    # the journal now commits every unit exactly once
    with s615.Journal(str(jpath)) as j:
        assert j.stats()[0] == total
        assert len({(u.kind, u.B, u.u, tuple(u.base)) for u in j.units()}) == total
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    assert f"[journal] {total} of {total} units already committed; searching 0" in p.stderr
    assert "[plant] recovered 8/8" in p.stderr
