#!/usr/bin/env python3
"""Record what the reference's own (6,1,5) programs print, as a test fixture.

Runs the reference binaries that `make -C oracle ref` compiles from the
reference sources into oracle/_ref (the GMP programs against the test-only
stand-in header oracle/gmpshim/gmpxx.h):

  fourcore_hunt_v3      Stage-1 units (.buc) and reduced-T jobs (.but) of
                        fixed B windows: line counts and sha256 of the files
                        (fourcore_hunt_v3.cpp:371-431).
  fourcore_cls5_gpu_v4  the class-5 peel + gate + probe on those units
                        against one shared table file (--load-table), for
                        r = 16, 20, 48 with and without the gate: the packed
                        unit count, the summary counters calls= and probes=,
                        the gate percentage and the SOLUTION lines
                        (fourcore_cls5_gpu_v4.cu:545-562, 611-709).
  fourcore_find_v4      --units on class 2-4 units (find3 leaf) and on class-1
                        units (find4), and --jobs on reduced-T job files (the
                        hunt tool's .but, and the same jobs written as .bbj by
                        the engine's s615_jobs_write): per-mode sums of its
                        [gate] batch counters, the job and failT counts and the
                        SOLUTION lines (fourcore_find_v4.cu:504-508, 1094-1222).

Tables come from the reference's own host builder (oracle/_ref/xor_build_save),
whose files the oracle reproduces byte for byte.  The counters of a class-5
run do not depend on the table, so the B ~ 3.2M slices use an N = 2,000 table
(the reference accepts a smaller --N than the units need, fourcore_cls5_gpu_v4.cu:697-701).

The GPU programs need a GPU: run this on a GPU machine and copy the output to
tests/golden/ref615.json; tests/test_oracle615.py compares the oracle with it
and tests/test_gpu_ref615.py the engine.

  python tests/golden/gen_ref615.py OUT.json
"""
import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.path.join(ROOT, "oracle", "_ref")
HUNT = os.path.join(REF, "fourcore_hunt_v3")
CLS5 = os.path.join(REF, "fourcore_cls5_gpu_v4")
FIND = os.path.join(REF, "fourcore_find_v4")
BUILD = os.path.join(REF, "xor_build_save")

# Stage-1 windows: (lo, hi, classes) -- the hunt tool's --lo/--hi are inclusive.
UNIT_WINDOWS = [
    (1000, 30000, "5"),            # the small CPU-runnable class-5 window
    (100000, 100299, "1,2,3,4,5"),
    (1000000, 1000299, "1,2,3,4,5"),
    (3200000, 3219999, "5"),       # the production-shape class-5 band
    (4500000, 4500999, "5"),
]
# Reduced-T expansions: (lo, hi, classes)
JOB_WINDOWS = [
    (150000, 150299, "2,3,4"),
    (1000000, 1000999, "1"),
    (2353974, 2354973, "1"),       # past the i128 wall (B^6 >= 2^128)
    (2353974, 2354003, "2,3,4"),
]
# Class-5 runs: (tag, lo, hi, N, r, gate)
CLS5_RUNS = [
    ("c1", 1000, 30000, 715, 16, True),
    ("c1", 1000, 30000, 715, 20, True),
    ("c1", 1000, 30000, 715, 48, True),
    ("c1", 1000, 30000, 715, 20, False),
    ("c1", 1000, 30000, 715, 48, False),
    ("band_a", 3200000, 3200006, 2000, 48, True),
    ("band_b", 3209997, 3210003, 2000, 48, True),
    ("band_c", 3219993, 3219999, 2000, 16, True),
    ("band_a", 3200000, 3200006, 2000, 48, False),
]
# find_v4 --units runs: (lo, hi, classes, r, gate).  Class 1 makes the
# reference build an N = 23,809 table on the host (a few minutes).
FIND_RUNS = [
    (150000, 150299, "2,3,4", 16, True),
    (150000, 150299, "2,3,4", 48, True),
    (150000, 150299, "2,3,4", 20, False),
    (1000000, 1000999, "1", 48, True),
    (1000000, 1000999, "1", 20, False),
]
# find_v4 --jobs runs on reduced-T job files: (format, lo, hi, classes, r, gate)
JOB_FILE_RUNS = [
    ("but", 150000, 150299, "2,3,4", 48, True),
    ("but", 150000, 150299, "2,3,4", 16, True),
    ("bbj", 150000, 150299, "2,3,4", 20, False),
]

DONE5 = re.compile(r"---- done cls5-gpu: solutions=(\d+) units=(\d+) calls=(\d+) probes=(\d+) time=(\S+)s ----")
PROG5 = re.compile(r"\[cls5-gpu\] units=\d+/\d+ calls=(\d+) probes=(\d+) gate=([\d.]+)%")
PACKED = re.compile(r"\[cls5-gpu\] packed (\d+)/(\d+) units")
GATE4 = re.compile(r"\[gate\] batch n=(\d+) mode=(\d) calls=(\d+) gated=(\d+) probes=(\d+)")
DONE4 = re.compile(r"---- done: solutions=(\d+) jobs=(\d+) failT=(\d+)(?: \((units|bbj) stream\))? ----")
UNITS4 = re.compile(r"\[units\] (\d+) from .* N=(\d+)")


def run(cmd, timeout=1800, env=None):
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, env=env)
    return p


def find_modes(stderr):
    """Per-mode sums of the [gate] batch lines (fourcore_find_v4.cu:504-508)."""
    modes = {}
    for m in GATE4.finditer(stderr):
        c = modes.setdefault(m.group(2), {"cands": 0, "calls": 0, "gated": 0, "probes": 0})
        c["cands"] += int(m.group(1))
        c["calls"] += int(m.group(3))
        c["gated"] += int(m.group(4))
        c["probes"] += int(m.group(5))
    return modes


def sha(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def emit_units(td, lo, hi, classes):
    path = os.path.join(td, f"u_{lo}_{hi}_{classes.replace(',', '')}.buc")
    if not os.path.exists(path):
        p = run([HUNT, "--lo", str(lo), "--hi", str(hi), "--classes", classes, "--emit-units", path])
        if p.returncode != 0:
            raise RuntimeError(p.stderr)
    return path


def table(td, N, r):
    path = os.path.join(td, f"xor_N{N}_r{r}.bin")
    if not os.path.exists(path):
        p = run([BUILD, "--N", str(N), "--r", str(r), "--out", path])
        if p.returncode != 0:
            raise RuntimeError(p.stderr)
    return path


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: gen_ref615.py OUT.json")
    out = sys.argv[1]
    fx = {"programs": "fourcore_hunt_v3, fourcore_cls5_gpu_v4, fourcore_find_v4, xor_build_save "
                      "(reference sources; GMP programs against oracle/gmpshim/gmpxx.h; nvcc sm_100a)",
          "units": [], "jobs": [], "cls5": [], "find": []}
    ok = True
    with tempfile.TemporaryDirectory() as td:
        for lo, hi, classes in UNIT_WINDOWS:
            path = emit_units(td, lo, hi, classes)
            with open(path) as f:
                lines = f.read().splitlines()
            per = {}
            for l in lines:
                per[l.split()[0]] = per.get(l.split()[0], 0) + 1
            fx["units"].append({"lo": lo, "hi": hi, "classes": classes, "lines": len(lines),
                                "per_class": per, "sha256": sha(path)})
            print(json.dumps(fx["units"][-1]))
        for lo, hi, classes in JOB_WINDOWS:
            ub = emit_units(td, lo, hi, classes)
            path = os.path.join(td, f"j_{lo}_{hi}.but")
            p = run([HUNT, "--lo", str(lo), "--hi", str(hi), "--classes", classes, "--expand",
                     "--emit", path])
            m = re.search(r"\[done\] eligible_B=(\d+) units=(\d+) T_jobs=(\d+) failT=(\d+)", p.stderr)
            with open(path) as f:
                n = sum(1 for _ in f)
            fx["jobs"].append({"lo": lo, "hi": hi, "classes": classes, "rc": p.returncode,
                               "lines": n, "sha256": sha(path), "units": int(m.group(2)),
                               "failT": int(m.group(4)), "units_sha256": sha(ub)})
            print(json.dumps(fx["jobs"][-1]))

        for tag, lo, hi, N, r, gate in CLS5_RUNS:
            ub = emit_units(td, lo, hi, "5")
            tb = table(td, N, r)
            cmd = [CLS5, "--units", ub, "--N", str(N), "--r", str(r), "--load-table", tb]
            if not gate:
                cmd.append("--no-gate")
            p = run(cmd)
            case = {"tag": tag, "lo": lo, "hi": hi, "N": N, "r": r, "gate": gate, "rc": p.returncode,
                    "cmd": " ".join(["oracle/_ref/fourcore_cls5_gpu_v4", "--units",
                                     f"<hunt_v3 --lo {lo} --hi {hi} --classes 5>", "--N", str(N),
                                     "--r", str(r), "--load-table", f"<xor_build_save --N {N} --r {r}>"]
                                    + ([] if gate else ["--no-gate"])),
                    "table_sha256": sha(tb)}
            d = DONE5.search(p.stdout)
            pk = PACKED.search(p.stderr)
            pr = PROG5.findall(p.stderr)
            if p.returncode != 0 or not d:
                case["error"] = (p.stderr.strip().splitlines() or ["?"])[-3:]
                ok = False
            else:
                case.update(solutions=int(d.group(1)), units=int(d.group(2)), calls=int(d.group(3)),
                            probes=int(d.group(4)), time_s=float(d.group(5)),
                            packed=int(pk.group(1)), lines=int(pk.group(2)),
                            gate_pct=pr[-1][2] if pr else None,
                            solution_lines=[l for l in p.stdout.splitlines() if l.startswith("SOLUTION")],
                            summary=d.group(0))
            fx["cls5"].append(case)
            print(json.dumps(case)[:400])

        # the reference's host table builder spills keys for large N
        scratch = os.path.join(td, "spill")
        os.makedirs(scratch, exist_ok=True)
        env = dict(os.environ, XOR_PEEL_SCRATCH=scratch)
        for lo, hi, classes, r, gate in FIND_RUNS:
            ub = emit_units(td, lo, hi, classes)
            cmd = [FIND, "--units", ub, "--r", str(r)]
            if not gate:
                cmd.append("--no-gate")
            p = run(cmd, env=env)
            case = {"lo": lo, "hi": hi, "classes": classes, "r": r, "gate": gate, "rc": p.returncode,
                    "cmd": " ".join(["oracle/_ref/fourcore_find_v4", "--units",
                                     f"<hunt_v3 --lo {lo} --hi {hi} --classes {classes}>", "--r", str(r)]
                                    + ([] if gate else ["--no-gate"]))}
            d = DONE4.search(p.stdout)
            u = UNITS4.search(p.stderr)
            if p.returncode != 0 or not d or not u:
                case["error"] = (p.stderr.strip().splitlines() or ["?"])[-3:]
                ok = False
            else:
                case.update(units=int(u.group(1)), N=int(u.group(2)), solutions=int(d.group(1)),
                            jobs=int(d.group(2)), failT=int(d.group(3)), modes=find_modes(p.stderr),
                            solution_lines=[l for l in p.stdout.splitlines() if l.startswith("SOLUTION")],
                            summary=d.group(0))
            fx["find"].append(case)
            print(json.dumps(case)[:400])

        fx["find_jobs"] = []
        for fmt, lo, hi, classes, r, gate in JOB_FILE_RUNS:
            but = os.path.join(td, f"j_{lo}_{hi}.but")
            if not os.path.exists(but):
                run([HUNT, "--lo", str(lo), "--hi", str(hi), "--classes", classes, "--expand",
                     "--emit", but])
            path = but
            if fmt == "bbj":   # the same jobs in the binary format, written by the engine
                sys.path.insert(0, os.path.join(ROOT, "six-one-five_b200"))
                import s615
                with open(but) as f:
                    rows = [[int(x) for x in l.split()] for l in f if l.strip()]
                arr = (s615.Unit * len(rows))()
                for k, (c, B, u, f1, f2, tlo, thi) in enumerate(rows):
                    arr[k] = s615.make_job(c, B, u, tlo | (thi << 64), f1, f2)
                path = os.path.join(td, f"j_{lo}_{hi}.bbj")
                s615.jobs_write(path, arr, len(rows))
            cmd = [FIND, "--jobs", path, "--r", str(r)]
            if not gate:
                cmd.append("--no-gate")
            p = run(cmd, env=env)
            case = {"format": fmt, "lo": lo, "hi": hi, "classes": classes, "r": r, "gate": gate,
                    "rc": p.returncode,
                    "cmd": " ".join(["oracle/_ref/fourcore_find_v4", "--jobs",
                                     f"<hunt_v3 --lo {lo} --hi {hi} --classes {classes} --expand"
                                     + (" as .bbj by s615_jobs_write" if fmt == "bbj" else "") + ">",
                                     "--r", str(r)] + ([] if gate else ["--no-gate"])),
                    "file_sha256": sha(path)}
            d = DONE4.search(p.stdout)
            if p.returncode != 0 or not d:
                case["error"] = (p.stderr.strip().splitlines() or ["?"])[-3:]
                ok = False
            else:
                case.update(solutions=int(d.group(1)), jobs=int(d.group(2)), failT=int(d.group(3)),
                            modes=find_modes(p.stderr),
                            solution_lines=[l for l in p.stdout.splitlines() if l.startswith("SOLUTION")],
                            summary=d.group(0))
            fx["find_jobs"].append(case)
            print(json.dumps(case)[:400])

    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    with open(out, "w") as f:
        json.dump(fx, f, indent=1)
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
