#!/usr/bin/env python3
"""Record the reference's own (6,1,7) Branch-A counts (classes 1-5) as a fixture.

Runs the reference GPU binary oracle/_ref/solve_617_v1 (built from the
reference sources by `make -C oracle ref`) on a few small B ranges and writes
what its summary prints (candidates, probes, exact / fp-false, gate-kill,
tri-skip counts, SOLUTION lines) to a JSON file.  It needs a GPU; run it on a
GPU machine and copy the output to tests/golden/ref617.json, which
tests/test_oracle617.py compares with the oracle on the same inputs.

  python tests/golden/gen_ref617.py OUT.json
"""
import json
import os
import re
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
BIN = os.path.join(ROOT, "oracle", "_ref", "solve_617_v1")

# (B_lo, B_hi, r, gate, tri, classes)
CASES = [
    (54301, 54400, 48, True, True, "5"),
    (54301, 54400, 16, True, True, "5"),
    (59801, 59900, 20, True, True, "5"),
    (63601, 63700, 48, True, True, "5"),
    (54301, 54400, 48, True, False, "5"),
    (54301, 54340, 20, False, True, "5"),
    (34701, 34800, 48, True, True, "1234"),
    (38101, 38200, 16, True, True, "1234"),
    (39701, 39800, 20, True, True, "1234"),
    (39701, 39760, 48, True, False, "34"),
    (24301, 24400, 48, True, True, "1"),
    (24301, 24400, 20, False, True, "1"),
    (28101, 28200, 16, True, False, "12"),
]

SUMMARY = re.compile(
    r"cls(\d): cands=(\d+) probes=(\S+) kernel=\S+ rate=\S+ probes/s exact=(\d+) fp-false=(\d+) "
    r"gate-kill=([\d.]+)%(?: tri-skip=[\d.]+% \((\d+)/(\d+) c4\))?")


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: gen_ref617.py OUT.json")
    out = sys.argv[1]
    cases = []
    for lo, hi, r, gate, tri, classes in CASES:
        cmd = [BIN, str(lo), str(hi), classes, "--branch-a-only", "--r", str(r), "--quiet"]
        if not gate:
            cmd.append("--no-gate")
        if not tri:
            cmd.append("--no-tri-gate")
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
        case = {"B_lo": lo, "B_hi": hi, "r": r, "gate": gate, "tri": tri, "classes": classes,
                "rc": p.returncode, "cmd": " ".join(["oracle/_ref/solve_617_v1"] + cmd[1:])}
        found = list(SUMMARY.finditer(p.stderr))
        if p.returncode != 0:
            case["error"] = p.stderr.strip().splitlines()[-3:]
        else:
            per = {}
            for m in found:
                c = {"cands": int(m.group(2)), "probes": m.group(3), "exact": int(m.group(4)),
                     "fp_false": int(m.group(5)), "gate_kill": m.group(6)}
                if m.group(7):
                    c.update(tri_skipped=int(m.group(7)), tri_total=int(m.group(8)))
                per[m.group(1)] = c
            case["per_class"] = per
            if "5" in per:   # the class-5 fields at the top level, as the first fixtures had them
                case.update(per["5"])
            case["solutions"] = [l for l in p.stdout.splitlines() if l.startswith("SOLUTION")]
        cases.append(case)
        print(json.dumps(case)[:300])
    os.makedirs(os.path.dirname(out), exist_ok=True)
    with open(out, "w") as f:
        json.dump({"binary": "solve_617_v1 (reference sources, nvcc sm_100a)", "cases": cases}, f,
                  indent=1)
    return 0 if all("error" not in c for c in cases) else 1


if __name__ == "__main__":
    sys.exit(main())
