#!/usr/bin/env python3
"""Regenerate tests/golden/golden.json.

Run in a container that has the reference tree (read only), given as the
first argument or in S615_REFERENCE.  It builds the reference's own buildable programs into oracle/_ref
(oracle/Makefile `ref`), runs them, and records their outputs next to exact
Python-integer values for the known-answer checks the reference's self-tests
make.  The GPU box never runs this script; tests read the JSON only.

  python tests/golden/gen_golden.py REFERENCE_DIR
"""
import hashlib
import json
import math
import os
import re
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("S615_REFERENCE", "")
OUT = os.path.join(ROOT, "tests", "golden", "golden.json")


def run(cmd, **kw):
    return subprocess.run(cmd, capture_output=True, text=True, timeout=600, **kw)


def main():
    if not os.path.isdir(REF):
        sys.exit("usage: gen_golden.py REFERENCE_DIR (or set S615_REFERENCE)")
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={REF}"], check=True,
                   stdout=subprocess.DEVNULL)
    g = {}

    # -- exact powers (fourcore_cls5_gpu_v4.cu:192-201 checks these x against GMP)
    g["pow6"] = {str(x): str(x**6) for x in (1, 42, 100003, 2353975, 2752470)}
    # -- peel sample (B=100003,u=17646,d=9,e=44): T = R/42^6 and its funnel key
    B, u, d, e = 100003, 17646, 9, 44
    R = B**6 - u**6 - (21 * d) ** 6 - (14 * e) ** 6
    assert R % 42**6 == 0
    g["peel_sample"] = {"B": B, "u": u, "d": d, "e": e, "T": str(R // 42**6),
                        "fp": str((R // 42**6) % 2**64)}
    # -- B^6 bit lengths (wall checks of fourcore_hunt_v3.cpp:67-79, cls5_gpu_v4.cu:257-260)
    g["bits"] = {str(b): (b**6).bit_length() for b in (2353973, 2353974, 2752470)}

    # -- reference CPU path: solve_516_v2 on config 1's window, class 5 only
    r = run([os.path.join(REF_BIN, "solve_516_v2"), "1000", "30000", "5"],
            env=dict(os.environ, OMP_NUM_THREADS="8"))
    m = re.search(r"unit candidates tested: (\d+)", r.stderr)
    g["solve_516_v2_1000_30000_cls5"] = {
        "units": int(m.group(1)),
        "solutions": [l for l in r.stdout.splitlines() if l.startswith("SOLUTION")],
        "eligible_B": int(re.search(r"eligible B \(odd, gcd\(B,21\)=1\): (\d+)", r.stderr).group(1)),
    }
    # the same window for every class (unit-rule pin for classes 1-4)
    r = run([os.path.join(REF_BIN, "solve_516_v2"), "1000", "5000", "all"],
            env=dict(os.environ, OMP_NUM_THREADS="8"))
    g["solve_516_v2_1000_5000_all_units"] = int(re.search(r"unit candidates tested: (\d+)", r.stderr).group(1))
    per = {}
    for c in "1234":
        r = run([os.path.join(REF_BIN, "solve_516_v2"), "1000", "5000", c],
                env=dict(os.environ, OMP_NUM_THREADS="8"))
        per[c] = int(re.search(r"unit candidates tested: (\d+)", r.stderr).group(1))
    g["solve_516_v2_1000_5000_units_by_class"] = per

    # -- reference host xor builder: header fields and sha256 of the file bytes
    tabs = {}
    with tempfile.TemporaryDirectory() as td:
        for N in (300, 715, 1000):
            for rb in (16, 20, 48):
                p = os.path.join(td, f"x{N}_{rb}.bin")
                rr = run([os.path.join(REF_BIN, "xor_build_save"), "--N", str(N), "--r", str(rb),
                          "--out", p])
                assert rr.returncode == 0, rr.stderr
                data = open(p, "rb").read()
                hdr = data[:64]
                vals = dict(zip(["magic", "version", "kind", "r", "w", "N"],
                                [int.from_bytes(hdr[i:i + 4], "little") for i in range(0, 24, 4)]))
                vals["n_keys"] = int.from_bytes(hdr[24:32], "little")
                vals["m_cells"] = int.from_bytes(hdr[32:40], "little")
                vals["mix_seed"] = int.from_bytes(hdr[40:48], "little")
                vals["sha256"] = hashlib.sha256(data).hexdigest()
                vals["bytes"] = len(data)
                tabs[f"{N}_{rb}"] = vals
    g["xor_build_save"] = tabs

    # -- the reference's own host suites pass here
    suites = {}
    for name in ("xor_filter_test", "xor_store_io_test", "v3_host_logic_test"):
        rr = run([os.path.join(REF_BIN, name)])
        suites[name] = {"rc": rr.returncode,
                        "tail": (rr.stdout + rr.stderr).strip().splitlines()[-1]}
    g["reference_suites"] = suites

    # -- gate cardinalities from the definition (fourcore_find_v4.cu:78-88)
    def pair_sums(q):
        return sorted({(i**6 + j**6) % q for i in range(q) for j in range(i, q)})
    g["gate"] = {"504": len(pair_sums(504)), "247": len(pair_sums(247))}

    # -- triple-sum gate sizes (build_tri_set, solve_617_v1.cu:334-345; its
    #    selftest requires 64 residues mod 504, :1382)
    def tri_sums(q):
        p = {pow(i, 6, q) for i in range(q)}
        p2 = {(a + b) % q for a in p for b in p}
        return sorted({(a + b) % q for a in p2 for b in p})
    g["tri_gate"] = {"504": len(tri_sums(504)), "247": len(tri_sums(247))}

    # -- known (6,1,7) identities of the Branch-A class-5 shape, read from the
    #    reference's 617-solutions-clean.txt: 7 does not divide B, four terms
    #    42c, one term 21d, u = 14u' and w = 6v' (the other two terms)
    known = []
    with open(os.path.join(REF, "617-solutions-clean.txt")) as f:
        for line in f:
            m = re.match(r"\s*(\d+)\s*=\s*([\d\s+]+)\|", line)
            if not m:
                continue
            B = int(m.group(1))
            t = sorted(int(x) for x in m.group(2).split("+"))
            assert sum(x**6 for x in t) == B**6
            if B % 7 == 0:
                continue
            c = [x for x in t if x % 42 == 0]
            d = [x for x in t if x % 21 == 0 and x % 42 != 0]
            u = [x for x in t if x % 14 == 0 and x % 42 != 0]
            w = [x for x in t if x % 6 == 0 and x % 42 != 0]
            if len(c) == 4 and len(d) == 1 and len(u) == 1 and len(w) == 1:
                known.append({"B": B, "terms": t, "u": u[0], "w": w[0], "d": d[0] // 21,
                              "c": [x // 42 for x in c]})
    g["known617_cls5"] = [k for k in known if k["B"] < 200000]

    with open(OUT, "w") as f:
        json.dump(g, f, indent=1, sort_keys=True)
    print("wrote", OUT)


if __name__ == "__main__":
    sys.exit(main())
