"""The (6,1,7) Branch-A class-5 oracle (CPU): candidate rule, recovery of the
reference's known identities, plants and the window rules, pinned against
the reference's own GPU binary where its fixture is present.

The oracle restates gen_class_cands(cls=5), k_find4_cls5 and verify_hit of
solve_617_v1.cu (:885-906, :563-657, :1040-1110).
"""
import json
import math
import os

import numpy as np
import pytest

import orc

M42 = 42**6
HERE = os.path.dirname(os.path.abspath(__file__))
REF617 = os.path.join(HERE, "golden", "ref617.json")


def eligible617(B):
    """Branch-A B values of the campaign loop (solve_617_v1.cu:1910-1913)."""
    return B >= 11 and B % 2 == 1 and B % 3 != 0 and B % 7 != 0


def test_candidates_follow_the_class_rule():
    for B in (54347, 100003, 233341):
        arr, n = orc.cands617(B)
        assert n > 0
        seen = set()
        for i in range(n):
            C = arr[i]
            base = C.base[0] | (C.base[1] << 64)
            assert C.B == B and C.u % 14 == 0 and C.w % 6 == 0 and C.u < B and C.w < B
            assert base == B**6 - C.u**6 - C.w**6 > 0
            assert pow(C.u, 6, 729) == pow(B, 6, 729)
            assert pow(C.w, 6, 7**6) == pow(B, 6, 7**6)
            assert C.lim == (B - 1) // 42 and C.fmax1 == (B - 1) // 21 and C.mod1 == 64
            res = sorted(C.res[k] for k in range(C.nres1))
            assert res == [r for r in range(64) if math.gcd(r, 2) == 1
                           and pow(21 * r, 6, 64) == pow(B, 6, 64)]
            # every grid row then has 42^6 | base - (21 d)^6
            for r in res[:2]:
                assert (base - (21 * r) ** 6) % M42 == 0
            seen.add((C.u, C.w))
        assert len(seen) == n
        # the anchor sets: u' over 6 classes mod 3^6, v' over 6 classes mod 7^6
        us = {u for u, _ in seen}
        assert all(pow(u // 14, 6, 729) * pow(14, 6, 729) % 729 == pow(B, 6, 729) for u in us)


def one_cand(B, u, w):
    arr, n = orc.cands617(B)
    idx = [i for i in range(n) if arr[i].u == u and arr[i].w == w]
    assert idx, (B, u, w)
    one = (orc.OrcCand617 * 1)()
    one[0] = arr[idx[0]]
    return one


def test_known_identities_recovered(golden):
    # every known identity of this shape with B < 160,000 comes back from its
    # own candidate, exactly once
    known = [k for k in golden["known617_cls5"] if k["B"] < 160000]
    assert len(known) >= 10
    N = max(k["B"] for k in known) // 42   # one table covers every c <= B/42
    t = orc.Table.build_pairs(N, 48)
    for k in known:
        B = k["B"]
        one = one_cand(B, k["u"], k["w"])
        hits, ctr = orc.run617(t, one, 1)
        lines = orc.verify617(one, hits, N)
        want = " ".join(f"a{i + 1}={x}" for i, x in enumerate(k["terms"]))
        assert len([l for l in lines if want in l]) == 1, (B, lines)
        assert ctr[2] == 3 * ctr[0]


def plant_cand(c, d, N):
    """The plant shape of solve_617_v1.cu:1564-1582."""
    base = (21 * d) ** 6 + M42 * sum(x**6 for x in c)
    C = orc.OrcCand617()
    C.base[0], C.base[1] = base % 2**64, base >> 64
    C.B, C.u, C.w, C.lim = 42 * N + 1, 14, 6, N
    C.mod1, C.fmax1, C.nres1 = 64, d, 1
    C.res[0] = d % 64
    return C


def window_reaches(c, N):
    """The reference's windows contain the plant: c4 = max with 3 c4^6 >= T
    and c3 = next with 3 c3^6 >= T - c4^6 (min_c_fix, :430-436)."""
    s = sorted(c)
    T = sum(x**6 for x in s)
    T2 = T - s[3] ** 6
    return 3 * s[3] ** 6 >= T and 3 * s[2] ** 6 >= T2 and s[3] <= N


def test_plants_and_the_window_rule():
    N = 600
    rng = np.random.RandomState(7)
    plants = []
    while len(plants) < 24:
        c = sorted(int(x) for x in rng.choice(np.arange(1, N + 1), 4, replace=False))
        d = int(rng.randint(1, 281))
        plants.append((c, d))
    # four close terms: T > 3 max^6, so the c4 window is empty and the
    # reference (and the oracle) cannot see it
    plants.append(([N - 3, N - 2, N - 1, N], 5))
    arr = (orc.OrcCand617 * len(plants))()
    for i, (c, d) in enumerate(plants):
        arr[i] = plant_cand(c, d, N)
    t = orc.Table.build_pairs(N, 48)
    hits, _ = orc.run617(t, arr, len(plants))
    lines = orc.verify617(arr, hits, N, planted=True)
    got = set()
    for l in lines:
        f = dict(kv.split("=") for kv in l.split()[1:])
        got.add((int(f["cand"]), tuple(sorted(int(f[k]) for k in "abcd"))))
    for i, (c, d) in enumerate(plants):
        assert ((i, tuple(c)) in got) == window_reaches(c, N), (i, c, d)
    assert not window_reaches(plants[-1][0], N)
    assert sum(window_reaches(c, N) for c, _ in plants) >= 16


def test_gate_switches_and_tiles():
    B = 54347
    arr, n = orc.cands617(B)
    t = orc.Table.build_pairs(B // 42, 16)
    h1, c1 = orc.run617(t, arr, n)
    h2, c2 = orc.run617(t, arr, n, use_gate=False)
    h3, c3 = orc.run617(t, arr, n, use_tri=False)
    # the gates are sound: every hit of the gated run is a hit without them
    key = lambda h: set(zip(h["cand"], h["c"], h["d"], h["e"], h["fp"]))
    assert key(h1) <= key(h2) and key(h1) <= key(h3)
    assert c2[1] == 0 and c2[0] > c1[0]
    assert c3[3] == c3[4] == 0 and c1[3] > c1[4] > 0
    # windows here are < 2048 wide: the reference's c4 tiles change nothing
    h4, c4 = orc.run617(t, arr, n, zmax=5)
    assert c4 == c1 and key(h4) == key(h1)


def test_tiles_repeat_wide_windows():
    # B = 600,001: c4 windows exceed 2048, so the reference's tile z >= 1
    # re-walks c4 >= lo4 + 2048 z (gpu_run, :960-968)
    B = 600001
    arr, n = orc.cands617(B)
    sel = [i for i in range(n) if arr[i].u == 181244]
    one = (orc.OrcCand617 * len(sel))()
    for k, i in enumerate(sel):
        one[k] = arr[i]
    t = orc.Table.build_pairs(300, 16)   # every c4 of this anchor fails the tri gate
    _, a = orc.run617(t, one, len(sel))
    _, b = orc.run617(t, one, len(sel), zmax=(B // 42 + 2047) // 2048)
    assert b[3] > a[3] > 0 and a[3] == a[4] and b[3] == b[4]


def oracle_case(case):
    """The oracle over one recorded reference run: per class the summary
    fields, plus all SOLUTION lines."""
    lo, hi, r = case["B_lo"], case["B_hi"], case["r"]
    N = hi // 42
    t = orc.Table.build_pairs(N, r)
    Bs = [B for B in range(lo, hi + 1) if eligible617(B)]
    per, lines = {}, []
    for cls in case.get("classes", "5"):
        st = [0, 0]
        if cls == "5":
            parts = [orc.cands617(B) for B in Bs]
            arr, n = orc.concat617([p for p in parts if p[1]])
            if not n:
                continue
            zmax = max(1, min(32, (max(arr[i].lim for i in range(n)) + 2047) // 2048))
            hits, c = orc.run617(t, arr, n, use_gate=case["gate"], use_tri=case["tri"], zmax=zmax)
            lines += orc.verify617(arr, hits, N, stats=st)
        else:
            parts = [orc.jobs617(B, int(cls)) for B in Bs]
            arr, n = orc.concat_jobs617([p for p in parts if p[1]])
            if not n:
                continue
            span = max(arr[i].hi - arr[i].lo + 1 for i in range(n))
            ymax = max(1, min(32, (span + 2047) // 2048))
            hits, c = orc.run617_find4(t, arr, n, use_gate=case["gate"], use_tri=case["tri"], ymax=ymax)
            lines += orc.verify617_find4(arr, hits, N, stats=st)
        rec = {"cands": n, "probes": "%.4e" % c[2], "exact": st[0], "fp_false": st[1],
               "gate_kill": "%.2f" % (100.0 * c[1] / max(1, c[1] + c[0]))}
        if case["tri"]:
            # every one of the 32 threads of the warp that walks a c4 counts it
            # (++l_tri_tot / ++l_tri_skip run per thread, solve_617_v1.cu:527-536, 604-614)
            rec.update(tri_skipped=32 * c[4], tri_total=32 * c[3])
        per[cls] = rec
    return per, lines


@pytest.mark.skipif(not os.path.exists(REF617), reason="reference GPU fixture not generated")
def test_counters_equal_reference_binary():
    """Counts printed by the reference's own solve_617_v1 (run on a GPU by
    tests/golden/gen_ref617.py) against the oracle on the same B range."""
    with open(REF617) as f:
        ref = json.load(f)
    cases = [c for c in ref["cases"] if "error" not in c]
    assert cases
    for case in cases:
        per, lines = oracle_case(case)
        want = case.get("per_class", {"5": {k: case[k] for k in ("cands", "probes", "exact", "fp_false",
                                                                  "gate_kill", "tri_skipped", "tri_total")
                                            if k in case}})
        assert per == want, case["cmd"]
        assert sorted(lines) == sorted(case["solutions"]), case["cmd"]
