"""Host-side checks of the engine library (no GPU calls)."""
import ctypes as C
import math
import os
import re
import subprocess

import numpy as np
import pytest

import orc
import s615

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "s615.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(s615_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = s615.lib()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(s615.SIGNATURES), set(names) ^ set(s615.SIGNATURES)
    out = subprocess.run(["nm", "-D", "--defined-only", s615.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r"\bT (s615_\w+)", out))
    assert set(names) <= exported


def test_struct_layouts_match_header():
    assert C.sizeof(s615.Header) == 64
    assert C.sizeof(s615.Hit) == 32      # reference Hit{u32 x5; u64 fp}
    assert C.sizeof(s615.Unit) == 72
    assert C.sizeof(s615.Counters) == 56
    assert C.sizeof(s615.Solution) == 120
    assert s615.HIT_DTYPE.itemsize == 32


def test_host_selftest():
    # pow6 KATs, gate = CRT product (27/504, 50/247), exact remainder, row identity
    assert s615.lib().s615_selftest_host() == 0


def test_unit_candidates_match_oracle():
    rng = np.random.RandomState(3)
    Bs = [100003, 2353975, 3200003] + [int(b) for b in rng.randint(1000, 5_000_000, size=60)]
    for B in Bs:
        if math.gcd(B, 42) != 1:
            continue
        for cls in (1, 2, 3, 4, 5):
            assert s615.unit_candidates(B, cls) == orc.unit_candidates(B, cls), (B, cls)


def test_617_candidates_match_oracle():
    # s615_617_candidates against the oracle's gen_class_cands(cls=5)
    rng = np.random.RandomState(17)
    Bs = [54347, 400471, 2353973] + [int(b) for b in rng.randint(12, 2_353_973, size=30)]
    for B in Bs:
        if B % 2 == 0 or B % 3 == 0 or B % 7 == 0:
            continue
        arr, n = s615.candidates617(B)
        oarr, on = orc.cands617(B)
        assert n == on, B
        assert [(arr[i].u, arr[i].w) for i in range(n)] == [(oarr[i].u, oarr[i].w) for i in range(on)]
        assert all(arr[i].cls == s615.S615_CLS_617 and arr[i].B == B for i in range(n))
    with pytest.raises(s615.S615Error):
        s615.candidates617(2353975)


def test_617_find4_jobs_match_oracle():
    # s615_617_jobs against the oracle's find5 expansion (classes 1-4): same
    # jobs in the same order, c4 window [lo, hi] in fmax2 / fmax1
    for B, cls in [(34781, 4), (38191, 4), (39779, 3), (34763, 1), (34763, 2), (38111, 3)]:
        arr, n = s615.jobs617(B, cls)
        oarr, on = orc.jobs617(B, cls)
        assert n == on, (B, cls)
        for i in range(n):
            a, o = arr[i], oarr[i]
            assert a.cls == s615.S615_CLS_617_FIND4 and a.B == B == o.B
            assert (a.u, a.w, a.res_e, a.res_d, a.lim) == (o.u, o.w, o.c5, cls, o.lim), (B, cls, i)
            assert (a.fmax2, a.fmax1) == (o.lo, o.hi), (B, cls, i)
            assert (a.base[0], a.base[1], a.base[2]) == (o.Q4[0], o.Q4[1], 0), (B, cls, i)
    with pytest.raises(s615.S615Error):
        s615.jobs617(34781, 5)


def test_open_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(s615.S615Error) as ei:
        s615.Engine(0)
    assert ei.value.status == -7


def test_cli_built_and_selftest():
    cli = os.path.join(ROOT, "six-one-five_b200", "bin", "s615_cls5")
    assert os.path.exists(cli)
    r = subprocess.run([cli, "--selftest-host"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PASS" in r.stdout


def test_band_unit_count_equals_reference_campaign():
    # the reference's 4.5M -> 5.0M class-5 campaign ran units=5765343 (its README's
    # coverage table); both band ends are even, so the count is the same for
    # open or closed bounds.  The engine's host rule and the oracle's both give it.
    import workloads as W
    assert len(W.cls5_units(4_500_000, 5_000_000)) == 5_765_343
    assert sum(len(orc.unit_candidates(B, 5)) for B in range(4_500_001, 5_000_000, 2)
               if B % 3 and B % 7) == 5_765_343
