"""The CPU oracle pinned against the reference's golden vectors (no GPU)."""
import hashlib
import math
import os

import numpy as np
import pytest

import orc


def test_pow6_kats(golden):
    # fourcore_cls5_gpu_v4.cu:192-201 (pow6_192 vs GMP at these x)
    for x, v in golden["pow6"].items():
        assert orc.pow6_192(int(x)) == int(v)


def test_peel_sample_T_and_funnel(golden):
    # fourcore_cls5_gpu_v4.cu:203-229: funnel fingerprint == T mod 2^64
    s = golden["peel_sample"]
    import ctypes as C
    T = np.zeros(2, dtype=np.uint64)
    assert orc.lib().orc_T_peel2(s["B"], s["u"], s["d"], s["e"], orc._ptr(T)) == 1
    assert int(T[0]) | (int(T[1]) << 64) == int(s["T"])
    U = orc.pack_unit(s["B"], s["u"])
    ok = C.c_int(0)
    fp = orc.lib().orc_funnel_fp(C.byref(U), s["d"], s["e"], C.byref(ok))
    assert ok.value == 1 and fp == int(s["fp"])


def test_past_wall_divisible_point():
    # fourcore_cls5_gpu_v4.cu:231-255: B=2353975,u=85710 has a divisible (d,e)
    B, u = 2353975, 85710
    U = orc.pack_unit(B, u)
    assert U is not None and U.nres1 == 6 and U.nres2 == 4
    e, d = U.res[0], U.res[U.nres1]
    R = B**6 - u**6 - (14 * e) ** 6 - (21 * d) ** 6
    assert R > 0 and R % 42**6 == 0
    assert (B**6).bit_length() > 127   # past the signed-i128 wall


def test_seed_counts():
    # fourcore_hunt_v3.cpp:49-66: 144/24/36/6/6 at B=100003
    assert [orc.seed_count(100003, c) for c in range(1, 6)] == [144, 24, 36, 6, 6]


def test_gate_cardinalities(golden):
    g504, g247 = orc.gate_tables()
    assert int(g504.sum()) == golden["gate"]["504"] == 27
    assert int(g247.sum()) == golden["gate"]["247"] == 50


def test_config1_unit_count_matches_reference_cpu_path(golden):
    # solve_516_v2 1000 30000 5 (the reference CPU path) tests 725 units
    n = 0
    for B in range(1000, 30001):
        if math.gcd(B, 42) == 1:
            n += len(orc.unit_candidates(B, 5))
    assert n == golden["solve_516_v2_1000_30000_cls5"]["units"] == 725
    assert golden["solve_516_v2_1000_30000_cls5"]["solutions"] == []


def test_unit_rule_other_classes(golden):
    per = golden["solve_516_v2_1000_5000_units_by_class"]
    for c in "1234":
        n = sum(len(orc.unit_candidates(B, int(c))) for B in range(1000, 5001) if math.gcd(B, 42) == 1)
        assert n == per[c]


@pytest.mark.parametrize("N,r", [(300, 16), (300, 48), (715, 16), (715, 20), (715, 48),
                                 (1000, 48)])
def test_oracle_builder_bytes_equal_reference(golden, oracle_table, N, r):
    # byte-identical to xor_build_save (the reference's host builder)
    t, path = oracle_table(N, r)
    g = golden["xor_build_save"][f"{N}_{r}"]
    data = open(path, "rb").read()
    assert len(data) == g["bytes"]
    assert hashlib.sha256(data).hexdigest() == g["sha256"]
    h = t.header
    assert (h.n_keys, h.m_cells, h.mix_seed, h.N, h.r) == (g["n_keys"], g["m_cells"], g["mix_seed"], N, r)


def test_oracle_xor_fn_zero_and_fpr(oracle_table):
    # xor_filter_test.cpp:55-87 shape: FN = 0, FPR within 8x of 2^-r
    t, _ = oracle_table(715, 16)
    p6 = [x**6 % 2**64 for x in range(716)]
    keys = np.array([(p6[i] + p6[j]) % 2**64 for i in range(1, 716) for j in range(i, 716)],
                    dtype=np.uint64)
    assert t.query(keys).all()
    rng = np.random.RandomState(11)
    p2 = rng.randint(0, 2**32, size=(2_000_000, 2), dtype=np.uint64)
    probe = (p2[:, 0] << np.uint64(32)) | p2[:, 1]
    probe = probe[~np.isin(probe, keys)]
    rate = t.query(probe).mean()
    assert 2**-16 / 8 <= rate <= 2**-16 * 8


def test_oracle_dedup_and_tiny():
    # xor_filter_test.cpp:44-53,89-96
    t = orc.Table.build_keys([7, 7, 8, 8, 8, 9], 20)
    assert t.header.n_keys == 3
    assert t.query([7, 8, 9]).all()
    t = orc.Table.build_keys([1, 42, 999, 123456789, 0xdeadbeefcafe], 16)
    assert t.query([1, 42, 999, 123456789, 0xdeadbeefcafe]).all()


def test_oracle_save_load_roundtrip(oracle_table, tmp_path):
    # xor_store_io_test.cpp:61-102
    t, path = oracle_table(300, 48)
    t2 = orc.Table.load(path, 300)
    assert t2.bytes() == t.bytes()
    with pytest.raises(RuntimeError):
        orc.Table.load(path, 301)
    assert 0 <= t2.fpr_smoke() <= 16


def test_oracle_plant_recovered(oracle_table):
    # solve_516_v3.cu:1149-1170 plant shape through the peel + verify
    t, _ = oracle_table(715, 48)
    e, d, c1, c2 = 280, 190, 13, 600
    base = (14 * e) ** 6 + (21 * d) ** 6 + 42**6 * (c1**6 + c2**6)
    U = orc.plant_unit(base, e, d, lim=715)
    arr = orc.units_array([U])
    hits, ctr = orc.cls5_run(t, arr, 1)
    assert ((hits["d"] == d) & (hits["e"] == e) & (hits["fp"] == (c1**6 + c2**6))).any()
    lines = orc.cls5_verify(arr, hits, 715)
    assert f"PLANT unit=0 d={d} e={e} c1={c1} c2={c2}" in lines


def test_oracle_counters_small_unit():
    # calls counts the full in-range rectangle; probes <= R>0 points
    import orc as o
    t = o.Table.build_pairs(100, 16)
    B = next(b for b in range(4001, 9000) if math.gcd(b, 42) == 1 and o.unit_candidates(b, 5))
    U = o.pack_unit(B, o.unit_candidates(B, 5)[0])
    hits, (calls, gated, probes) = o.cls5_run(t, o.units_array([U]), 1)
    ne = sum(len(range(U.res[i], U.fmax1 + 1, 729)) for i in range(U.nres1))
    nd = sum(len(range(U.res[U.nres1 + i], U.fmax2 + 1, 64)) for i in range(U.nres2))
    assert calls == ne * nd
    assert probes + gated <= calls


def test_residue_and_mt64_helpers():
    # the FPR tests' helpers: std::mt19937_64's 10,000th draw from the default
    # seed is the C++ standard's check value, and a table's residue
    # (cell ^ cell ^ cell ^ fingerprint) is zero exactly where the query says "maybe"
    assert int(orc.mt64(5489, 10000)[-1]) == 9981545732273789042
    t = orc.Table.build_pairs(300, 8)
    keys = np.concatenate([orc.mt64(7, 200_000), np.array([pow(3, 6, 2**64) + pow(5, 6, 2**64)],
                                                           dtype=np.uint64)])
    res = t.residue(keys)
    np.testing.assert_array_equal((res == 0).astype(np.uint8), t.query(keys))
    assert res[-1] == 0 and 0 < int((res == 0).sum()) < 200_000 // 64
