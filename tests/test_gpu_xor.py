"""Device xor filter: query parity and the device builder (GPU)."""
import numpy as np
import pytest

import orc
import s615

pytestmark = pytest.mark.gpu


def pair_keys(N):
    p6 = [pow(x, 6, 2**64) for x in range(N + 1)]
    return np.array([(p6[i] + p6[j]) % 2**64 for i in range(1, N + 1) for j in range(i, N + 1)],
                    dtype=np.uint64)


def random_keys(n, seed):
    rng = np.random.RandomState(seed)
    p = rng.randint(0, 2**32, size=(n, 2), dtype=np.uint64)
    return (p[:, 0] << np.uint64(32)) | p[:, 1]


@pytest.mark.parametrize("r", [16, 20, 48])
@pytest.mark.parametrize("layout", [s615.LAYOUT_WIDE, s615.LAYOUT_PACKED])
def test_query_parity_on_reference_table(engine, oracle_table, r, layout):
    # the oracle table's bytes equal the reference builder's (test_oracle.py)
    t, path = oracle_table(715, r)
    tid = engine.load_table(path, 715, layout)
    try:
        keys = pair_keys(715)
        assert engine.query(tid, keys).all()                  # FN = 0
        probe = np.concatenate([random_keys(1_000_000, r), keys[::7] + np.uint64(1)])
        np.testing.assert_array_equal(engine.query(tid, probe), t.query(probe))
    finally:
        engine.free_table(tid)


def test_load_refuses_wrong_N_and_bad_file(engine, oracle_table, tmp_path):
    _, path = oracle_table(300, 48)
    with pytest.raises(s615.S615Error) as ei:
        engine.load_table(path, 301)
    assert ei.value.status == -4
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"\0" * 64)
    with pytest.raises(s615.S615Error) as ei:
        engine.load_table(str(bad), 0)
    assert ei.value.status == -3
    with pytest.raises(s615.S615Error) as ei:
        engine.load_table(str(tmp_path / "missing.bin"), 0)
    assert ei.value.status == -2


@pytest.mark.parametrize("N,r", [(300, 16), (300, 48), (715, 16), (715, 48), (1000, 20)])
def test_device_build_matches_reference_header(engine, golden, oracle_table, tmp_path, N, r):
    tid = engine.build_table(N, r)
    try:
        h = engine.table_info(tid).hdr
        g = golden["xor_build_save"][f"{N}_{r}"]
        assert (h.magic, h.version, h.kind, h.r, h.N) == (g["magic"], g["version"], g["kind"], r, N)
        assert (h.n_keys, h.m_cells, h.mix_seed) == (g["n_keys"], g["m_cells"], g["mix_seed"])
        keys = pair_keys(N)
        assert engine.query(tid, keys).all()
        # the saved file loads in the reference-format reader and answers the same
        path = str(tmp_path / "dev.bin")
        engine.save_table(tid, path)
        ot = orc.Table.load(path, N)
        assert ot.header.m_cells == h.m_cells
        assert ot.query(keys).all()
        probe = random_keys(500_000, N + r)
        np.testing.assert_array_equal(ot.query(probe), engine.query(tid, probe))
        assert 0 <= ot.fpr_smoke() <= 16
        # reload through the engine: same answers
        tid2 = engine.load_table(path, N)
        np.testing.assert_array_equal(engine.query(tid2, probe), engine.query(tid, probe))
        engine.free_table(tid2)
    finally:
        engine.free_table(tid)


def test_device_build_structural_duplicates(engine):
    # i^6 mod 2^64 collides for 2-adically large i (every multiple of 2048 maps
    # to 0): the unique-key count must equal the reference's sort+unique count
    N = 5000
    keys = pair_keys(N)
    n_unique = np.unique(keys).size
    assert n_unique < keys.size
    tid = engine.build_table(N, 16)
    try:
        h = engine.table_info(tid).hdr
        assert h.n_keys == n_unique
        assert h.m_cells == orc.lib().orc_capacity_for(n_unique)
        assert engine.query(tid, keys).all()
    finally:
        engine.free_table(tid)


def test_build_keys_dedup_tiny_and_retry(engine):
    # xor_filter_test.cpp:44-53, 89-96, 162-184
    tid = engine.build_table_keys([7, 7, 8, 8, 8, 9], 20)
    assert engine.table_info(tid).hdr.n_keys == 3
    assert engine.query(tid, [7, 8, 9]).all()
    engine.free_table(tid)
    tiny = [1, 42, 999, 123456789, 0xDEADBEEFCAFE]
    tid = engine.build_table_keys(tiny, 16)
    assert engine.query(tid, tiny).all()
    engine.query(tid, [0x1111222233334444])
    engine.free_table(tid)
    seq = [0xDEADBEEF00000000 + i for i in range(5000)]
    tid = None
    for outer in range(8):
        try:
            tid = engine.build_table_keys(seq, 16, 0x615615615615615 + outer * 0x9E3779B97F4A7C15)
            break
        except s615.S615Error as e:
            assert e.status == -10
    assert tid is not None
    assert engine.table_info(tid).hdr.n_keys == 5000
    assert engine.query(tid, seq).all()
    engine.free_table(tid)


@pytest.mark.parametrize("keys_n", [10_000, 100_000])
def test_build_keys_matches_oracle_seed_outcome(engine, keys_n):
    # same key set and seed -> same header (n, m, seed), FN = 0 on both
    rng = np.random.RandomState(keys_n)
    keys = random_keys(keys_n, keys_n)
    ot = orc.Table.build_keys(keys, 16)
    tid = engine.build_table_keys(keys, 16)
    h, oh = engine.table_info(tid).hdr, ot.header
    assert (h.n_keys, h.m_cells, h.mix_seed) == (oh.n_keys, oh.m_cells, oh.mix_seed)
    assert engine.query(tid, keys).all()
    engine.free_table(tid)


def test_device_build_past_u32_cells(engine):
    # N = 84,000 gives m > 2^32 cells: the peel lists hold offsets within a
    # third of the table (block < 2^32) and the cell words' key indices reach
    # past 2^31.  No false negative on a sample of pair keys, and the
    # false-positive rate at r = 20 within four binomial standard deviations.
    N, r = 84000, 20
    tid = engine.build_table(N, r)
    try:
        h = engine.table_info(tid).hdr
        assert h.m_cells > 2**32
        rng = np.random.RandomState(84)
        i = rng.randint(1, N + 1, size=2_000_000).astype(np.uint64)
        j = rng.randint(1, N + 1, size=2_000_000).astype(np.uint64)
        p6 = lambda x: x * x * x * x * x * x   # mod 2^64 in uint64 arithmetic
        keys = p6(i) + p6(j)
        assert engine.query(tid, keys).all()
        n = 50_000_000
        fp = int(engine.query(tid, orc.mt64(0xF15EED + h.n_keys, n)).sum())
        mu, sd = n * 2.0**-r, (n * 2.0**-r * (1 - 2.0**-r)) ** 0.5
        assert abs(fp - mu) <= 4 * sd, (fp, mu, sd)
    finally:
        engine.free_table(tid)


def test_device_build_same_bytes_under_a_tight_budget(engine):
    # The builder picks its form by the HBM it may use: by default the binned
    # incidence and the peel lists with each claimed key's index and hash; with
    # a 400 MB budget (N = 3,000: ~110 MB of build buffers) the incidence adds
    # straight into the cell words and the peel keeps only the claimed cells;
    # with 100 MB there is no room for the claimed-cell list (22.5 MB) and
    # every round scans all cells.  The rounds are the same, so the cells are
    # too, byte for byte.
    N, r = 3000, 20
    tid = engine.build_table(N, r)
    try:
        h0, p0 = engine.export_table(tid)
    finally:
        engine.free_table(tid)
    for budget in (400 << 20, 100 << 20):
        with s615.Engine(0, hbm_budget=budget) as tight:
            t2 = tight.build_table(N, r)
            h1, p1 = tight.export_table(t2)
        assert bytes(h0) == bytes(h1), budget
        np.testing.assert_array_equal(p0, p1)
