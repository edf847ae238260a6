"""False-positive rate of device-built tables within binomial bounds (GPU).

The reference's FPR test (spike/ribbon/xor_filter_test.cpp:55-87) draws
non-keys from std::mt19937_64 seeded with 0xF15EED + n (n = the number of
keys), skips drawn values that are keys, and compares the "maybe" rate with
2^-r.  Here the tables are the search's own pair tables (keys i^6 + j^6 mod
2^64, 1 <= i <= j <= N) built on the device, the same non-key stream comes
from the oracle, and the count of false positives must lie within four
binomial standard deviations of n * 2^-r.

For r = 48 no sample reaches a false positive (2^-48), so the test reads the
device-built table back and checks the filter's residue instead:
cell(i0) ^ cell(i1) ^ cell(i2) ^ fingerprint is uniform over 48 bits for a
non-key, and the rate of residues with their low 16 bits zero must be 2^-16
within the same bounds (and no residue may be zero).
"""
import math

import numpy as np
import pytest

import orc

pytestmark = pytest.mark.gpu

SIGMAS = 4.0


def pair_keys(N):
    p6 = np.array([pow(x, 6, 2**64) for x in range(N + 1)], dtype=np.uint64)
    i, j = np.triu_indices(N, 0)
    return np.unique(p6[i + 1] + p6[j + 1])


def within(count, n, p):
    mu = n * p
    sd = math.sqrt(n * p * (1 - p))
    return abs(count - mu) <= SIGMAS * sd, (count, mu, sd)


def non_keys(n_keys, n, keyset=None):
    """The reference test's stream, keys removed when the key set is given."""
    draws = orc.mt64(0xF15EED + n_keys, n)
    if keyset is not None:
        draws = draws[~np.isin(draws, keyset)]
    return draws


# (N, r, non-keys drawn): about 150 expected false positives at r = 16 and
# 95 at r = 20.  For N = 24,000 (2.9e8 keys) the draws are not filtered: a
# uniform 64-bit draw is a key with probability 1.6e-11, so 1e8 draws hold
# a key with probability below 0.002.
CASES = [(2000, 16, 10_000_000), (2000, 20, 100_000_000),
         (24000, 16, 10_000_000), (24000, 20, 100_000_000)]


@pytest.mark.parametrize("N,r,n", CASES)
def test_fpr_binomial(engine, N, r, n):
    tid = engine.build_table(N, r)
    try:
        h = engine.table_info(tid).hdr
        keyset = pair_keys(N) if N <= 2000 else None
        if keyset is not None:
            assert h.n_keys == keyset.size
            assert engine.query(tid, keyset).all()          # no false negative
        draws = non_keys(h.n_keys, n, keyset)
        fp = int(engine.query(tid, draws).sum())
        ok, why = within(fp, draws.size, 2.0 ** -r)
        assert ok, why
    finally:
        engine.free_table(tid)


@pytest.mark.parametrize("N", [2000, 24000])
def test_r48_residue_uniform(engine, N):
    tid = engine.build_table(N, 48)
    try:
        hb, pk = engine.export_table(tid)
        ot = orc.Table.from_memory(hb, pk)
        del pk
        n = 20_000_000
        draws = non_keys(ot.header.n_keys, n, pair_keys(N) if N <= 2000 else None)
        res = ot.residue(draws)
        assert int((res == 0).sum()) == 0                    # 2^-48 per draw
        ok, why = within(int(((res & np.uint64(0xFFFF)) == 0).sum()), draws.size, 2.0 ** -16)
        assert ok, why
        # the device query agrees with the residue on every draw
        q = engine.query(tid, draws[:2_000_000])
        np.testing.assert_array_equal(q, (res[:2_000_000] == 0).astype(q.dtype))
    finally:
        engine.free_table(tid)
