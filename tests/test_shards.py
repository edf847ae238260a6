"""Pair-space shards in the oracle (spike/ribbon/shard.hpp:19-24).

shard_of_key(k) = mix64(k + seed) % S; shard s of a set holds exactly the pair
keys routed to it, and the set's query asks only the key's own shard.
"""
import numpy as np
import pytest

import orc

M64 = 2**64 - 1


def mix64(x):   # spike/ribbon/mix64.hpp:13-20
    x ^= x >> 33
    x = (x * 0xFF51AFD7ED558CCD) & M64
    x ^= x >> 33
    x = (x * 0xC4CEB9FE1A85EC53) & M64
    x ^= x >> 33
    return x


def pair_keys(N):
    return np.array(sorted({(i**6 + j**6) & M64 for i in range(1, N + 1) for j in range(i, N + 1)}),
                    dtype=np.uint64)


def test_shard_rule_is_mix_then_mod():
    rng = np.random.RandomState(3)
    for k in [0, 1, M64, 2**63] + [int(x) for x in rng.randint(0, 2**63, 200, dtype=np.int64)]:
        for S in (2, 3, 8, 64):
            assert orc.shard_of(k, S) == mix64((k + orc.SHARD_SEED) & M64) % S


@pytest.mark.parametrize("S", [2, 5])
def test_shards_partition_the_key_set(S):
    N, r = 400, 20
    parts = [orc.Table.build_pairs_shard(N, r, S, s) for s in range(S)]
    keys = pair_keys(N)
    owner = np.array([orc.shard_of(int(k), S) for k in keys])
    for s, p in enumerate(parts):
        h = p.header
        assert (h.shard_count, h.shard_index, h.shard_mode, h.N, h.r) == (S, s, 0, N, r)
        assert h.n_keys == int((owner == s).sum())
        assert p.query(keys[owner == s]).all()          # every key of the shard: no false negative
    ts = orc.Table.shard_set(parts)
    assert ts.header.n_keys == len(keys) == orc.Table.build_pairs(N, r).header.n_keys
    assert ts.query(keys).all()
    assert 0 <= ts.fpr_smoke() <= 16
    rng = np.random.RandomState(S)
    rk = rng.randint(0, 2**63, 1 << 20, dtype=np.int64).astype(np.uint64)
    fp = int(ts.query(rk).sum())
    assert fp <= 8 * (1 << 20) / 2**r + 4                 # FPR within 8x of 2^-r
