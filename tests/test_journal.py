"""Restart journal of a campaign (host only, no GPU).

The journal records committed blocks of completed units with their raw hits
and verified solutions.  A reopened journal knows every committed unit and
solution; a block torn by a crash (any prefix of its bytes) is dropped and cut
off, and blocks appended afterwards read back normally.
"""
import ctypes as C
import os

import numpy as np
import pytest

import s615


def units(n, B0=3_200_003, kind=0):
    arr = (s615.Unit * n)()
    for i in range(n):
        arr[i].cls, arr[i].kind, arr[i].B, arr[i].u = 5, kind, B0 + 2 * i, 6 * (i + 1)
        if kind == 1:
            arr[i].base[0], arr[i].base[1], arr[i].base[2] = 2**64 - 1 - i, i, 7
            arr[i].res_e, arr[i].res_d, arr[i].fmax1, arr[i].fmax2, arr[i].lim = 3, 4, 3, 4, 76667
    return arr


def hits(n_units, k):
    h = np.zeros(k, dtype=s615.HIT_DTYPE)
    h["unit"] = np.arange(k) % n_units
    h["d"], h["e"], h["fp"] = 21 + np.arange(k), 44, np.uint64(2**63 + 5)
    return h


def solution(unit, B):
    s = s615.Solution()
    s.unit, s.kind, s.cls, s.B, s.u, s.d, s.e, s.c1, s.c2 = unit, 1, 5, B, 6, 9, 44, 3, 4
    s.a[0], s.a[4], s.gcd = 1, 2**40, 1
    return s


def test_journal_roundtrip_and_torn_tail(tmp_path):
    path = str(tmp_path / "j.log")
    a, b, c = units(4), units(3, 4_000_001, kind=1), units(2, 5_000_001)
    with s615.Journal(path) as j:
        assert j.stats() == (0, 0, 0)
        j.append(a, 4, hits(4, 5), [solution(2, a[2].B)])
        j.append(b, 3)
        assert j.has(a[3]) and j.has(b[0]) and not j.has(c[0])
    with s615.Journal(path) as j:
        assert j.stats() == (7, 5, 1)
        got = j.units()
        assert [(u.B, u.u, u.kind, u.base[0]) for u in got] == \
            [(u.B, u.u, u.kind, u.base[0]) for u in list(a) + list(b)]
        (s,) = j.solutions()
        assert (s.unit, s.B, s.a[4], s.gcd) == (2, a[2].B, 2**40, 1)
        # a unit that differs in any field is not the committed one
        other = units(1, a[0].B)[0]
        other.u += 6
        assert not j.has(other)
    good = os.path.getsize(path)
    with s615.Journal(path) as j:
        j.append(c, 2, hits(2, 3))
    full = open(path, "rb").read()
    # every torn prefix of the last block reads as the two committed blocks
    for cut in range(good, len(full), 7):
        with open(path, "wb") as f:
            f.write(full[:cut])
        with s615.Journal(path) as j:
            assert j.stats() == (7, 5, 1)
            assert not j.has(c[1])
        assert os.path.getsize(path) == good
    # a corrupted committed block ends what is read (and is cut off)
    bad = bytearray(full)
    bad[good + 10] ^= 0x01
    with open(path, "wb") as f:
        f.write(bytes(bad))
    with s615.Journal(path) as j:
        assert j.stats() == (7, 5, 1)
        j.append(c, 2)
    with s615.Journal(path) as j:
        assert j.stats() == (9, 5, 1) and j.has(c[1])


def test_journal_rejects_out_of_range_indices(tmp_path):
    with s615.Journal(str(tmp_path / "j.log")) as j:
        with pytest.raises(s615.S615Error):
            j.append(units(2), 2, hits(3, 3))      # hit unit index 2 >= 2 units
        with pytest.raises(s615.S615Error):
            j.append(units(1), 1, None, [solution(1, 7)])
        assert j.stats() == (0, 0, 0)
