"""s615_cls5_run_noalloc against s615_cls5_run (GPU).

The no-allocation entry point serves callers that cannot allocate device
memory when they search (their HBM is owned by another allocator, or
cudaMalloc's latency and implicit synchronisation are not acceptable on their
thread).  It must return exactly what the allocating entry point returns:
the same raw hits (as a multiset; hit order is not defined) and the same
calls / gated / probes / pos counters -- integer results, so the tolerance is
zero.  It is called twice in a row because all calls share one fixed device
array that keeps the previous call's contents.

This file is collected last so that a stopping run has already run every
other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import orc
import s615
import workloads as W

pytestmark = pytest.mark.gpu

N = 715


def sorted_hits(h):
    a = np.stack([h["unit"].astype(np.uint64), h["d"].astype(np.uint64), h["e"].astype(np.uint64),
                  h["fp"]], axis=1)
    return a[np.lexsort(a.T[::-1])] if a.size else a.reshape(0, 4)


def run_noalloc(eng, tid, arr, n, cap=1 << 14):
    hits = (s615.Hit * cap)()
    nh = C.c_size_t(0)
    ctr = s615.Counters()
    st = s615.lib().s615_cls5_run_noalloc(eng._ctx, tid, C.cast(arr, C.c_void_p), n, 0,
                                         C.cast(hits, C.c_void_p), cap, C.byref(nh), C.byref(ctr))
    return st, s615.hits_to_array(hits, min(nh.value, cap)), ctr


def test_noalloc_matches_allocating_entry_point(engine, tmp_path):
    t = orc.Table.build_pairs(N, 16)
    path = str(tmp_path / "t.bin")
    t.save(path)
    tid = engine.load_table(path, N)
    try:
        units = W.cls5_units(1000, 30000)
        plants = W.plants(8, 0, 1000, 30000, N)
        arr, n = W.unit_array(units, plants, N)
        ref_hits, ref_ctr = engine.cls5_run(tid, arr, n)
        assert len(ref_hits) > 0
        for _ in range(2):   # twice in a row: the shared array must not leak state
            st, hits, ctr = run_noalloc(engine, tid, arr, n)
            assert st == 0
            assert (ctr.calls, ctr.gated, ctr.probes, ctr.pos, ctr.hits) == (
                ref_ctr.calls, ref_ctr.gated, ref_ctr.probes, ref_ctr.pos, ref_ctr.hits)
            np.testing.assert_array_equal(sorted_hits(hits), sorted_hits(ref_hits))
        # a smaller second batch right after: counters restart from zero
        arr2, n2 = W.unit_array(units[:100], plants[:2], N)
        ref2, rc2 = engine.cls5_run(tid, arr2, n2)
        st, h2, c2 = run_noalloc(engine, tid, arr2, n2)
        assert st == 0 and (c2.calls, c2.probes, c2.hits) == (rc2.calls, rc2.probes, rc2.hits)
        np.testing.assert_array_equal(sorted_hits(h2), sorted_hits(ref2))
        # sizes beyond the fixed maximum are refused
        big, nb = W.unit_array(units * 6, [], N)
        assert nb > 4096
        st, _, _ = run_noalloc(engine, tid, big, nb)
        assert st == -1
    finally:
        engine.free_table(tid)
