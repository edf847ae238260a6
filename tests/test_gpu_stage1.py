"""Stage-1 units generated and packed on the device (s615_prepare_band) (GPU).

The device batch must hold exactly the host rule's units in the same order
and give the same hits and counters as the host-packed batch.
"""
import pytest

import s615
import workloads as W

pytestmark = pytest.mark.gpu


def key(h):
    return sorted((int(x["unit"]), int(x["d"]), int(x["e"]), int(x["fp"])) for x in h)


@pytest.mark.parametrize("lo,hi,N,r", [(1000, 30000, 715, 16), (3200000, 3200800, 76200, 48)])
def test_band_equals_host_packing(engine, oracle_table, lo, hi, N, r):
    if N == 715:
        _, path = oracle_table(N, r)
        tid = engine.load_table(path, N)
    else:
        tid = engine.build_table(N, r)
    try:
        units, n, hits, ctr = engine.run_band(tid, lo, hi)
        host = W.cls5_units(lo, hi)
        assert [(units[i].B, units[i].u) for i in range(n)] == host
        if lo == 1000:
            assert n == 725                     # solve_516_v2's unit count on this window
        arr, hn = W.unit_array(host, [], N)
        hh, hc = engine.run(tid, arr, hn)
        assert (ctr.calls, ctr.gated, ctr.probes, ctr.pos) == (hc.calls, hc.gated, hc.probes, hc.pos)
        assert key(hits) == key(hh)
        sols = engine.verify(units, n, hits, N)
        assert sorted(s615.solution_line(s) for s in sols) == \
            sorted(s615.solution_line(s) for s in engine.verify(arr, hn, hh, N))
    finally:
        engine.free_table(tid)


def test_band_without_eligible_b(engine, oracle_table):
    _, path = oracle_table(300, 16)
    tid = engine.load_table(path, 300)
    try:
        units, n, hits, ctr = engine.run_band(tid, 12, 12)
        assert n == 0 and len(hits) == 0 and ctr.calls == 0
    finally:
        engine.free_table(tid)
