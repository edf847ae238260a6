"""The autotuner (s615_autotune) on the device (GPU).

It times every candidate (rows per class 2-5 item x blocks per SM) on a
batch, keeps the fastest for batches of that size, and never changes results.
"""
import pytest

import s615
import workloads as W

pytestmark = pytest.mark.gpu


def key(hits):
    return sorted(tuple(int(h[f]) for f in ("unit", "d", "e", "c4", "fp")) for h in hits)


@pytest.mark.parametrize("flags,trials", [(0, 15), (s615.F_SHARP, 9)])
def test_autotune_picks_the_fastest_and_keeps_results(engine, oracle_table, flags, trials):
    N = 2000
    _, path = oracle_table(N, 16)
    tid = engine.load_table(path, N)
    try:
        units = [(5, B, u) for B, u in W.cls5_units(80001, 84000)][:96]
        units += [(c, B, u) for B in range(80001, 80400) if W.eligible(B)
                  for c in (2, 4) for u in s615.unit_candidates(B, c)][:32]
        arr, n = W.mixed_unit_array(units, [], [], N)
        h0, c0 = engine.run(tid, arr, n, flags)              # the default rule
        table, best = engine.autotune(tid, arr, n, flags)
        assert len(table) == trials
        assert {(r, b) for r, b, _ in table} == {(r, b) for r in (16, 32, 64)
                                                   for b in range(1, trials // 3 + 1)}
        assert best[2] == min(ms for _, _, ms in table) and best[2] > 0
        h1, c1 = engine.run(tid, arr, n, flags)              # now the tuned setting
        fields = ("calls", "gated", "probes", "pos", "hits")
        assert key(h1) == key(h0)
        assert [getattr(c1, f) for f in fields] == [getattr(c0, f) for f in fields]
        engine.tune_reset()
    finally:
        engine.free_table(tid)
