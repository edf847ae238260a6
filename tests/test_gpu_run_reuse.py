"""s615_run keeps its batch between calls: results must not depend on what ran
before (smaller, larger, overflowing or failed calls, table builds that take the
buffers back), and dropped units keep their input index; freed batches leave
their device buffers in the context's pool for the next batch (GPU)."""
import ctypes as C

import numpy as np
import pytest

import s615
import workloads as W

pytestmark = pytest.mark.gpu

N1 = 715


def key(hits, ctr):
    a = sorted((int(h["unit"]), int(h["d"]), int(h["e"]), int(h["fp"])) for h in hits)
    return (ctr.calls, ctr.gated, ctr.probes, ctr.pos), a


@pytest.fixture(scope="module")
def setup(engine, oracle_table):
    _, path = oracle_table(N1, 16)
    tid = engine.load_table(path, N1)
    units = W.cls5_units(1000, 30000)
    plants = W.plants(8, 0, 1000, 30000, N1)
    small = W.unit_array(units[:40], [], N1)
    large = W.unit_array(units, plants, N1)
    yield tid, small, large
    engine.free_table(tid)


def test_results_do_not_depend_on_earlier_calls(engine, setup):
    tid, (sa, sn), (la, ln) = setup
    first_small = key(*engine.run(tid, sa, sn))
    first_large = key(*engine.run(tid, la, ln))
    assert first_large[0][2] > first_small[0][2] > 0
    for _ in range(2):
        assert key(*engine.run(tid, sa, sn)) == first_small     # a larger batch ran before
        assert key(*engine.run(tid, la, ln)) == first_large     # buffers grow back
    # an overflowing call reports the true count and leaves the next call intact
    with pytest.raises(s615.S615Error) as ei:
        engine.run(tid, la, ln, hit_cap=1)
    assert ei.value.status == -9
    assert key(*engine.run(tid, sa, sn)) == first_small
    # a failed call (a refused unit) keeps nothing and breaks nothing
    bad, bn = W.unit_array([(40_000_001, 6)], [], N1)
    with pytest.raises(s615.S615Error):
        engine.run(tid, bad, bn)
    assert key(*engine.run(tid, la, ln)) == first_large
    # a table build takes the kept buffers back
    t2 = engine.build_table(300, 16)
    engine.free_table(t2)
    assert key(*engine.run(tid, la, ln)) == first_large
    # the plain form and the kept batch agree
    assert key(*engine.run(tid, sa, sn, flags=s615.F_PLAIN)) == first_small


def test_dropped_units_keep_input_indices(engine, setup):
    tid, _, (la, ln) = setup
    base = key(*engine.run(tid, la, ln))
    # the same units with a dropped unit (u >= B) after every third one
    units = W.cls5_units(1000, 30000)
    plants = W.plants(8, 0, 1000, 30000, N1)
    arr, _ = W.unit_array(units, plants, N1)
    mixed, where = [], []
    for i in range(ln):
        where.append(len(mixed))
        mixed.append(arr[i])
        if i % 3 == 0:
            d = s615.Unit()
            d.cls, d.kind, d.B, d.u = 5, 0, 1003, 1008
            mixed.append(d)
    marr = (s615.Unit * len(mixed))(*mixed)
    hits, ctr = engine.run(tid, marr, len(mixed))
    back = {w: i for i, w in enumerate(where)}
    assert all(int(h["unit"]) in back for h in hits)
    hits = hits.copy()
    hits["unit"] = [back[int(u)] for u in hits["unit"]]
    assert key(hits, ctr) == base


def test_prepare_free_cycles_reuse_the_pool(engine, setup):
    tid, (sa, sn), (la, ln) = setup
    lib = s615.lib()

    def mem_free():
        f, t = C.c_size_t(0), C.c_size_t(0)
        s615._check(lib.s615_mem_info(engine._ctx, C.byref(f), C.byref(t)), "mem_info")
        return f.value

    def cycle(arr, n):
        b = C.c_void_p()
        s615._check(lib.s615_prepare(engine._ctx, C.cast(arr, C.c_void_p), n, C.byref(b)), "prepare")
        s615._check(lib.s615_run_batch(engine._ctx, tid, b, 0, None), "run_batch")
        hits = (s615.Hit * 4096)()
        nh, ctr = C.c_size_t(0), s615.Counters()
        s615._check(lib.s615_batch_results(engine._ctx, b, C.cast(hits, C.c_void_p), 4096,
                                           C.byref(nh), C.byref(ctr)), "results")
        s615._check(lib.s615_batch_free(engine._ctx, b), "batch_free")
        return key(s615.hits_to_array(hits, nh.value), ctr)

    t2 = engine.build_table(300, 16)   # gives back the kept batch and the pool
    engine.free_table(t2)
    want_l, want_s = key(*engine.run(tid, la, ln)), key(*engine.run(tid, sa, sn))
    t2 = engine.build_table(300, 16)
    engine.free_table(t2)
    before = mem_free()
    assert cycle(la, ln) == want_l
    held = mem_free()
    assert held < before          # the freed batch's buffers stay in the pool
    for _ in range(3):
        assert cycle(la, ln) == want_l
        assert cycle(sa, sn) == want_s
        assert mem_free() >= held - (4 << 20)   # taken from the pool, not allocated again
    t2 = engine.build_table(300, 16)          # a table build empties the pool
    engine.free_table(t2)
    assert mem_free() > held


def test_free_without_sync_does_not_hand_over_live_buffers(engine):
    """s615_batch_free right after an asynchronous s615_run_batch: the batch's
    buffers go to the pool only once its kernel is done, so the next batch,
    which takes them, gets its own results (a kernel still running would keep
    writing its counters and hits into them)."""
    import torch
    N = 23810                                   # B <= 1,000,020
    tid = engine.build_table(N, 48)
    lib = s615.lib()
    try:
        ua = W.cls5_units(1_000_000, 1_004_000)    # ~2e10 points: tens of ms on the device
        ub = W.cls5_units(990_000, 990_010)
        aa, na = W.unit_array(ua, [], N)
        ab, nb = W.unit_array(ub, [], N)
        want = key(*engine.run(tid, ab, nb))
        t2 = engine.build_table(300, 16)           # an empty pool and no kept batch
        engine.free_table(t2)
        stream = torch.cuda.Stream()
        for _ in range(3):
            a = C.c_void_p()
            s615._check(lib.s615_prepare(engine._ctx, C.cast(aa, C.c_void_p), na, C.byref(a)), "prepare")
            s615._check(lib.s615_run_batch(engine._ctx, tid, a, 0, C.c_void_p(stream.cuda_stream)),
                        "run_batch")
            s615._check(lib.s615_batch_free(engine._ctx, a), "batch_free")   # no sync before it
            b = C.c_void_p()
            s615._check(lib.s615_prepare(engine._ctx, C.cast(ab, C.c_void_p), nb, C.byref(b)), "prepare")
            s615._check(lib.s615_run_batch(engine._ctx, tid, b, 0, None), "run_batch")
            hits = (s615.Hit * 4096)()
            nh, ctr = C.c_size_t(0), s615.Counters()
            s615._check(lib.s615_batch_results(engine._ctx, b, C.cast(hits, C.c_void_p), 4096,
                                               C.byref(nh), C.byref(ctr)), "results")
            s615._check(lib.s615_batch_free(engine._ctx, b), "batch_free")
            assert key(s615.hits_to_array(hits, nh.value), ctr) == want
        torch.cuda.synchronize()
    finally:
        engine.free_table(tid)
