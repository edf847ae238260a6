"""Serving loop (s615_serve_start / s615_submit / s615_poll) on the device (GPU).

Requests for two resident tables and three unit kinds arrive from two threads
while others run; the worker coalesces them into batches.  Each request's hits
and verified solutions must equal those of s615_run + s615_verify on its units
alone.
"""
import threading
import time

import numpy as np
import pytest

import s615
import workloads as W

pytestmark = pytest.mark.gpu


def hit_key(h):
    return sorted((int(x["unit"]), int(x["d"]), int(x["e"]), int(x["c4"]), int(x["fp"])) for x in h)


def sol_key(sols):
    return sorted((s.unit, s.kind, s.cls, s.d, s.e, s.c1, s.c2, s.c3, s.c4, tuple(s.a)) for s in sols)


def slice_units(arr, lo, hi):
    out = (s615.Unit * max(hi - lo, 1))()
    for i in range(lo, hi):
        out[i - lo] = arr[i]
    return out, hi - lo


def test_serving_mix_equals_alone(engine, oracle_table):
    N1, N2 = 715, 54400 // 42
    _, p1 = oracle_table(N1, 20)
    _, p2 = oracle_table(N2, 16)
    t1 = engine.load_table(p1, N1)
    t2 = engine.load_table(p2, N2)
    try:
        # table 1: config-1 class-5 units and plants; table 2: (6,1,7) candidates
        u5 = W.cls5_units(1000, 30000)
        plants = W.plants(8, 0, 1000, 30000, N1)
        a5, n5 = W.unit_array(u5, plants, N1)
        trip = []
        for B in range(54301, 54341):
            if B % 2 and B % 3 and B % 7:
                arr, n = s615.candidates617(B)
                trip += [(arr[i].B, arr[i].u, arr[i].w) for i in range(n)]
        a7, n7 = s615.make_units617(trip)
        reqs = []
        step5 = max(1, n5 // 12)
        for lo in range(0, n5, step5):
            reqs.append((t1, N1) + slice_units(a5, lo, min(n5, lo + step5)))
        step7 = max(1, n7 // 6)
        for lo in range(0, n7, step7):
            reqs.append((t2, N2) + slice_units(a7, lo, min(n7, lo + step7)))

        alone = []
        for tid, N, arr, n in reqs:
            h, _ = engine.run(tid, arr, n)
            alone.append((hit_key(h), sol_key(engine.verify(arr, n, h, N))))

        engine.serve_start(slots=2)
        try:
            with pytest.raises(s615.S615Error) as e:
                engine.run(t1, reqs[0][2], reqs[0][3])
            assert e.value.status == -12      # BUSY while serving
            tickets = {}
            lock = threading.Lock()

            def client(idx):
                for i in idx:
                    tid, _, arr, n = reqs[i]
                    t = engine.submit(tid, arr, n)
                    with lock:
                        tickets[t] = i

            th = [threading.Thread(target=client, args=(list(range(k, len(reqs), 2)),))
                  for k in range(2)]
            for x in th:
                x.start()
            got = {}
            deadline = time.time() + 120
            while len(got) < len(reqs) and time.time() < deadline:
                for r in engine.poll(wait_ms=200):
                    got[r["ticket"]] = r
            for x in th:
                x.join()
        finally:
            engine.serve_stop()
        assert len(got) == len(reqs)
        mixed = 0
        for t, r in got.items():
            i = tickets[t]
            assert r["status"] == 0
            assert r["n_units"] == reqs[i][3]
            assert (hit_key(r["hits"]), sol_key(r["solutions"])) == alone[i], i
            assert 0 <= r["queued_ms"] <= r["latency_ms"]
            mixed += r["batch_requests"] > 1
        assert mixed > 0          # some requests shared a batch
        # the plants of table 1 are found through the loop too
        assert sum(len(r["solutions"]) for r in got.values()) >= len(plants)
        # the context is usable again after the loop stops
        h, _ = engine.run(t1, reqs[0][2], reqs[0][3])
        assert hit_key(h) == alone[0][0]
    finally:
        engine.free_table(t1)
        engine.free_table(t2)
