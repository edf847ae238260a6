"""Failures injected on the host (GPU): bad table files, the FPR-smoke refusal,
the command line's missing-table path, an admission budget too small for a
batch, and a request producer that dies while the serving loop runs.  None of
them faults, traps or hangs the GPU: each makes a call fail on the host side
and checks the status it returns, then that the context still works.

The reference makes a table that fails to load fatal unless --allow-rebuild
(fourcore_cls5_gpu_v4.cu:568-584) and refuses a table whose FPR smoke finds
more than 16 of 200k probe keys (:588-592, fourcore_xor_store.hpp:54-65).
"""
import os
import re
import subprocess
import threading

import pytest

import orc
import s615
import workloads as W

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN5 = os.path.join(ROOT, "six-one-five_b200", "bin", "s615_cls5")
DONE = re.compile(r"---- done cls5-gpu: solutions=(\d+) units=(\d+) calls=(\d+) probes=(\d+)")


def poll_n(engine, n):
    """The next n finished requests (60 s at most without one finishing)."""
    out, idle = [], 0
    while len(out) < n:
        got = engine.poll(wait_ms=1000)
        out += got
        idle = 0 if got else idle + 1
        assert idle < 60, "no request finished within 60 s"
    return out


def status_of(fn):
    with pytest.raises(s615.S615Error) as ei:
        fn()
    return ei.value.status


def test_truncated_and_padded_table_files(engine, oracle_table, tmp_path):
    _, path = oracle_table(300, 48)
    raw = open(path, "rb").read()
    short = tmp_path / "short.bin"
    short.write_bytes(raw[: 64 + (len(raw) - 64) // 2])     # header + half the cells
    assert status_of(lambda: engine.load_table(str(short), 300)) == -2          # S615_E_IO
    head = tmp_path / "head.bin"
    head.write_bytes(raw[:40])                               # not even a header
    assert status_of(lambda: engine.load_table(str(head), 300)) == -2
    # the context is intact: the good file still loads
    tid = engine.load_table(path, 300)
    try:
        assert engine.table_info(tid).hdr.N == 300
    finally:
        engine.free_table(tid)


def test_fpr_smoke_refuses_a_table_that_matches_too_often(engine, oracle_table):
    # r = 8: about 200,000 / 256 = 781 smoke hits, far above the 16 allowed
    assert status_of(lambda: engine.build_table(300, 8)) == -5                 # S615_E_FPR_SMOKE
    _, path8 = oracle_table(300, 8)
    assert status_of(lambda: engine.load_table(path8, 300)) == -5
    # r = 16 passes (about 3 hits), and nothing was left resident by the refusals
    tid = engine.build_table(300, 16)
    engine.free_table(tid)


def test_cli_missing_table_is_fatal_unless_allow_rebuild(tmp_path, oracle_table):
    N = 715
    t, _ = oracle_table(N, 48)
    units = W.cls5_units(1000, 30000)
    buc = tmp_path / "u.buc"
    W.write_buc(str(buc), units)
    missing = str(tmp_path / "missing.bin")
    args = [BIN5, "--units", str(buc), "--N", str(N), "--load-table", missing, "--r", "48"]
    p = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert p.returncode == 1 and "--allow-rebuild" in p.stderr
    assert "---- done" not in p.stdout
    p = subprocess.run(args + ["--allow-rebuild"], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    m = DONE.search(p.stdout)
    assert m, p.stdout
    # the device-built table holds the same key relation: the same counters
    arr = orc.units_array([orc.pack_unit(B, u) for B, u in units])
    _, (calls, _, probes) = orc.cls5_run(t, arr, len(units))
    assert (int(m.group(2)), int(m.group(3)), int(m.group(4))) == (len(units), calls, probes)
    # a table the FPR smoke refuses is fatal, --allow-rebuild or not
    _, path8 = oracle_table(N, 8)
    p = subprocess.run([BIN5, "--units", str(buc), "--N", str(N), "--load-table", path8, "--r", "8",
                        "--allow-rebuild"], capture_output=True, text=True, timeout=600)
    assert p.returncode == 1 and "FPR smoke" in p.stderr and "---- done" not in p.stdout


def test_serving_admission_out_of_budget(engine, oracle_table):
    N = 715
    _, path = oracle_table(N, 48)
    tid = engine.load_table(path, N)
    units = W.cls5_units(1000, 30000)[:50]
    arr, n = W.unit_array(units, [], N)
    lib = s615.lib()
    try:
        want, _ = engine.run(tid, arr, n)
        t2 = engine.build_table(300, 16)   # gives back s615_run's kept batch and the batch pool
        engine.free_table(t2)
        s615._check(lib.s615_set_budget(engine._ctx, 1), "set_budget")   # nothing more fits
        engine.serve_start(slots=2)
        try:
            t = engine.submit(tid, arr, n)
            [r] = poll_n(engine, 1)
            assert r["ticket"] == t and r["status"] == -6                          # S615_E_OOM
        finally:
            engine.serve_stop()
        s615._check(lib.s615_set_budget(engine._ctx, 0), "set_budget")   # all device memory
        engine.serve_start(slots=2)
        try:
            t = engine.submit(tid, arr, n)
            [r] = poll_n(engine, 1)
            assert r["ticket"] == t and r["status"] == 0
            key = lambda h: sorted((int(x["unit"]), int(x["d"]), int(x["e"]), int(x["fp"])) for x in h)
            assert key(r["hits"]) == key(want)
        finally:
            engine.serve_stop()
    finally:
        s615._check(lib.s615_set_budget(engine._ctx, 0), "set_budget")
        engine.free_table(tid)


def test_serving_survives_a_producer_that_dies(engine, oracle_table):
    N = 715
    _, path = oracle_table(N, 20)
    tid = engine.load_table(path, N)
    units = W.cls5_units(1000, 30000)
    plants = W.plants(8, 0, 1000, 30000, N)
    arr, n = W.unit_array(units, plants, N)
    step = 40
    reqs = []
    for lo in range(0, n, step):
        k = min(step, n - lo)
        sub = (s615.Unit * k)(*[arr[lo + i] for i in range(k)])
        reqs.append((sub, k))
    key = lambda h: sorted((int(x["unit"]), int(x["d"]), int(x["e"]), int(x["fp"])) for x in h)
    try:
        alone = [key(engine.run(tid, a, k)[0]) for a, k in reqs]
        tickets, lock = {}, threading.Lock()

        def producer(idx, die_after):
            for j, i in enumerate(idx):
                if j == die_after:
                    raise RuntimeError("producer stopped")   # dies mid-stream
                t = engine.submit(tid, *reqs[i])
                with lock:
                    tickets[t] = i

        errors = []

        def run(idx, die_after):
            try:
                producer(idx, die_after)
            except RuntimeError as e:
                errors.append(str(e))

        engine.serve_start(slots=2)
        try:
            half = list(range(0, len(reqs), 2)), list(range(1, len(reqs), 2))
            th = [threading.Thread(target=run, args=(half[0], len(half[0]) // 2)),
                  threading.Thread(target=run, args=(half[1], None))]
            for x in th:
                x.start()
            for x in th:
                x.join()
            assert errors == ["producer stopped"]
            done = {}
            for r in poll_n(engine, len(tickets)):
                assert r["status"] == 0
                done[r["ticket"]] = key(r["hits"])
            # every request that was submitted completes with its units' own hits
            assert all(done[t] == alone[i] for t, i in tickets.items())
            assert len(tickets) == len(half[1]) + len(half[0]) // 2
        finally:
            engine.serve_stop()
    finally:
        engine.free_table(tid)
