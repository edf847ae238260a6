#!/usr/bin/env python3
"""Benchmark: class-5 peel probes/sec and eligible-B/hour at B~3.2M on B200.

One step = one pass of the cls5 hot path (2-D (d,e) free peel, mod-124,488
gate, xor probe) over the production-shape band B in [3,200,000, 3,220,000]
(all ~155k Stage-1 cls5 units plus 32 seeded plants) against an r=48 xor
table for N = ceil(B_max/42) built on the device.  `value` is R>0 grid
points ("peel probes") per second with units already resident in HBM;
`e2e` is the same metric through the C ABI with host buffers.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): each rank owns its own 20,000-B band (weak scaling),
no collective on the data path; rank 0 prints one JSON line.  With
--shards S the ranks instead split one pair-space shard set (a table too
large for one GPU): each holds its range of shards and runs the whole band
(strong scaling); the hits are gathered once at the end.

  python bench.py --workload cls617 [--impl ours|reference]
  python bench.py --workload jobs    (reduced-T jobs through a .bbj file)

measures the (6,1,7) Branch-A class-5 search instead: one step is every
candidate of the eligible B in [400,401, 400,441) (a slice of the band
B in [400,000, 440,000]) plus 128 plants, against the N=10,476 r=48 table;
`value` counts probes the way the reference's summary does (3 per post-gate
xor probe).  `classes_1_4` times one pass over the same band's classes 1-4
find4 jobs.  Its reference arm runs the reference's own GPU binary
(oracle/_ref/solve_617_v1, built from the reference sources) on the same band.
"""
import argparse
import ctypes as C
import json
import math
import os
import re
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "six-one-five_b200"), os.path.join(ROOT, "oracle")]

METRIC = "cls5 peel probes/sec and eligible-B/hour at B≈3.2M, 1 B200; p99 unit latency"
UNIT = "peel_probes/s"
BAND_LO, BAND_W = 3_200_000, 20_000
PROBE_BYTES = 108          # 3 cells x 1.125 sectors x 32 B per post-gate xor probe (r=48)
N_PLANTS = 32


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--band-width", type=int, default=BAND_W)
    ap.add_argument("--band-lo", type=int, default=BAND_LO,
                    help="first B of rank 0's band (a smaller band/table for profiling)")
    ap.add_argument("--N", type=int, default=0, help="table N (default ceil(B_max/42))")
    ap.add_argument("--r", type=int, default=48)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-find4", action="store_true", help="cls617: skip the classes 1-4 pass")
    ap.add_argument("--shards", type=int, default=1,
                    help="cls5: a pair-space shard set of S tables (S >= 2) instead of one table")
    ap.add_argument("--layout", default="auto", choices=["auto", "wide", "packed"])
    ap.add_argument("--workload", default="cls5",
                    choices=["cls5", "cls617", "mix", "serve", "jobs", "cfg1"])
    ap.add_argument("--units", type=int, default=0, help="mix: units per step (default 200,000)")
    ap.add_argument("--seconds", type=float, default=10.0, help="serve: seconds of arrivals")
    ap.add_argument("--slots", type=int, default=2, help="serve: batches in flight")
    ap.add_argument("--no-l2-window", action="store_true",
                    help="cls5: time the pass without the peel's L2-persisting access window")
    ap.add_argument("--reference-gpu", type=int, default=15536,
                    help="cls5: run the reference's fourcore_cls5_gpu_v4 on K evenly spaced band "
                         "units (default: a tenth of the band; 0: the whole band; -1: skip)")
    return ap.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        pg = dist
    return rank, world, local, pg


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def probe_only_ceiling(lib, eng, tid, stream, n=1 << 28):
    """The probe's binding ceiling, measured in this process on the same
    resident table: the engine's own xor query kernel (k_xor_query -- the
    probe's hash, 64-bit cell indices and the same three cell loads per key,
    with no sieve around them) over n uniformly random keys, CUDA events on
    the launch stream, best of three after one warm launch.  Returns (cell
    reads/s, ms per launch)."""
    import torch

    import s615
    keys = torch.empty(n, dtype=torch.int64, device="cuda").random_(generator=None)
    out = torch.empty(n, dtype=torch.uint8, device="cuda")
    sptr = C.c_void_p(stream.cuda_stream)

    def go():
        s615._check(lib.s615_xor_query_dev(eng._ctx, tid, C.c_void_p(keys.data_ptr()), n,
                                           C.c_void_p(out.data_ptr()), sptr), "xor_query_dev")

    go()
    torch.cuda.synchronize()
    best = None
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        go()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del keys, out
    return 3 * n / (best / 1e3), best


def random_access_roof(lib, eng, tid, stream, probes, dur_s):
    """The probe's binding roofline: the pass's cell reads/s (3 per post-gate
    probe) over the probe-only ceiling on the same table."""
    ceil, ms = probe_only_ceiling(lib, eng, tid, stream)
    got = 3 * probes / dur_s
    return {"achieved_reads_per_s": got, "ceiling_reads_per_s": ceil,
            "frac": round(got / ceil, 4) if ceil else None,
            "ceiling_source": "k_xor_query (s615_xor_query_dev) on 2^28 uniformly random keys against "
                              f"the same resident table, same process, after the timed region: {ms:.2f} ms"}


def log(msg):
    print(f"[bench] {msg}", file=sys.stderr, flush=True)


def batch_h2d(lib, batch):
    """Bytes s615_prepare copied host-to-device for this batch (unit records +
    work items), the same the C-ABI entry points copy per call."""
    nu, ni, hb = C.c_size_t(0), C.c_size_t(0), C.c_size_t(0)
    lib.s615_batch_size(batch, C.byref(nu), C.byref(ni), C.byref(hb))
    return hb.value


def timed_steps(lib, eng, tid, batch, stream, flags, steps):
    """CUDA-event time of `steps` back-to-back s615_run_batch calls (ms) and
    the counters of the last one."""
    import torch

    import s615
    sptr = C.c_void_p(stream.cuda_stream)
    s615._check(lib.s615_run_batch(eng._ctx, tid, batch, flags, sptr), "run_batch")   # warm
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        s615._check(lib.s615_run_batch(eng._ctx, tid, batch, flags, sptr), "run_batch")
    e1.record(stream)
    torch.cuda.synchronize()
    ctr = s615.Counters()
    nh = C.c_size_t(0)
    lib.s615_batch_results(eng._ctx, batch, None, 0, C.byref(nh), C.byref(ctr))
    return e0.elapsed_time(e1), ctr


def serve_latency(eng, tid, units, N, rate=5000.0, secs=8.0, req_units=50, seed=5, tune=False,
                  warmup_s=0.5, window_s=10.0):
    """Per-unit latency under a Poisson stream of requests through the serving
    loop (s615_submit / s615_poll): `rate` units/s in requests of `req_units`
    units drawn from the band; a unit's latency is its request's
    submit-to-verified-result time.  Requests submitted in the first
    `warmup_s` seconds (while the loop's slots grow their buffers) are served
    but not counted.  p50/p99 are also given per `window_s` window of
    submission time.  With tune, s615_autotune first tunes batches of one and
    two requests (the loop's usual batches) on samples of the band."""
    import numpy as np

    import s615
    import workloads as W
    rng = np.random.RandomState(seed)
    tuned = None
    if tune:
        tuned = []
        for k in (req_units, 2 * req_units):
            pick = [units[i] for i in rng.randint(0, len(units), size=k)]
            arr, n = W.unit_array(pick, [], N)
            _, best = eng.autotune(tid, arr, n)
            tuned.append({"units": k, "item_rows": best[0], "blocks_per_sm": best[1]})
    eng.serve_start(slots=2)
    lat, batch_reqs, sent, warm, when = [], [], 0, set(), {}
    by_window = {}

    def take(r):
        if r["ticket"] not in warm:
            lat.extend([r["latency_ms"]] * r["n_units"])
            by_window.setdefault(int(when[r["ticket"]] // window_s), []).extend(
                [r["latency_ms"]] * r["n_units"])
            batch_reqs.append(r["batch_requests"])

    try:
        t0 = time.perf_counter()
        nxt = t0
        done = 0
        while time.perf_counter() - t0 < secs:
            now = time.perf_counter()
            while nxt <= now:
                pick = [units[i] for i in rng.randint(0, len(units), size=req_units)]
                arr, n = W.unit_array(pick, [], N)
                t = eng.submit(tid, arr, n)
                when[t] = now - t0
                if now - t0 < warmup_s:
                    warm.add(t)
                sent += 1
                nxt += rng.exponential(req_units / rate)
            for r in eng.poll(wait_ms=1):
                take(r)
                done += 1
            time.sleep(max(0.0, min(0.001, nxt - time.perf_counter())))
        while done < sent:
            for r in eng.poll(wait_ms=100):
                take(r)
                done += 1
    finally:
        eng.serve_stop()
        if tune:
            eng.tune_reset()
    lat = np.array(lat)
    windows = [{"from_s": k * window_s, "units": len(v),
                "p50_ms": round(float(np.percentile(v, 50)), 3),
                "p99_ms": round(float(np.percentile(v, 99)), 3)}
               for k, v in sorted(by_window.items()) if len(v) >= 100]
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "p99_ms_per_window": windows,
            "units": int(lat.size), "requests": sent, "warmup_requests_not_counted": len(warm),
            "seconds": secs, "offered_units_per_s": rate,
            "request_units": req_units, "mean_requests_per_batch": float(np.mean(batch_reqs)),
            "tuned": tuned,
            "loop": "s615_serve_start(slots=2) + s615_submit/s615_poll, Poisson arrivals"}


def reference_gpu_cls5(lib, eng, tid, units, N, r, stream, max_units=0):
    """The reference's own class-5 program (fourcore_cls5_gpu_v4, compiled
    from the reference sources into oracle/_ref) on the same Stage-1 units
    and the same table bytes (the engine's table saved in the reference's
    file format and given to it with --load-table), on this GPU: its summary
    counters (calls=, probes=) must equal the engine's on the same units, and
    its time= (the chunk loop: 16 units per launch, per-chunk sync and host
    verify) is set against the engine's device time for those units."""
    import shutil
    import tempfile

    import s615
    import workloads as W
    exe = os.path.join(ROOT, "oracle", "_ref", "fourcore_cls5_gpu_v4")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/fourcore_cls5_gpu_v4 not built"}
    if max_units and len(units) > max_units:
        idx = [round(i * (len(units) - 1) / (max_units - 1)) for i in range(max_units)]
        units = [units[i] for i in idx]
    info = eng.table_info(tid)
    file_bytes = 64 + (info.hdr.m_cells * info.hdr.r + 7) // 8 + 8
    tmp = os.environ.get("TMPDIR") or tempfile.gettempdir()
    free = shutil.disk_usage(tmp).free
    if free < file_bytes * 1.05 + (2 << 30):
        return {"unavailable": f"the table file needs {file_bytes / 1e9:.1f} GB of disk, "
                               f"{free / 1e9:.1f} GB free in {tmp}"}
    try:
        import psutil
        if psutil.virtual_memory().available < file_bytes * 1.3 + (8 << 30):
            return {"unavailable": "not enough host memory for the reference to read the table"}
    except ImportError:
        pass
    d = tempfile.mkdtemp(dir=tmp)
    try:
        path = os.path.join(d, f"xor_N{N}_r{r}.bin")
        t0 = time.perf_counter()
        eng.save_table(tid, path)
        save_s = time.perf_counter() - t0
        buc = os.path.join(d, "band.buc")
        W.write_buc(buc, units)
        t0 = time.perf_counter()
        p = subprocess.run([exe, "--units", buc, "--N", str(N), "--r", str(r), "--load-table", path,
                            "--quiet"], capture_output=True, text=True, timeout=3600)
        wall = time.perf_counter() - t0
        m = re.search(r"---- done cls5-gpu: solutions=(\d+) units=(\d+) calls=(\d+) probes=(\d+) "
                      r"time=([\d.]+)s", p.stdout)
        if p.returncode != 0 or not m:
            return {"unavailable": "fourcore_cls5_gpu_v4 failed: " +
                                   " ".join(p.stderr.strip().splitlines()[-2:])}
    finally:
        shutil.rmtree(d, ignore_errors=True)
    # the engine on exactly these units (no plants), device time
    arr, n = W.unit_array(units, [], N)
    b = C.c_void_p()
    s615._check(lib.s615_prepare(eng._ctx, C.cast(arr, C.c_void_p), n, C.byref(b)), "prepare")
    ms, c = timed_steps(lib, eng, tid, b, stream, 0, 1)
    s615._check(lib.s615_batch_free(eng._ctx, b), "batch_free")
    ref_s = float(m.group(5))
    return {"program": "oracle/_ref/fourcore_cls5_gpu_v4 (reference sources, nvcc sm_100a)",
            "units": int(m.group(2)), "calls": int(m.group(3)), "probes": int(m.group(4)),
            "solutions": int(m.group(1)),
            "counters_equal": (int(m.group(3)), int(m.group(4))) == (c.calls, c.probes),
            "time_s": ref_s, "process_wall_s": round(wall, 1), "table_save_s": round(save_s, 1),
            "peel_probes_per_s": c.pos / ref_s if ref_s else None,
            "engine_ms_same_units": ms, "engine_over_reference": ref_s / (ms / 1e3) if ms else None,
            "note": "time= is the reference's own summary figure (after table upload; its 16-unit "
                    "chunk loop with per-chunk sync and host verify); R>0 points are the engine's "
                    "count for the same units (the reference does not print them)"}


def band_units(lo, hi):
    import workloads as W
    return W.cls5_units(lo, hi)


def eligible_count(lo, hi):
    return sum(1 for B in range(lo, hi + 1) if math.gcd(B, 42) == 1)


def cpu_sample_rate(table, units, plants_n, N, budget_s=15.0, check=None):
    """Oracle (CPU restatement of k_cls5_192) on a bounded sample of the same
    units and table: R>0 points per second with all host threads."""
    import numpy as np

    import orc
    cores = os.cpu_count() or 1
    step = max(1, len(units) // 4096)
    pool = units[::step]
    one = orc.units_array([orc.pack_unit(*pool[0])])
    t0 = time.perf_counter()
    _, c1 = orc.cls5_run(table, one, 1, threads=1)
    t_unit = max(time.perf_counter() - t0, 1e-3)
    n = max(cores, min(len(pool), int(cores * budget_s / t_unit)))
    n = min(n, len(pool))
    idx = np.linspace(0, len(pool) - 1, n).astype(int)
    sample = [pool[i] for i in idx]
    arr = orc.units_array([orc.pack_unit(B, u) for B, u in sample])
    t0 = time.perf_counter()
    hits, (calls, gated, probes) = orc.cls5_run(table, arr, len(sample), threads=cores)
    dt = time.perf_counter() - t0
    return {"value": (gated + probes) / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{len(sample)} of the band's units (evenly spaced), same r=48 table; "
                      f"{gated + probes:.3e} R>0 points in {dt:.1f} s",
            "_counters": (calls, gated, probes)}, sample, hits


REF_TABLE_N = 8000   # the reference arm's host-built table (see run_reference)


def run_reference(args, rank):
    """--impl reference: the reference's CPU path restated (oracle port of
    k_cls5_192 with the reference's per-point 192-bit peel, mod-192 gate and
    funnel key) on the box's host cores.  Units come from the oracle's own
    Stage-1 rule, so this process maps only oracle/ libraries.  Each timed
    step is an evenly spaced sample of 32 units per host thread (dynamic
    scheduling over units keeps every thread busy); warm-up steps take one
    unit per thread."""
    if rank != 0:
        return 0
    import orc
    lo, hi = args.band_lo, args.band_lo + args.band_width
    units = [(B, u) for B in range(lo, hi) if math.gcd(B, 42) == 1 for u in orc.unit_candidates(B, 5)]
    # the reference's host table builder needs hours and ~100 GB at N=76,667;
    # the reference arm probes a host-built N=8,000 table instead (~240 MB, past
    # the host's last-level cache, so the probes are DRAM reads as they are on
    # the band's table; probes are ~3% of the points and the per-point 192-bit
    # peel dominates CPU time)
    table = orc.Table.build_pairs(REF_TABLE_N, args.r)
    cores = os.cpu_count() or 1
    rates, samples = [], []
    for s in range(args.warmup + args.steps):
        per = 32 * cores if s >= args.warmup else cores
        stride = max(1, len(units) // per)
        chunk = units[(s * 7919) % stride::stride][:per]
        arr = orc.units_array([orc.pack_unit(B, u) for B, u in chunk])
        t0 = time.perf_counter()
        _, (calls, gated, probes) = orc.cls5_run(table, arr, len(chunk), threads=cores)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            rates.append((gated + probes) / dt)
            samples.append(len(chunk))
    v = statistics.mean(rates)
    assert "s615" not in sys.modules, "the reference arm must not load the engine"
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64", "data": "synthetic",
            "config": {"workload": f"cls5 band B in [{lo}, {hi}), Stage-1 units (oracle rule); "
                                   f"reference arm: the oracle port of k_cls5_192 on {samples[0]} "
                                   f"evenly spaced units per step ({samples[0] // cores} per host "
                                   f"thread) against a host-built N={REF_TABLE_N} r={args.r} table "
                                   f"(the engine arm probes N=76,667)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{samples[0]} units per step x {args.steps} steps"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------ (6,1,7) class-5 workload
METRIC617 = "(6,1,7) Branch-A cls5 probes/sec (3 per post-gate xor probe), B in [400k,440k], 1 B200"
UNIT617 = "probes/s"
LO617, W617, N617, PLANTS617 = 400_401, 40, 10_476, 128


def eligible617(B):
    return B >= 11 and B % 2 == 1 and B % 3 != 0 and B % 7 != 0


def plants617(n, seed, N):
    """Planted 7-term bases in the reference's plant shape
    (solve_617_v1.cu:1564-1582), drawn so that the planted c4 and c3 lie in
    the windows k_find4_cls5 searches (3 c4^6 >= T, 3 c3^6 >= T - c4^6)."""
    import numpy as np
    rng = np.random.RandomState(seed)
    out = []
    while len(out) < n:
        c = sorted(int(x) for x in rng.choice(np.arange(1, N + 1), 4, replace=False))
        T = sum(x**6 for x in c)
        if 3 * c[3] ** 6 < T or 3 * c[2] ** 6 < T - c[3] ** 6:
            continue
        d = int(rng.randint(1, 281))
        out.append((c, d, (21 * d) ** 6 + 42**6 * T))
    return out


def run617(args, rank, world, local, dist):
    import numpy as np
    import torch

    import s615

    torch.cuda.set_device(local)
    width = args.band_width if args.band_width != BAND_W else W617
    lo = (args.band_lo if args.band_lo != BAND_LO else LO617) + rank * width
    hi = lo + width
    N = args.N or N617
    eng = s615.Engine(local)
    t0 = time.perf_counter()
    tid = eng.build_table(N, args.r)
    build_s = time.perf_counter() - t0
    Bs = [B for B in range(lo, hi) if eligible617(B)]
    cands = []
    for B in Bs:
        arr, n = s615.candidates617(B)
        cands += [arr[i] for i in range(n)]
    plants = plants617(PLANTS617, 617 + rank, N)
    n = len(cands) + len(plants)
    units = (s615.Unit * n)()
    for i, x in enumerate(cands):
        units[i] = x
    for j, (c, d, base) in enumerate(plants):
        units[len(cands) + j] = s615.make_plant617(base, d, N, B=42 * N + 1)
    log(f"rank {rank}: {len(Bs)} B in [{lo}, {hi}): {len(cands)} candidates + {len(plants)} plants")

    lib = s615.lib()
    batch = C.c_void_p()
    s615._check(lib.s615_prepare(eng._ctx, C.cast(units, C.c_void_p), n, C.byref(batch)), "prepare")
    stream = torch.cuda.Stream()
    sptr = C.c_void_p(stream.cuda_stream)

    def step():
        s615._check(lib.s615_run_batch(eng._ctx, tid, batch, 0, sptr), "run_batch")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    launches0 = eng.launches
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    for k in range(args.steps):
        step()
        ev[k + 1].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    cl = clocks.stop()
    launches = eng.launches - launches0
    per_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[args.steps])

    hits = (s615.Hit * (1 << 20))()
    nh = C.c_size_t(0)
    ctr = s615.Counters()
    s615._check(lib.s615_batch_results(eng._ctx, batch, C.cast(hits, C.c_void_p), 1 << 20,
                                       C.byref(nh), C.byref(ctr)), "results")
    harr = s615.hits_to_array(hits, nh.value)
    sols = eng.verify(units, n, harr, N)
    got = {(s.unit, tuple(sorted((s.c1, s.c2, s.c3, s.c4))), s.d) for s in sols if s.kind == 1}
    recovered = sum(1 for j, (c, d, _) in enumerate(plants)
                    if (len(cands) + j, tuple(c), d) in got)
    solutions = [s615.solution_line(s) for s in sols if s.kind == 0]
    import shard
    total_ms, tot = shard.merge(dist, "cuda", total_ms,
                                {"probes": ctr.probes, "pos": ctr.pos, "B": len(Bs)})
    value = 3 * tot["probes"] * args.steps / (total_ms / 1e3)
    step_s = total_ms / args.steps / 1e3

    # e2e: s615_run with host unit records in and hits + counters out
    e2e_steps = max(1, min(args.steps, 2))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        h2, c2 = eng.run(tid, units, n, hit_cap=1 << 16)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    assert c2.probes == ctr.probes and c2.tri_total == ctr.tri_total
    # whole job over the ranks: the slowest rank's e2e step against all ranks' probes
    e2e_ms, e2e_job = shard.merge(dist, "cuda", e2e_s * 1e3, {"probes": ctr.probes})

    sharp = None
    if rank == 0:
        sms, sctr = timed_steps(lib, eng, tid, batch, stream, s615.F_SHARP, 1)
        sharp = {"c3_points_per_s": sctr.pos / (sms / 1e3), "ms_per_step": sms,
                 "post_gate_probes": sctr.probes,
                 "speedup_vs_default": (total_ms / args.steps) / sms,
                 "flag": "S615_F_SHARP (extra sound residue tests; raw hits a subset)"}

    find4 = None
    if rank == 0 and not args.no_find4:
        find4 = run617_find4(lib, eng, tid, stream, Bs)

    peak, peak_kind = measured_peaks()
    achieved = ctr.probes * PROBE_BYTES / (statistics.mean(per_ms) / 1e3) / 1e9
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_kind": f"{peak_kind} hbm_gbs (burst)",
            "traffic": None, "algorithmic_bytes_per_launch": ctr.probes * PROBE_BYTES}
    if rank == 0:
        roof["random_access"] = random_access_roof(lib, eng, tid, stream, ctr.probes,
                                                   statistics.mean(per_ms) / 1e3)

    cpu = None
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        import orc
        hb, pk = eng.export_table(tid)
        ot = orc.Table.from_memory(hb, pk)
        cores = os.cpu_count() or 1
        # a bounded sample: 2 candidates per host thread, evenly spaced over the
        # step's candidates, one OpenMP run over them
        allc = orc.concat617([orc.cands617(B) for B in Bs])
        idx = np.linspace(0, allc[1] - 1, min(allc[1], 2 * cores)).astype(int)
        samp = (orc.OrcCand617 * len(idx))()
        for k, i in enumerate(idx):
            samp[k] = allc[0][i]
        t0 = time.perf_counter()
        _, c = orc.run617(ot, samp, len(idx), threads=cores)
        took = time.perf_counter() - t0
        cpu = {"value": 3 * c[0] / took, "unit": UNIT617, "cores": cores, "kind": "port",
               "sample": f"{len(idx)} evenly spaced candidates of the step ({c[0]} post-gate probes "
                         f"in {took:.1f} s; oracle restatement of k_find4_cls5)"}
        del ot, pk

    line = {
        "metric": METRIC617, "value": value, "unit": UNIT617, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u128", "data": "synthetic",
        "config": {"workload": f"(6,1,7) cls5: every candidate of the {len(Bs)} eligible B in "
                               f"[{lo}, {hi}) per rank ({len(cands)} candidates) + {len(plants)} plants; "
                               f"xor table N={N} r={args.r} built on device",
                   "N": N, "r": args.r,
                   "l2": "table %.2f GB, larger than L2" % (eng.table_info(tid).device_bytes / 1e9),
                   "parallelism": f"replicas-by-band x{world}"},
        "B_per_hour": tot["B"] / step_s * 3600,
        "c3_points_per_s": tot["pos"] / step_s,
        "counters": {"c3_points": ctr.pos, "gated": ctr.gated, "post_gate_probes": ctr.probes,
                     "tri_total": ctr.tri_total, "tri_skipped": ctr.tri_skipped, "hits": ctr.hits},
        "plants_recovered": f"{recovered}/{len(plants)}", "solutions": solutions,
        "table_build_s": round(build_s, 2),
        "e2e": {"value": 3 * e2e_job["probes"] / (e2e_ms / 1e3), "unit": UNIT617,
                "h2d_bytes_per_step": batch_h2d(lib, batch),
                "d2h_bytes_per_step": C.sizeof(s615.Counters) + len(h2) * 32},
        "gpu_launches": launches,
        "roofline": roof,
        "cpu_baseline": cpu,
        "sharp_gate": sharp,
        "classes_1_4": find4,
        "clocks": cl,
    }
    s615._check(lib.s615_batch_free(eng._ctx, batch), "batch_free")
    eng.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run617_find4(lib, eng, tid, stream, Bs):
    """(6,1,7) classes 1-4 of the same B band: every find4 job of
    s615_617_jobs (the reference's find5 expansion, solve_617_v1.cu:807-884)
    in one batch, one CUDA-event timed pass after a warm pass."""
    import s615
    t0 = time.perf_counter()
    units, n = s615.jobs617_band(Bs)
    jobs_s = time.perf_counter() - t0
    if not n:
        return None
    batch = C.c_void_p()
    t0 = time.perf_counter()
    s615._check(lib.s615_prepare(eng._ctx, C.cast(units, C.c_void_p), n, C.byref(batch)), "prepare")
    prep_s = time.perf_counter() - t0
    ms, ctr = timed_steps(lib, eng, tid, batch, stream, 0, 1)
    s615._check(lib.s615_batch_free(eng._ctx, batch), "batch_free")
    return {"jobs": n, "probes": 3 * ctr.probes, "ms_per_step": ms,
            "probes_per_s": 3 * ctr.probes / (ms / 1e3), "c4_total": ctr.tri_total,
            "c4_tri_skipped": ctr.tri_skipped, "c3_points": ctr.pos, "hits": ctr.hits,
            "host_jobs_s": round(jobs_s, 2), "host_prepare_s": round(prep_s, 2)}


def run617_reference(args, rank):
    """--workload cls617 --impl reference: the reference's own GPU binary
    (solve_617_v1, compiled from the reference sources into oracle/_ref) on
    the same band; its summary's kernel time and probe rate."""
    if rank != 0:
        return 0
    exe = os.path.join(ROOT, "oracle", "_ref", "solve_617_v1")
    width = args.band_width if args.band_width != BAND_W else W617
    lo = args.band_lo if args.band_lo != BAND_LO else LO617
    hi = lo + width - 1
    base = {"impl": "reference", "metric": METRIC617, "unit": UNIT617}
    if not os.path.exists(exe):
        print(json.dumps({**base, "unavailable": "oracle/_ref/solve_617_v1 not built"}), flush=True)
        return 0
    rates, secs = [], []
    for s in range(max(1, args.steps)):
        p = subprocess.run([exe, str(lo), str(hi), "5", "--branch-a-only", "--r", str(args.r),
                            "--quiet"], capture_output=True, text=True, timeout=3600)
        m = re.search(r"cls5: cands=(\d+) probes=(\S+) kernel=([\d.]+)s rate=(\S+) probes/s", p.stderr)
        if p.returncode != 0 or not m:
            print(json.dumps({**base, "unavailable": "solve_617_v1 failed: " +
                              " ".join(p.stderr.strip().splitlines()[-2:])}), flush=True)
            return 0
        rates.append(float(m.group(4)))
        secs.append(float(m.group(3)))
    v = statistics.mean(rates)
    find4 = None
    if not args.no_find4:
        # classes 1-4 of the same band, one run: summed kernel time of its
        # per-class k_find4 launches
        p = subprocess.run([exe, str(lo), str(hi), "1234", "--branch-a-only", "--r", str(args.r),
                            "--quiet"], capture_output=True, text=True, timeout=3600)
        per = re.findall(r"cls(\d): cands=(\d+) probes=(\S+) kernel=([\d.]+)s", p.stderr)
        if p.returncode == 0 and per:
            probes = sum(float(x[2]) for x in per)
            ksec = sum(float(x[3]) for x in per)
            find4 = {"jobs": sum(int(x[1]) for x in per), "probes": probes, "ms_per_step": ksec * 1e3,
                     "probes_per_s": probes / ksec if ksec else None,
                     "per_class": {x[0]: {"jobs": int(x[1]), "probes": float(x[2]),
                                          "kernel_s": float(x[3])} for x in per},
                     "note": "kernel seconds as the summary prints them (0.1 s resolution)"}
    line = {**base, "value": v, "n_gpus": 1, "steps": len(rates), "warmup": 0,
            "ms_per_step": statistics.mean(secs) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u128", "data": "synthetic",
            "config": {"workload": f"(6,1,7) cls5 band B in [{lo}, {hi}], reference solve_617_v1 "
                                   f"--branch-a-only --r {args.r} (table N={hi // 42} built on the host)"},
            "cpu_baseline": None,
            "e2e": {"value": v, "unit": UNIT617, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "classes_1_4": find4,
            "note": "kernel time as the reference's summary prints it (k_find4_cls5 launches only)"}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------ mixed classes and serving
METRIC_MIX = "mixed-class units/s (classes 2:4%/3:1%/4:48%/5:47%, B log-uniform [1M,4M]), 1 B200"
METRIC_SERVE = "per-unit latency p50/p99 through the serving loop (Poisson 5,000 units/s), 1 B200"


def solve_516_cfg1(points, runs=15):
    """The reference's own CPU path on config 1 (`solve_516_v2 1000 30000 5`,
    OpenMP over every host core; solve_516_v2.cpp:488-563), timed without
    its pair-index build.  Its search is an exact pair-sum index rather than
    the xor probe, so the rate is quoted per R>0 point of the same 725 units
    (`points`, the oracle's count).  None when the program was not built."""
    exe = os.path.join(ROOT, "oracle", "_ref", "solve_516_v2")
    if not os.path.exists(exe):
        return None
    search = []
    units = sols = None
    for _ in range(runs):
        t0 = time.perf_counter()
        p = subprocess.run([exe, "1000", "30000", "5"], capture_output=True, text=True, timeout=120)
        wall = time.perf_counter() - t0
        if p.returncode != 0:
            return None
        m = re.search(r"index built in (\d+) ms", p.stderr)
        search.append(wall - (int(m.group(1)) / 1e3 if m else 0.0))
        mu = re.search(r"unit candidates tested: (\d+)", p.stderr)
        ms = re.search(r"total solutions: (\d+)", p.stderr)
        units = int(mu.group(1)) if mu else None
        sols = int(ms.group(1)) if ms else None
    t = statistics.median(search)
    return {"value": points / t, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
            "sample": f"oracle/_ref/solve_516_v2 1000 30000 5, median of {runs} runs: "
                      f"{t * 1e3:.1f} ms of search (process wall minus its printed index build) "
                      f"for {units} units, {sols} solutions; rate per R>0 point of those units"}


def run_cfg1(args, rank, world, local, dist):
    """--workload cfg1: the small CPU-runnable configuration -- every class-5
    unit of B in [1000, 30000] (725) plus 8 plants against an N = 715, r = 48
    table built on the device (1.9 MB) -- timed with and without the peel's
    L2-persisting access window, and the oracle on the host cores beside it."""
    import numpy as np
    import torch

    import orc
    import s615
    import workloads as W
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    N = 715
    eng = s615.Engine(local)
    tid = eng.build_table(N, args.r)
    units = W.cls5_units(1000, 30000)
    plants = W.plants(8, 0, 1000, 30000, N)
    arr, n = W.unit_array(units, plants, N)
    lib = s615.lib()
    b = C.c_void_p()
    s615._check(lib.s615_prepare(eng._ctx, C.cast(arr, C.c_void_p), n, C.byref(b)), "prepare")
    stream = torch.cuda.Stream()
    res = {}
    for name, fl in (("window", 0), ("no_window", s615.F_NO_L2_WINDOW)):
        for _ in range(args.warmup):
            timed_steps(lib, eng, tid, b, stream, fl, 1)
        ms, c = timed_steps(lib, eng, tid, b, stream, fl, max(args.steps, 50))
        res[name] = {"ms_per_pass": ms / max(args.steps, 50), "pos": c.pos, "probes": c.probes}
    s615._check(lib.s615_batch_free(eng._ctx, b), "batch_free")
    hb, pk = eng.export_table(tid)
    ot = orc.Table.from_memory(hb, pk)
    oarr = orc.units_array([orc.pack_unit(B, u) for B, u in units])
    t0 = time.perf_counter()
    _, (calls, gated, probes) = orc.cls5_run(ot, oarr, len(units))
    cpu_s = time.perf_counter() - t0
    eng.close()
    port = {"value": (gated + probes) / cpu_s, "unit": UNIT, "cores": os.cpu_count(),
            "kind": "port", "sample": f"all {len(units)} units once"}
    ref = solve_516_cfg1(gated + probes)
    v = res["window"]["pos"] / (res["window"]["ms_per_pass"] / 1e3)
    line = {"metric": "cls5 peel probes/sec, B in [1000, 30000] (config 1), 1 B200", "value": v,
            "unit": UNIT, "n_gpus": 1, "steps": max(args.steps, 50), "warmup": args.warmup,
            "ms_per_step": res["window"]["ms_per_pass"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": f"config 1: {len(units)} Stage-1 units + 8 plants, N={N} r={args.r} "
                                   "table built on the device (1.9 MB: fits L2)"},
            "l2_window": res,
            "cpu_baseline": ref or port,
            "cpu_port": port}
    print(json.dumps(line), flush=True)
    return 0


def run_mix(args, rank, world, local, dist):
    """200,000 Stage-1 units of classes 2-5 in one persistent batch (the mixed
    queue), B log-uniform on [1M, 4M], 64 plants, N = 95,239 (B <= 4M)."""
    import numpy as np
    import torch

    import s615
    import workloads as W
    torch.cuda.set_device(local)
    n_units = args.units or 200_000
    N = args.N or math.ceil(4_000_000 / 42)
    eng = s615.Engine(local)
    t0 = time.perf_counter()
    tid = eng.build_table(N, args.r)
    build_s = time.perf_counter() - t0
    units = W.mixed_units(n_units, 3 + rank, 1_000_000, 4_000_000)
    p5 = W.plants(32, 33 + rank, 1_000_000, 4_000_000, N)
    p24 = W.plants234(32, 34 + rank, 1_000_000, 4_000_000, N)
    arr, n = W.mixed_unit_array(units, p5, p24, N)
    lib = s615.lib()
    batch = C.c_void_p()
    s615._check(lib.s615_prepare(eng._ctx, C.cast(arr, C.c_void_p), n, C.byref(batch)), "prepare")
    stream = torch.cuda.Stream()
    sptr = C.c_void_p(stream.cuda_stream)
    for _ in range(args.warmup):
        s615._check(lib.s615_run_batch(eng._ctx, tid, batch, 0, sptr), "run_batch")
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    launches0 = eng.launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        s615._check(lib.s615_run_batch(eng._ctx, tid, batch, 0, sptr), "run_batch")
    e1.record(stream)
    torch.cuda.synchronize()
    cl = clocks.stop()
    launches = eng.launches - launches0
    ms = e0.elapsed_time(e1)
    hits = (s615.Hit * (1 << 20))()
    nh = C.c_size_t(0)
    ctr = s615.Counters()
    s615._check(lib.s615_batch_results(eng._ctx, batch, C.cast(hits, C.c_void_p), 1 << 20,
                                       C.byref(nh), C.byref(ctr)), "results")
    sms, sctr = timed_steps(lib, eng, tid, batch, stream, s615.F_SHARP, 1)
    sharp = {"ms_per_step": sms, "units_per_s": n / (sms / 1e3), "post_gate_probes": sctr.probes,
             "speedup_vs_default": (ms / args.steps) / sms,
             "flag": "S615_F_SHARP (extra sound residue tests; raw hits a subset)"}
    sols = eng.verify(arr, n, s615.hits_to_array(hits, nh.value), N, cap=65536)
    k5 = len(units)
    got5 = {(s.unit, s.d, s.e, s.c1, s.c2) for s in sols if s.kind == 1 and s.cls == 5}
    rec5 = sum((k5 + j, p.d, p.e, p.c1, p.c2) in got5 for j, p in enumerate(p5))
    got24 = {(s.unit, s.d, (s.c1, s.c2, s.c3)) for s in sols if s.kind == 1 and s.cls != 5}
    rec24 = sum((k5 + len(p5) + j, d, c) in got24 for j, (_, _, d, c, _) in enumerate(p24))
    t0 = time.perf_counter()
    h2, c2 = eng.run(tid, arr, n, hit_cap=1 << 16)
    e2e_s = time.perf_counter() - t0
    assert c2.pos == ctr.pos and c2.probes == ctr.probes
    import collections

    import shard
    mix = collections.Counter(c for c, _, _ in units)
    # whole job over the ranks: the slowest rank's time against all ranks' units
    job_ms, job = shard.merge(dist, "cuda", ms, {"units": n})
    e2e_ms, e2e_job = shard.merge(dist, "cuda", e2e_s * 1e3, {"units": n})
    step_s = job_ms / args.steps / 1e3
    # the probe's roofline for one launch (all steps are the same pass)
    peak, peak_kind = measured_peaks()
    per_s = (ms / args.steps) / 1e3
    achieved = ctr.probes * PROBE_BYTES / per_s / 1e9
    mix_roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_kind": f"{peak_kind} hbm_gbs (burst)",
                "traffic": None, "algorithmic_bytes_per_launch": ctr.probes * PROBE_BYTES,
                "random_access": random_access_roof(lib, eng, tid, stream, ctr.probes, per_s)
                if rank == 0 else None}
    line = {"metric": METRIC_MIX, "value": job["units"] / step_s, "unit": "units/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": job_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic",
            "config": {"workload": f"{len(units)} Stage-1 units {dict(sorted(mix.items()))} + 64 plants, "
                                   f"one persistent batch; xor table N={N} r={args.r} on device",
                       "N": N, "r": args.r,
                       "l2": "table %.1f GB, larger than L2" % (eng.table_info(tid).device_bytes / 1e9)},
            "points_per_s": ctr.pos / step_s,
            "counters": {"calls": ctr.calls, "gated": ctr.gated, "probes": ctr.probes, "pos": ctr.pos},
            "plants_recovered": f"{rec5 + rec24}/{len(p5) + len(p24)}",
            "solutions": [s615.solution_line(s) for s in sols if s.kind == 0],
            "table_build_s": round(build_s, 2),
            "e2e": {"value": e2e_job["units"] / (e2e_ms / 1e3), "unit": "units/s",
                    "h2d_bytes_per_step": batch_h2d(lib, batch),
                    "d2h_bytes_per_step": C.sizeof(s615.Counters) + len(h2) * C.sizeof(s615.Hit)},
            "gpu_launches": launches, "roofline": mix_roof, "cpu_baseline": None,
            "sharp_gate": sharp, "clocks": cl}
    s615._check(lib.s615_batch_free(eng._ctx, batch), "batch_free")
    eng.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


METRIC_JOBS = ("reduced-T jobs/s (.bbj file, classes 1-4 of the mixed stream, B log-uniform "
               "[1M,4M]), 1 B200")


def run_jobs(args, rank, world, local, dist):
    """Stage-1 units of classes 1-4 drawn like the mixed stream (B log-uniform
    on [1M, 4M]) expanded into reduced-T jobs (expand_unit), written to a .bbj
    file and read back; one step = one device pass over every job (find3 rows
    for classes 2-4, find4 for class 1) against the N = 95,239 table."""
    import tempfile

    import numpy as np
    import torch

    import s615
    import workloads as W
    torch.cuda.set_device(local)
    n_units = args.units or 20_000
    N = args.N or math.ceil(4_000_000 / 42)
    eng = s615.Engine(local)
    t0 = time.perf_counter()
    tid = eng.build_table(N, args.r)
    build_s = time.perf_counter() - t0
    units = W.mixed_units(n_units, 5 + rank, 1_000_000, 4_000_000,
                          mix={1: 0.01, 2: 0.04, 3: 0.01, 4: 0.48})
    t0 = time.perf_counter()
    jobs, n, fail_t = s615.expand_units(units)
    expand_s = time.perf_counter() - t0
    path = os.path.join(tempfile.gettempdir(), f"s615_bench_jobs_{rank}.bbj")
    t0 = time.perf_counter()
    s615.jobs_write(path, jobs, n)
    write_s = time.perf_counter() - t0
    file_bytes = os.path.getsize(path)
    t0 = time.perf_counter()
    jobs, n2, _ = s615.jobs_read(path)
    read_s = time.perf_counter() - t0
    assert n2 == n
    log(f"rank {rank}: {len(units)} units -> {n} jobs ({file_bytes / 1e6:.1f} MB .bbj)")

    lib = s615.lib()
    stream = torch.cuda.Stream()
    sptr = C.c_void_p(stream.cuda_stream)
    batch = C.c_void_p()
    s615._check(lib.s615_prepare(eng._ctx, C.cast(jobs, C.c_void_p), n, C.byref(batch)), "prepare")
    for _ in range(args.warmup):
        s615._check(lib.s615_run_batch(eng._ctx, tid, batch, 0, sptr), "run_batch")
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    launches0 = eng.launches
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    for k in range(args.steps):
        s615._check(lib.s615_run_batch(eng._ctx, tid, batch, 0, sptr), "run_batch")
        ev[k + 1].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    cl = clocks.stop()
    launches = eng.launches - launches0
    per_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[args.steps])
    hits = (s615.Hit * (1 << 20))()
    nh = C.c_size_t(0)
    ctr = s615.Counters()
    s615._check(lib.s615_batch_results(eng._ctx, batch, C.cast(hits, C.c_void_p), 1 << 20,
                                       C.byref(nh), C.byref(ctr)), "results")
    sms, sctr = timed_steps(lib, eng, tid, batch, stream, s615.F_SHARP, 1)
    sharp = {"ms_per_step": sms, "jobs_per_s": n / (sms / 1e3), "post_gate_probes": sctr.probes,
             "speedup_vs_default": (total_ms / args.steps) / sms,
             "flag": "S615_F_SHARP (extra sound residue tests; raw hits a subset)"}
    sols = eng.verify(jobs, n, s615.hits_to_array(hits, nh.value), N, cap=65536)
    h2d = batch_h2d(lib, batch)
    s615._check(lib.s615_batch_free(eng._ctx, batch), "batch_free")

    # the same Stage-1 units searched directly (no job format): same rows
    uarr = (s615.Unit * len(units))()
    for i, (c, B, u) in enumerate(units):
        uarr[i].cls, uarr[i].B, uarr[i].u = c, B, u
    s615._check(lib.s615_prepare(eng._ctx, C.cast(uarr, C.c_void_p), len(units), C.byref(batch)),
                "prepare")
    units_ms, uctr = timed_steps(lib, eng, tid, batch, stream, 0, 1)
    s615._check(lib.s615_batch_free(eng._ctx, batch), "batch_free")
    assert (uctr.pos, uctr.probes) == (ctr.calls, ctr.probes)

    # e2e: the .bbj file read into the caller's host buffer (allocated once, as a
    # reader of file after file keeps it), then s615_run (host jobs in, hits +
    # counters out)
    jbuf = (s615.Unit * n)()
    e2e_steps = max(1, min(args.steps, 2))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        j3, n3, _ = s615.jobs_read(path, out=jbuf)
        h3, c3 = eng.run(tid, j3, n3, hit_cap=1 << 16)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    # the same step one C-ABI call per phase
    ph = {}
    t0 = time.perf_counter()
    j3, n3, _ = s615.jobs_read(path, out=jbuf)
    ph["bbj_read_ms"] = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    b3 = C.c_void_p()
    s615._check(lib.s615_prepare(eng._ctx, C.cast(j3, C.c_void_p), n3, C.byref(b3)), "prepare")
    ph["prepare_ms"] = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    s615._check(lib.s615_run_batch(eng._ctx, tid, b3, 0, None), "run_batch")
    hb3 = (s615.Hit * (1 << 16))()
    nh3, c4 = C.c_size_t(0), s615.Counters()
    s615._check(lib.s615_batch_results(eng._ctx, b3, C.cast(hb3, C.c_void_p), 1 << 16,
                                       C.byref(nh3), C.byref(c4)), "results")
    ph["run_and_results_ms"] = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    s615._check(lib.s615_batch_free(eng._ctx, b3), "batch_free")
    ph["free_ms"] = (time.perf_counter() - t0) * 1e3
    e2e_phases = {k: round(v, 1) for k, v in ph.items()}
    log(f"jobs e2e phases: {e2e_phases}")
    assert c3.probes == ctr.probes
    os.remove(path)

    cpu = None
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        import orc
        cores = os.cpu_count() or 1
        table = orc.Table.build_pairs(2000, args.r)

        def sample(count):
            idx = np.linspace(0, n - 1, min(n, count)).astype(int)
            samp = (orc.OrcJob * len(idx))()
            for k, i in enumerate(idx):
                J = jobs[int(i)]
                samp[k].cls, samp[k].lim, samp[k].B, samp[k].u = J.cls, (J.B - 1) // 42, J.B, J.u
                samp[k].free1, samp[k].free2 = J.res_d, J.res_e
                samp[k].T[0], samp[k].T[1] = J.base[0], J.base[1]
            t0 = time.perf_counter()
            _, oc = orc.run_jobs(table, samp, len(idx), threads=cores)
            return idx, oc, time.perf_counter() - t0

        idx, oc, took = sample(64 * cores)          # calibration, then ~10 s of CPU work
        idx, oc, took = sample(int(len(idx) * 10.0 / max(took, 1e-3)))
        cpu = {"value": len(idx) / took, "unit": "jobs/s", "cores": cores, "kind": "port",
               "sample": f"{len(idx)} evenly spaced jobs of the step ({oc[0]:.3e} c3/c4 points in "
                         f"{took:.1f} s; oracle restatement of run_batch, probing a host-built "
                         f"N=2000 r={args.r} table)"}

    import collections
    import shard
    total_ms, tot = shard.merge(dist, "cuda", total_ms, {"jobs": n})
    e2e_ms, e2e_job = shard.merge(dist, "cuda", e2e_s * 1e3, {"jobs": n})
    step_s = total_ms / args.steps / 1e3
    peak, peak_kind = measured_peaks()
    achieved = ctr.probes * PROBE_BYTES / (statistics.mean(per_ms) / 1e3) / 1e9
    mix = collections.Counter(c for c, _, _ in units)
    jmix = collections.Counter(jobs[i].cls for i in range(0, n, max(1, n // 100000)))
    line = {"metric": METRIC_JOBS, "value": tot["jobs"] / step_s, "unit": "jobs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u128",
            "data": "synthetic",
            "config": {"workload": f"{len(units)} Stage-1 units {dict(sorted(mix.items()))} expanded "
                                   f"into {n} reduced-T jobs (.bbj {file_bytes / 1e6:.1f} MB); xor "
                                   f"table N={N} r={args.r} on device",
                       "N": N, "r": args.r,
                       "l2": "table %.1f GB, larger than L2" % (eng.table_info(tid).device_bytes / 1e9),
                       "parallelism": f"replicas x{world}"},
            "points_per_s": ctr.calls / step_s,
            "counters": {"calls": ctr.calls, "gated": ctr.gated, "probes": ctr.probes, "hits": ctr.hits},
            "jobs_by_class_sampled": dict(sorted(jmix.items())),
            "exact_matches": len(sols),
            "solutions": [s615.solution_line(s) for s in sols if s.kind == 0],
            "units_path": {"ms_per_step": units_ms, "jobs_over_units_time": (total_ms / args.steps) / units_ms},
            "host": {"expand_s": round(expand_s, 2), "fail_t": fail_t, "bbj_write_s": round(write_s, 2),
                     "bbj_read_s": round(read_s, 2), "bbj_bytes": file_bytes},
            "table_build_s": round(build_s, 2),
            "e2e": {"value": e2e_job["jobs"] / (e2e_ms / 1e3), "unit": "jobs/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": C.sizeof(s615.Counters) + len(h3) * C.sizeof(s615.Hit),
                    "includes": ".bbj read + s615_run", "phases": e2e_phases},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_kind": f"{peak_kind} hbm_gbs (burst)",
                         "traffic": None, "algorithmic_bytes_per_launch": ctr.probes * PROBE_BYTES,
                         "random_access": (random_access_roof(
                             lib, eng, tid, stream, ctr.probes, statistics.mean(per_ms) / 1e3)
                             if rank == 0 else None)},
            "cpu_baseline": cpu, "sharp_gate": sharp, "clocks": cl}
    eng.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_serve(args, rank, world, local, dist):
    """Serving with four resident tables: requests of 50 units arrive as a
    Poisson stream (5,000 units/s); B uniform on [1M, 5M], classes mixed
    2:4%/3:1%/4:48%/5:47%; each request goes to the smallest table whose N
    covers its B; 256 planted targets ride in the stream; the context's HBM
    admission budget is 150 GB."""
    import numpy as np

    import s615
    import workloads as W
    if rank != 0:
        return 0
    eng = s615.Engine(local)
    Ns = [24_000, 48_000, 76_000, 120_000]

    def layout_for(N):
        """--layout auto: WIDE (one sector per cell) while the table's WIDE
        bytes (about 8 x 1.23 x N^2 / 2) stay under 68 GiB, PACKED above.
        Random reads run at full rate up to ~64 GiB and lose little just past
        it: at N = 120,000 (65.9 GiB WIDE) a class-5 pass ran 1.41x faster
        WIDE than PACKED (53 GB)."""
        if args.layout != "auto":
            return s615.LAYOUT_WIDE if args.layout == "wide" else s615.LAYOUT_PACKED
        return s615.LAYOUT_WIDE if 8 * 1.23 * N * N / 2 <= 68 * 2**30 else s615.LAYOUT_PACKED

    tids, builds = {}, {}
    for N in sorted(Ns, reverse=True):      # the largest build needs the most scratch
        t0 = time.perf_counter()
        try:
            tids[N] = eng.build_table(N, args.r, layout=layout_for(N))
            builds[N] = round(time.perf_counter() - t0, 2)
        except s615.S615Error as e:
            log(f"table N={N}: {e}")
    resident = sum(eng.table_info(t).device_bytes for t in tids.values())
    s615._check(s615.lib().s615_set_budget(eng._ctx, 150_000_000_000), "set_budget")
    ranges = []
    lo = 1_000_000
    for N in sorted(tids):
        hi = min(5_000_000, 42 * N + 1)
        if hi > lo:
            ranges.append((N, lo, hi))
            lo = hi + 1
    rng = np.random.RandomState(55)
    widths = np.array([hi - lo for _, lo, hi in ranges], dtype=float)
    p_tab = widths / widths.sum()
    rate, req_units, secs = 5000.0, 50, args.seconds
    plants_left = 256
    planted = {}          # (ticket, index) -> expected solution key
    eng.serve_start(slots=args.slots)
    lat, sent, done, got_plants = [], 0, 0, 0
    rows = []             # (submitted at, table N, latency ms, units) per request
    sub_at = {}           # ticket -> (seconds after start, table N)
    t_start = time.perf_counter()
    nxt = t_start
    try:
        while time.perf_counter() - t_start < secs:
            now = time.perf_counter()
            while nxt <= now:
                ti = int(rng.choice(len(ranges), p=p_tab))
                N, blo, bhi = ranges[ti]
                us = W.mixed_units(req_units, int(rng.randint(1 << 30)), blo, bhi, log_uniform=False)
                p5 = []
                if plants_left > 0 and rng.rand() < 0.5:
                    p5 = W.plants(1, int(rng.randint(1 << 30)), blo, bhi, N)
                arr, n = W.mixed_unit_array(us, p5, [], N)
                t = eng.submit(tids[N], arr, n)
                sub_at[t] = (now - t_start, N)
                if p5:
                    p = p5[0]
                    planted[t] = (len(us), p.d, p.e, p.c1, p.c2)
                    plants_left -= 1
                sent += 1
                nxt += rng.exponential(req_units / rate)
            for r in eng.poll(wait_ms=1):
                lat += [r["latency_ms"]] * r["n_units"]
                rows.append((*sub_at.pop(r["ticket"]), r["latency_ms"], r["n_units"]))
                done += 1
                if r["ticket"] in planted:
                    got = {(s.unit, s.d, s.e, s.c1, s.c2) for s in r["solutions"] if s.kind == 1}
                    got_plants += planted[r["ticket"]] in got
            time.sleep(max(0.0, min(0.001, nxt - time.perf_counter())))
        while done < sent:
            for r in eng.poll(wait_ms=100):
                lat += [r["latency_ms"]] * r["n_units"]
                rows.append((*sub_at.pop(r["ticket"]), r["latency_ms"], r["n_units"]))
                done += 1
                if r["ticket"] in planted:
                    got = {(s.unit, s.d, s.e, s.c1, s.c2) for s in r["solutions"] if s.kind == 1}
                    got_plants += planted[r["ticket"]] in got
    finally:
        eng.serve_stop()
    wall = time.perf_counter() - t_start
    lat = np.array(lat)

    def pcts(sel):
        """Unit-weighted p50 / p99 of the requests `sel` picks."""
        v = np.repeat([r[2] for r in rows if sel(r)], [r[3] for r in rows if sel(r)])
        return ({"units": int(v.size), "p50_ms": round(float(np.percentile(v, 50)), 3),
                 "p99_ms": round(float(np.percentile(v, 99)), 3)} if v.size else None)

    win = max(10.0, secs / 10)
    windows = [dict(from_s=round(w0, 1), **pcts(lambda r, w0=w0: w0 <= r[0] < w0 + win))
               for w0 in np.arange(0.0, secs, win) if pcts(lambda r, w0=w0: w0 <= r[0] < w0 + win)]
    per_table = {str(N): pcts(lambda r, N=N: r[1] == N) for N in sorted(tids)}
    line = {"metric": METRIC_SERVE, "value": float(np.percentile(lat, 99)), "unit": "ms",
            "n_gpus": 1, "steps": sent, "warmup": 0, "ms_per_step": None, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": f"Poisson {rate:.0f} units/s for {secs:.0f} s in {req_units}-unit requests, "
                                   "classes 2:4%/3:1%/4:48%/5:47%, B uniform [1M,5M]; resident tables "
                                   + ", ".join(f"N={N} " + ("wide" if eng.table_info(tids[N]).layout == s615.LAYOUT_WIDE
                                                             else "packed") for N in sorted(tids))
                                   + " (r=%d)" % args.r,
                       "hbm_budget_gb": 150, "resident_table_gb": round(resident / 1e9, 2)},
            "p50_unit_latency_ms": float(np.percentile(lat, 50)),
            "p99_unit_latency_ms": float(np.percentile(lat, 99)),
            "p99_ms_per_window": windows, "latency_per_table": per_table,
            "units_completed": int(lat.size), "requests": sent,
            "completed_units_per_s": lat.size / wall,
            "plants_recovered": f"{got_plants}/{len(planted)}",
            "table_build_s": builds,
            "e2e": None, "gpu_launches": eng.launches, "roofline": None, "cpu_baseline": None}
    eng.close()
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    rank, world, local, dist = dist_setup(args)
    if args.workload == "cfg1":
        return run_cfg1(args, rank, world, local, dist)
    if args.workload == "mix":
        return run_mix(args, rank, world, local, dist)
    if args.workload == "serve":
        return run_serve(args, rank, world, local, dist)
    if args.workload == "jobs":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "metric": METRIC_JOBS, "unavailable":
                                  "the reference's job runner (fourcore_find_v4) builds its N=95,239 "
                                  "table on the host before searching (hours, ~100 GB); its counters on "
                                  "job files are pinned on small windows by tests/golden/ref615.json, "
                                  "and the line's cpu_baseline is the oracle port"}),
                      flush=True)
            return 0
        return run_jobs(args, rank, world, local, dist)
    if args.workload == "cls617":
        if args.impl == "reference":
            return run617_reference(args, rank)
        return run617(args, rank, world, local, dist)
    if args.impl == "reference":
        return run_reference(args, rank)

    import numpy as np
    import torch

    import s615
    import shard
    import workloads as W

    torch.cuda.set_device(local)
    # --shards S over several GPUs splits the set: every rank runs the whole
    # band on its own range of shards (a table too large for one GPU)
    split = args.shards > 1 and world > 1
    if split:
        lo, hi = args.band_lo, args.band_lo + args.band_width
        N = args.N or math.ceil(hi / 42)
    else:
        lo, hi = shard.rank_band(args.band_lo, args.band_width, rank)
        N = args.N or shard.table_N(args.band_lo, args.band_width, world)
    eng = s615.Engine(local)
    layout = {"auto": s615.LAYOUT_AUTO, "wide": s615.LAYOUT_WIDE, "packed": s615.LAYOUT_PACKED}[args.layout]
    t0 = time.perf_counter()
    if split:
        s_lo, s_hi = shard.shard_range(rank, world, args.shards)
        tid = eng.build_table_shard_range(N, args.r, args.shards, s_lo, s_hi, layout)
    elif args.shards > 1:
        tid = eng.build_table_sharded(N, args.r, args.shards, layout)
    else:
        tid = eng.build_table(N, args.r, layout)
    build_s = time.perf_counter() - t0
    log(f"rank {rank}: table N={N} r={args.r} shards={args.shards} built in {build_s:.1f} s")
    units = band_units(lo, hi - 1)   # B in [lo, hi): bands of ranks do not overlap
    log(f"rank {rank}: {len(units)} units in [{lo}, {hi})")
    plants = W.plants(N_PLANTS, 1000 + (0 if split else rank), lo, hi, N)
    arr, n = W.unit_array(units, plants, N)

    lib = s615.lib()
    batch = C.c_void_p()
    s615._check(lib.s615_prepare(eng._ctx, C.cast(arr, C.c_void_p), n, C.byref(batch)),
                "prepare")
    # a real stream handle: the engine launches on it and the events below are
    # recorded on it (handle 0 would mean "the engine's own stream")
    stream = torch.cuda.Stream()
    sptr = C.c_void_p(stream.cuda_stream)

    run_flags = s615.F_NO_L2_WINDOW if args.no_l2_window else 0

    def step():
        s615._check(lib.s615_run_batch(eng._ctx, tid, batch, run_flags, sptr), "run_batch")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    launches0 = eng.launches
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    for k in range(args.steps):
        step()
        ev[k + 1].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    cl = clocks.stop()
    launches = eng.launches - launches0
    per_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[args.steps])

    hits = (s615.Hit * (1 << 20))()
    nh = C.c_size_t(0)
    ctr = s615.Counters()
    s615._check(lib.s615_batch_results(eng._ctx, batch, C.cast(hits, C.c_void_p), 1 << 20,
                                            C.byref(nh), C.byref(ctr)), "results")
    harr = s615.hits_to_array(hits, nh.value)
    counts = {"calls": ctr.calls, "gated": ctr.gated, "probes": ctr.probes, "pos": ctr.pos,
              "eligible": eligible_count(lo, hi - 1)}
    if split:   # slowest rank's time; the same counters on every rank; the union of the hits
        total_ms, tot, harr = shard.merge_split(dist, "cuda", total_ms, counts, harr)
    else:       # slowest rank's time, counters summed over ranks
        total_ms, tot = shard.merge(dist, "cuda", total_ms, counts)
    log(f"timed {args.steps} steps: {total_ms:.1f} ms; pos={ctr.pos} probes={ctr.probes} hits={nh.value}")
    sols = eng.verify(arr, n, harr, N)
    # a plant counts when its exact planted (d, e, c1, c2) is among the verified
    # identities (an even d can add a second, equally valid identity 21d = 42c)
    got = {(s.unit, s.d, s.e, s.c1, s.c2) for s in sols if s.kind == 1}
    recovered = sum(1 for j, p in enumerate(plants)
                    if (len(units) + j, p.d, p.e, p.c1, p.c2) in got)
    solutions = [s615.solution_line(s) for s in sols if s.kind == 0]

    pos_all = tot["pos"]
    value = pos_all * args.steps / (total_ms / 1e3)
    eligible = tot["eligible"]
    ms_step = total_ms / args.steps

    # e2e: the public C ABI with host buffers (unit records up, hits + counters down)
    # (s615_cls5_verify's exact verification of the step's raw hits is inside
    # the timed span: eligible B count as cleared only once verified)
    e2e_steps = max(1, min(args.steps, 3))
    h2d = batch_h2d(lib, batch)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        h2, c2 = eng.cls5_run(tid, arr, n, hit_cap=1 << 16)
        sols2 = eng.verify(arr, n, h2, N)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    log(f"e2e through s615_cls5_run + s615_verify: {e2e_s * 1e3:.1f} ms per step "
        f"(device step {total_ms / args.steps:.1f} ms)")
    assert c2.pos == ctr.pos and c2.probes == ctr.probes and len(sols2) == len(sols)
    d2h = C.sizeof(s615.Counters) + len(h2) * 32
    # whole-job e2e over the ranks: the slowest rank's e2e step (MAX) against
    # the job's points (pos_all: summed over replica bands; a shard split's
    # ranks search the same points), with every rank's copies counted
    e2e_ms, e2e_bytes = shard.merge(dist, "cuda", e2e_s * 1e3, {"h2d": h2d, "d2h": d2h})
    e2e_job_s = e2e_ms / 1e3
    # where the e2e step goes: the same work as s615_run, one C-ABI call per phase
    e2e_phases = None
    if rank == 0:
        ph = {}
        t0 = time.perf_counter()
        b2 = C.c_void_p()
        s615._check(lib.s615_prepare(eng._ctx, C.cast(arr, C.c_void_p), n, C.byref(b2)), "prepare")
        ph["prepare_ms"] = (time.perf_counter() - t0) * 1e3
        t0 = time.perf_counter()
        s615._check(lib.s615_run_batch(eng._ctx, tid, b2, 0, None), "run_batch")
        hb = (s615.Hit * (1 << 16))()
        nh2, c3 = C.c_size_t(0), s615.Counters()
        s615._check(lib.s615_batch_results(eng._ctx, b2, C.cast(hb, C.c_void_p), 1 << 16,
                                           C.byref(nh2), C.byref(c3)), "results")
        ph["run_and_results_ms"] = (time.perf_counter() - t0) * 1e3
        t0 = time.perf_counter()
        s615._check(lib.s615_batch_free(eng._ctx, b2), "batch_free")
        ph["free_ms"] = (time.perf_counter() - t0) * 1e3
        e2e_phases = {k: round(v, 1) for k, v in ph.items()}
        e2e_phases["note"] = ("a fresh batch through s615_prepare / s615_run_batch / "
                              "s615_batch_free; s615_cls5_run reuses the context's kept batch")
        log(f"e2e phases: {e2e_phases}")

    peak, peak_kind = measured_peaks()
    dur_s = statistics.mean(per_ms) / 1e3
    achieved = ctr.probes * PROBE_BYTES / dur_s / 1e9
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_kind": f"{peak_kind} hbm_gbs (burst)",
            # DRAM bytes need a profiler; this run has none (the ncu capture of the
            # same pass is summarised beside the kernel's roofline in the design notes)
            "traffic": None,
            "algorithmic_bytes_per_launch": ctr.probes * PROBE_BYTES}
    if rank == 0 and args.shards == 1:
        roof["random_access"] = random_access_roof(lib, eng, tid, stream, ctr.probes, dur_s)
        log("random-access roofline: %.3e cell reads/s of %s measured (%s)" % (
            roof["random_access"]["achieved_reads_per_s"],
            "%.3e" % roof["random_access"]["ceiling_reads_per_s"]
            if roof["random_access"]["ceiling_reads_per_s"] else "n/a",
            roof["random_access"]["frac"]))
    # DRAM bytes the probe moves: each cell read misses L2 and fills one 64-byte
    # line (ld.global.cg.L2::64B; a one-pass ncu capture of the full pass
    # measured 191.7 B per post-gate probe); against the same copy peak
    dram = 3 * 64 * ctr.probes / dur_s / 1e9
    roof["dram_fills"] = {"bytes_per_cell_read": 64, "achieved": round(dram, 1), "peak": peak,
                          "unit": "GB/s", "frac": round(dram / peak, 4)}

    # plain per-unit-launch form on a bounded sample of the same band
    plain = None
    if not args.no_plain and rank == 0:
        samp = units[:: max(1, len(units) // 1500)]
        parr, pn = W.unit_array(samp, [], N)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, pc = eng.cls5_run(tid, parr, pn, flags=s615.F_PLAIN, hit_cap=1 << 16)
        pdt = time.perf_counter() - t0
        p_rate = pc.pos / pdt
        plain = {"peel_probes_per_s": p_rate, "units": pn,
                 "eligible_B_per_hour": p_rate / (ctr.pos / eligible_count(lo, hi - 1)) * 3600,
                 "batched_over_plain": value / world / p_rate}

    # the band form: units generated and packed on the device from (B_lo, B_hi)
    band_e2e = None
    if rank == 0 and not args.no_plain:
        t0 = time.perf_counter()
        _, bn, bh, bctr = eng.run_band(tid, lo, hi - 1, hit_cap=1 << 16)
        bs = time.perf_counter() - t0
        band_e2e = {"value": bctr.pos / bs, "unit": UNIT, "units": bn, "seconds": bs,
                    # per-B and per-unit counts/offsets for the two prefix sums
                    "h2d_bytes_per_step": 4 * (hi - lo) + 4 * bn,
                    "d2h_bytes_per_step": 4 * (hi - lo) + 4 * bn + 16 * bn
                    + C.sizeof(s615.Counters) + 32 * len(bh),
                    "call": "s615_prepare_band + s615_batch_units + s615_run_batch + s615_batch_results"}
        log(f"band form (device Stage-1): {bs * 1e3:.1f} ms for {bn} units")

    # the opt-in sharper gate (S615_F_SHARP) on the same batch: same points,
    # fewer probes, the same verified solutions (tests/test_gpu_sharp.py)
    sharp = None
    if rank == 0 and not args.no_plain:
        sms, sctr = timed_steps(lib, eng, tid, batch, stream, s615.F_SHARP, 2)
        sharp = {"value": sctr.pos * 2 / (sms / 1e3), "unit": UNIT, "ms_per_step": sms / 2,
                 "post_gate_probes": sctr.probes, "pos": sctr.pos,
                 "speedup_vs_default": ms_step / (sms / 2),
                 "flag": "S615_F_SHARP (extra sound residue tests; raw hits a subset)"}
        log(f"sharp gate: {sms / 2:.1f} ms per step, probes {sctr.probes}")

    # per-unit latency through the serving loop under a config-5-like stream
    serve = None
    tune = None
    if rank == 0 and not args.no_plain:
        # the autotuner on a request-sized and a mid-sized sample of the band
        # (its choices are forgotten again: the numbers above use the default rule)
        tune = []
        for k in (64, 1024):
            idx = np.linspace(0, len(units) - 1, k).astype(int)
            sarr, sn = W.unit_array([units[i] for i in idx], [], N)
            table, best = eng.autotune(tid, sarr, sn)
            tune.append({"units": k, "best": {"item_rows": best[0], "blocks_per_sm": best[1],
                                              "ms": round(best[2], 3)},
                         "trials": [[r, b, round(ms, 3)] for r, b, ms in table]})
        eng.tune_reset()
    serve_tuned = None
    if rank == 0 and not args.no_plain:
        # the default rule carries the headline p50/p99; the tuned loop is reported beside it
        # (the tuner times batches alone; serving overlaps two, where its choice of fewer
        # blocks per SM lowers p50 and raises p99)
        serve = serve_latency(eng, tid, units, N, secs=60.0)
        serve_tuned = serve_latency(eng, tid, units, N, tune=True)
        log(f"serving: p50 {serve['p50_ms']:.2f} ms, p99 {serve['p99_ms']:.2f} ms per unit; "
            f"tuned p50 {serve_tuned['p50_ms']:.2f} ms, p99 {serve_tuned['p99_ms']:.2f} ms")

    ref_gpu = None
    if rank == 0 and world == 1 and args.shards == 1 and args.reference_gpu >= 0:
        ref_gpu = reference_gpu_cls5(lib, eng, tid, units, N, args.r, stream, args.reference_gpu)
        log(f"reference GPU program: {ref_gpu}")

    cpu = None
    parity = None
    if not args.no_cpu_baseline and rank == 0 and world == 1 and args.shards == 1:
        import orc
        hb, pk = eng.export_table(tid)
        ot = orc.Table.from_memory(hb, pk)
        cpu, sample, ohits = cpu_sample_rate(ot, units, 0, N)
        del ot, pk
        # the timed configuration itself against the oracle: the engine on the
        # sampled units with the same table must give the oracle's counters and
        # raw hits (unit index within the sample, d, e, fp)
        sarr, sn = W.unit_array(sample, [], N)
        shits, sctr = eng.cls5_run(tid, sarr, sn, hit_cap=1 << 20)
        okey = sorted(zip(ohits["unit"].tolist(), ohits["d"].tolist(), ohits["e"].tolist(),
                          ohits["fp"].tolist()))
        skey = sorted(zip(shits["unit"].tolist(), shits["d"].tolist(), shits["e"].tolist(),
                          shits["fp"].tolist()))
        oc = cpu.pop("_counters")
        parity = {"units": sn, "equal": okey == skey and (sctr.calls, sctr.gated, sctr.probes) == oc,
                  "raw_hits": len(skey), "oracle_raw_hits": len(okey),
                  "counters": {"calls": sctr.calls, "gated": sctr.gated, "probes": sctr.probes},
                  "oracle_counters": {"calls": oc[0], "gated": oc[1], "probes": oc[2]},
                  "what": "engine (s615_cls5_run) vs oracle on the CPU-baseline sample, same "
                          f"N={N} r={args.r} device-built table"}
        log(f"parity on {sn} sampled units: {parity['equal']} ({len(skey)} raw hits)")

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "strong" if split else "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": f"cls5 band B in [{lo}, {hi}){' (all ranks)' if split else ' per rank'}: "
                               f"{len(units)} Stage-1 units + "
                               f"{N_PLANTS} plants; xor table N={N} r={args.r} built on device"
                               + (f" as {args.shards} pair-space shards" if args.shards > 1 else ""),
                   "shards": args.shards,
                   "units_per_rank": n, "N": N, "r": args.r,
                   "l2": "inputs larger than L2 (table %.1f GB)" % (eng.table_info(tid).device_bytes / 1e9),
                   "l2_window": not args.no_l2_window,
                   "parallelism": (f"shard-split x{world}: each rank holds {args.shards // world}+ of "
                                   f"{args.shards} shards and runs the whole band" if split
                                   else f"replicas-by-band x{world}")},
        "eligible_B_per_hour": eligible * args.steps / (total_ms / 1e3) * 3600,
        # the same through the C ABI with host buffers, exact verification included
        "eligible_B_per_hour_e2e_with_verify": eligible / e2e_job_s * 3600,
        "p99_unit_latency_ms": serve["p99_ms"] if serve else None,
        "p50_unit_latency_ms": serve["p50_ms"] if serve else None,
        "serving": serve,
        "serving_tuned": serve_tuned,
        "autotune": tune,
        "counters": {"calls": tot["calls"], "gated": tot["gated"], "probes": tot["probes"],
                     "pos": pos_all},
        "plants_recovered": f"{recovered}/{N_PLANTS}", "solutions": solutions,
        "table_build_s": round(build_s, 2),
        "e2e": {"value": pos_all / e2e_job_s, "unit": UNIT, "h2d_bytes_per_step": e2e_bytes["h2d"],
                "d2h_bytes_per_step": e2e_bytes["d2h"], "phases": e2e_phases},
        "gpu_launches": launches,
        "roofline": roof,
        "cpu_baseline": cpu,
        "parity_sample": parity,
        "reference_gpu": ref_gpu,
        "plain_form": plain,
        "sharp_gate": sharp,
        "clocks": cl,
    }
    s615._check(lib.s615_batch_free(eng._ctx, batch), "batch_free")
    eng.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if parity is not None and not parity["equal"]:
        log("PARITY FAILURE: the engine and the oracle differ on the sampled units")
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
