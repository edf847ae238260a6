"""ctypes binding of the engine's C ABI (include/s615.h).

This is the Python-side view a user (or the tests and bench) gets of
``lib/libs615.so``: the same entry points, the same structs, errors raised as
:class:`S615Error` carrying the C status.  There is no fallback: if the
library is missing or no GPU is present, calls that need the device fail.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Iterable, List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# S615_CHECKED=1 loads the checked build (`make -C six-one-five_b200 checked`):
# the same library whose kernels check every index they use (s615_check_flags).
LIB_PATH = os.path.join(HERE, "lib", "libs615_checked.so" if os.environ.get("S615_CHECKED") == "1"
                        else "libs615.so")

S615_OK = 0
STATUS = {
    -1: "ARG", -2: "IO", -3: "FORMAT", -4: "N_MISMATCH", -5: "FPR_SMOKE", -6: "OOM",
    -7: "DEVICE", -8: "TIMEOUT", -9: "OVERFLOW", -10: "BUILD", -11: "NOTABLE", -12: "BUSY",
}
LAYOUT_AUTO, LAYOUT_PACKED, LAYOUT_WIDE = 0, 1, 2
F_NO_GATE, F_PLAIN, F_NO_TRI, F_SHARP, F_NO_L2_WINDOW = 1, 2, 4, 8, 16
S615_CLS_617 = 7
S615_CLS_617_FIND4 = 8
S615_KIND_JOB = 2


class S615Error(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"{what}: {STATUS.get(status, status)} ({status})")
        self.status = status


class Header(C.Structure):
    _fields_ = [("magic", C.c_uint32), ("version", C.c_uint32), ("kind", C.c_uint32),
                ("r", C.c_uint32), ("w", C.c_uint32), ("N", C.c_uint32),
                ("n_keys", C.c_uint64), ("m_cells", C.c_uint64), ("mix_seed", C.c_uint64),
                ("shard_count", C.c_uint32), ("shard_index", C.c_uint32),
                ("shard_mode", C.c_uint32), ("reserved", C.c_uint32)]


class TableInfo(C.Structure):
    _fields_ = [("hdr", Header), ("layout", C.c_int), ("cell_bytes", C.c_int),
                ("device_bytes", C.c_uint64)]


class Unit(C.Structure):
    _fields_ = [("cls", C.c_uint32), ("kind", C.c_uint32), ("B", C.c_uint64), ("u", C.c_uint64),
                ("base", C.c_uint64 * 3), ("fmax1", C.c_uint32), ("fmax2", C.c_uint32),
                ("res_e", C.c_uint32), ("res_d", C.c_uint32), ("lim", C.c_uint32),
                ("w", C.c_uint32)]


class Hit(C.Structure):
    _fields_ = [("unit", C.c_uint32), ("a", C.c_uint32), ("b", C.c_uint32), ("d", C.c_uint32),
                ("e", C.c_uint32), ("c4", C.c_uint32), ("fp", C.c_uint64)]


class Counters(C.Structure):
    _fields_ = [("calls", C.c_uint64), ("gated", C.c_uint64), ("probes", C.c_uint64),
                ("pos", C.c_uint64), ("hits", C.c_uint64), ("tri_total", C.c_uint64),
                ("tri_skipped", C.c_uint64)]


class Solution(C.Structure):
    _fields_ = [("unit", C.c_uint32), ("kind", C.c_uint32), ("cls", C.c_uint32), ("c3", C.c_uint32),
                ("B", C.c_uint64), ("u", C.c_uint64),
                ("d", C.c_uint32), ("e", C.c_uint32), ("c1", C.c_uint32), ("c2", C.c_uint32),
                ("c4", C.c_uint32), ("w", C.c_uint32), ("a", C.c_int64 * 7), ("gcd", C.c_int64)]


class Result(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("status", C.c_int32), ("table_id", C.c_int32),
                ("n_units", C.c_uint64), ("n_hits", C.c_uint64), ("n_solutions", C.c_uint64),
                ("hits", C.POINTER(Hit)), ("solutions", C.POINTER(Solution)),
                ("counters", Counters), ("batch_requests", C.c_uint32), ("pad", C.c_uint32),
                ("queued_ms", C.c_double), ("latency_ms", C.c_double)]


assert C.sizeof(Header) == 64
assert C.sizeof(Hit) == 32
assert C.sizeof(Unit) == 72
assert C.sizeof(Counters) == 56
assert C.sizeof(Solution) == 120

HIT_DTYPE = np.dtype([("unit", "<u4"), ("a", "<u4"), ("b", "<u4"), ("d", "<u4"), ("e", "<u4"),
                      ("c4", "<u4"), ("fp", "<u8")])

# Every entry point declared in include/s615.h, with its ctypes signature.
_P = C.c_void_p
SIGNATURES = {
    "s615_strerror": (C.c_char_p, [C.c_int]),
    "s615_open": (C.c_int, [C.c_int, C.c_size_t, C.POINTER(_P)]),
    "s615_close": (C.c_int, [_P]),
    "s615_launch_count": (C.c_uint64, [_P]),
    "s615_checked_build": (C.c_int, []),
    "s615_check_flags": (C.c_int, [_P, C.POINTER(C.c_uint32)]),
    "s615_set_budget": (C.c_int, [_P, C.c_size_t]),
    "s615_load_table": (C.c_int, [_P, C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "s615_build_table": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "s615_build_table_keys": (C.c_int, [_P, _P, C.c_size_t, C.c_int, C.c_uint64, C.c_int,
                                        C.POINTER(C.c_int)]),
    "s615_save_table": (C.c_int, [_P, C.c_int, C.c_char_p]),
    "s615_build_table_sharded": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.POINTER(C.c_int)]),
    "s615_load_table_shards": (C.c_int, [_P, C.POINTER(C.c_char_p), C.c_int, C.c_int, C.c_int,
                                         C.POINTER(C.c_int)]),
    "s615_save_table_shard": (C.c_int, [_P, C.c_int, C.c_int, C.c_char_p]),
    "s615_set_probe_groups": (C.c_int, [_P, C.c_int, C.c_int]),
    "s615_autotune": (C.c_int, [_P, C.c_int, _P, C.c_size_t, C.c_uint, _P, C.c_size_t,
                                C.POINTER(C.c_size_t), _P]),
    "s615_tune_reset": (C.c_int, [_P]),
    "s615_build_table_shard_range": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                               C.c_int, C.POINTER(C.c_int)]),
    "s615_export_table": (C.c_int, [_P, C.c_int, C.POINTER(Header), _P, C.c_size_t,
                                    C.POINTER(C.c_size_t)]),
    "s615_get_table_info": (C.c_int, [_P, C.c_int, C.POINTER(TableInfo)]),
    "s615_free_table": (C.c_int, [_P, C.c_int]),
    "s615_fpr_smoke": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int)]),
    "s615_xor_query": (C.c_int, [_P, C.c_int, _P, C.c_size_t, _P]),
    "s615_xor_query_dev": (C.c_int, [_P, C.c_int, _P, C.c_size_t, _P, _P]),
    "s615_mem_info": (C.c_int, [_P, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "s615_unit_candidates": (C.c_int, [C.c_uint64, C.c_int, _P, C.c_size_t,
                                       C.POINTER(C.c_size_t)]),
    "s615_unit_status": (C.c_int, [_P]),
    "s615_617_candidates": (C.c_int, [C.c_uint64, _P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "s615_617_jobs": (C.c_int, [C.c_uint64, C.c_int, _P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "s615_expand_unit": (C.c_int, [_P, _P, C.c_size_t, C.POINTER(C.c_size_t),
                                   C.POINTER(C.c_uint64)]),
    "s615_jobs_open": (C.c_int, [C.c_char_p, C.POINTER(_P), _P]),
    "s615_jobs_next": (C.c_int, [_P, _P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "s615_jobs_close": (C.c_int, [_P, _P]),
    "s615_jobs_write": (C.c_int, [C.c_char_p, _P, C.c_size_t]),
    "s615_run": (C.c_int, [_P, C.c_int, _P, C.c_size_t, C.c_uint, _P, C.c_size_t,
                           C.POINTER(C.c_size_t), C.POINTER(Counters)]),
    "s615_cls5_run": (C.c_int, [_P, C.c_int, _P, C.c_size_t, C.c_uint, _P, C.c_size_t,
                                C.POINTER(C.c_size_t), C.POINTER(Counters)]),
    "s615_cls5_run_noalloc": (C.c_int, [_P, C.c_int, _P, C.c_size_t, C.c_uint, _P, C.c_size_t,
                                        C.POINTER(C.c_size_t), C.POINTER(Counters)]),
    "s615_prepare": (C.c_int, [_P, _P, C.c_size_t, C.POINTER(_P)]),
    "s615_run_batch": (C.c_int, [_P, C.c_int, _P, C.c_uint, _P]),
    "s615_batch_results": (C.c_int, [_P, _P, _P, C.c_size_t, C.POINTER(C.c_size_t),
                                     C.POINTER(Counters)]),
    "s615_batch_free": (C.c_int, [_P, _P]),
    "s615_batch_size": (C.c_int, [_P, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                  C.POINTER(C.c_size_t)]),
    "s615_prepare_band": (C.c_int, [_P, C.c_uint64, C.c_uint64, C.POINTER(_P)]),
    "s615_batch_units": (C.c_int, [_P, _P, _P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "s615_verify": (C.c_int, [_P, _P, C.c_size_t, _P, C.c_size_t, C.c_int, _P, C.c_size_t,
                              C.POINTER(C.c_size_t)]),
    "s615_cls5_verify": (C.c_int, [_P, _P, C.c_size_t, _P, C.c_size_t, C.c_int, _P, C.c_size_t,
                                   C.POINTER(C.c_size_t)]),
    "s615_selftest_host": (C.c_int, []),
    "s615_journal_open": (C.c_int, [C.c_char_p, C.POINTER(_P)]),
    "s615_journal_has": (C.c_int, [_P, _P]),
    "s615_journal_stats": (C.c_int, [_P, _P, _P, _P]),
    "s615_journal_units": (C.c_int, [_P, _P, C.c_size_t, _P]),
    "s615_journal_solutions": (C.c_int, [_P, _P, C.c_size_t, _P]),
    "s615_journal_append": (C.c_int, [_P, _P, C.c_size_t, _P, C.c_size_t, _P, C.c_size_t]),
    "s615_journal_close": (C.c_int, [_P]),
    "s615_serve_start": (C.c_int, [_P, C.c_int, C.c_size_t]),
    "s615_submit": (C.c_int, [_P, C.c_int, _P, C.c_size_t, C.c_uint, C.POINTER(C.c_uint64)]),
    "s615_poll": (C.c_int, [_P, _P, C.c_size_t, C.POINTER(C.c_size_t), C.c_int]),
    "s615_release": (C.c_int, [_P, C.c_uint64]),
    "s615_serve_stop": (C.c_int, [_P]),
}

_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """Load lib/libs615.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} missing: run `make -C six-one-five_b200`"
                          + (" checked" if LIB_PATH.endswith("_checked.so") else ""))
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(status: int, what: str) -> int:
    if status != S615_OK:
        raise S615Error(status, what)
    return status


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def unit_candidates(B: int, cls: int = 5) -> List[int]:
    n = C.c_size_t(0)
    buf = np.zeros(4096, dtype=np.uint64)
    st = lib().s615_unit_candidates(B, cls, _ptr(buf), buf.size, C.byref(n))
    if st not in (S615_OK, -9):
        _check(st, "unit_candidates")
    if n.value > buf.size:
        buf = np.zeros(n.value, dtype=np.uint64)
        _check(lib().s615_unit_candidates(B, cls, _ptr(buf), buf.size, C.byref(n)), "unit_candidates")
    return [int(x) for x in buf[: n.value]]


def make_units(pairs: Iterable[Tuple[int, int]]) -> "C.Array":
    pairs = list(pairs)
    arr = (Unit * max(len(pairs), 1))()
    for i, (B, u) in enumerate(pairs):
        arr[i].cls = 5
        arr[i].kind = 0
        arr[i].B = B
        arr[i].u = u
    return arr, len(pairs)


def make_plant(base: int, e: int, d: int, lim: int, u: int = 0, B: int = 0) -> Unit:
    """A planted cls5 unit: base given, single residue per axis, fmax = the planted value."""
    x = Unit()
    x.cls, x.kind, x.B, x.u = 5, 1, B, u
    for i in range(3):
        x.base[i] = (base >> (64 * i)) & (2**64 - 1)
    x.fmax1, x.fmax2, x.res_e, x.res_d, x.lim = e, d, e % 729, d % 64, lim
    return x


CLS234_MOD = {2: 729, 3: 64, 4: 46656}


def make_plant234(cls: int, base: int, d: int, lim: int, u: int = 0, B: int = 0) -> Unit:
    """A planted cls2-4 unit: base given, one free-term residue, fmax = d."""
    x = Unit()
    x.cls, x.kind, x.B, x.u = cls, 1, B, u
    for i in range(3):
        x.base[i] = (base >> (64 * i)) & (2**64 - 1)
    x.fmax1, x.res_d, x.lim = d, d % CLS234_MOD[cls], lim
    return x


def candidates617(B: int):
    """s615_617_candidates: the (6,1,7) class-5 units of one B (array, count)."""
    n = C.c_size_t(0)
    st = lib().s615_617_candidates(B, None, 0, C.byref(n))
    if st not in (S615_OK, -9):
        _check(st, "617_candidates")
    arr = (Unit * max(n.value, 1))()
    _check(lib().s615_617_candidates(B, C.cast(arr, C.c_void_p), n.value, C.byref(n)),
           "617_candidates")
    return arr, n.value


def make_plant1(c: Sequence[int], lim: int, B: int = 0) -> Unit:
    """A planted class-1 (find4) target: base = 42^6 (c1^6 + c2^6 + c3^6 + c4^6)."""
    base = 42**6 * sum(x**6 for x in c)
    x = Unit()
    x.cls, x.kind, x.B, x.lim = 1, 1, B, lim
    for i in range(3):
        x.base[i] = (base >> (64 * i)) & (2**64 - 1)
    return x


def jobs617(B: int, cls: int):
    """s615_617_jobs: the (6,1,7) class-`cls` (1-4) find4 jobs of one B (array, count)."""
    n = C.c_size_t(0)
    st = lib().s615_617_jobs(B, cls, None, 0, C.byref(n))
    if st not in (S615_OK, -9):
        _check(st, "617_jobs")
    arr = (Unit * max(n.value, 1))()
    _check(lib().s615_617_jobs(B, cls, C.cast(arr, C.c_void_p), n.value, C.byref(n)), "617_jobs")
    return arr, n.value


class TuneEntry(C.Structure):
    _fields_ = [("item_rows", C.c_uint32), ("blocks_per_sm", C.c_uint32), ("ms", C.c_float)]


class JobsInfo(C.Structure):
    _fields_ = [("n_jobs", C.c_uint64), ("min_B", C.c_uint32), ("max_B", C.c_uint32),
                ("binary", C.c_uint32), ("pad", C.c_uint32), ("bad_lines", C.c_uint64)]


def make_job(cls: int, B: int, u: int, T: int, free1: int = 0, free2: int = 0, lim: int = 0) -> Unit:
    """A reduced-T job (kind 2): fourcore_find_v4's Job{cls, B, u, free1, free2, T}."""
    J = Unit()
    J.cls, J.kind, J.B, J.u = cls, S615_KIND_JOB, B, u
    J.base[0], J.base[1] = T % 2**64, T >> 64
    J.res_d, J.res_e, J.lim = free1, free2, lim
    return J


def expand_unit(B: int, u: int, cls: int):
    """s615_expand_unit: (jobs, n, failT) of one Stage-1 unit."""
    unit = Unit()
    unit.cls, unit.B, unit.u = cls, B, u
    n, fail = C.c_size_t(0), C.c_uint64(0)
    st = lib().s615_expand_unit(C.byref(unit), None, 0, C.byref(n), C.byref(fail))
    if st not in (S615_OK, -9):
        _check(st, "expand_unit")
    arr = (Unit * max(n.value, 1))()
    _check(lib().s615_expand_unit(C.byref(unit), C.cast(arr, C.c_void_p), n.value, C.byref(n),
                                  C.byref(fail)), "expand_unit")
    return arr, n.value, fail.value


def expand_units(units):
    """s615_expand_unit over (cls, B, u) Stage-1 units, concatenated in unit
    order: (jobs array, n, failT)."""
    chunks, n, fails = [], 0, 0
    sz = C.sizeof(Unit)
    unit = Unit()
    cnt, fail = C.c_size_t(0), C.c_uint64(0)
    buf = (Unit * 1)()
    for c, B, u in units:
        unit.cls, unit.B, unit.u = c, B, u
        st = lib().s615_expand_unit(C.byref(unit), C.cast(buf, C.c_void_p), len(buf), C.byref(cnt),
                                    C.byref(fail))
        if st == -9:
            buf = (Unit * (cnt.value + cnt.value // 2))()
            st = lib().s615_expand_unit(C.byref(unit), C.cast(buf, C.c_void_p), len(buf), C.byref(cnt),
                                        C.byref(fail))
        _check(st, "expand_unit")
        chunks.append(C.string_at(C.addressof(buf), cnt.value * sz))
        n += cnt.value
        fails += fail.value
    out = (Unit * max(n, 1))()
    if n:
        C.memmove(out, b"".join(chunks), n * sz)
    return out, n, fails


def jobs_write(path: str, jobs, n: int) -> None:
    """s615_jobs_write: a .bbj (binary) or text job file."""
    _check(lib().s615_jobs_write(path.encode(), C.cast(jobs, C.c_void_p), n), "jobs_write")


def jobs_read(path: str, chunk: int = 1 << 16, out=None):
    """Every job of a .bbj or text job file: (array, n, JobsInfo).

    `out`, a Unit array, is filled and returned instead of a new array when a
    .bbj file's jobs fit it (a caller reading file after file reuses one
    buffer; a new array is allocated when they do not fit)."""
    f = C.c_void_p()
    info = JobsInfo()
    _check(lib().s615_jobs_open(path.encode(), C.byref(f), C.byref(info)), "jobs_open")
    parts, n = [], 0
    try:
        if info.binary and info.n_jobs:   # the header's count in one read, then anything after it
            fits = out is not None and len(out) >= info.n_jobs
            first = out if fits else (Unit * info.n_jobs)()
            k = C.c_size_t(0)
            _check(lib().s615_jobs_next(f, C.cast(first, C.c_void_p), info.n_jobs, C.byref(k)),
                   "jobs_next")
            n = k.value
            if n < info.n_jobs:
                return first, n, info
            parts.append(first)
        while True:
            buf = (Unit * chunk)()
            k = C.c_size_t(0)
            _check(lib().s615_jobs_next(f, C.cast(buf, C.c_void_p), chunk, C.byref(k)), "jobs_next")
            if not k.value:
                break
            parts.append(C.string_at(C.addressof(buf), k.value * C.sizeof(Unit)))
            n += k.value
    finally:
        lib().s615_jobs_close(f, C.byref(info))
    if len(parts) == 1 and not isinstance(parts[0], bytes):
        return parts[0], n, info
    whole = (Unit * max(n, 1))()
    off = 0
    for p in parts:   # the header-count read, then the chunks after it
        size = len(p) if isinstance(p, bytes) else info.n_jobs * C.sizeof(Unit)
        C.memmove(C.byref(whole, off), p, size)
        off += size
    return whole, n, info


def jobs617_band(Bs: Iterable[int], classes: Iterable[int] = (1, 2, 3, 4)):
    """The find4 jobs of every B in `Bs` for each (6,1,7) class in `classes`,
    concatenated class by class in B order (array, count)."""
    Bs = list(Bs)
    chunks, n = [], 0
    sz = C.sizeof(Unit)
    for cls in classes:
        for B in Bs:
            arr, k = jobs617(B, cls)
            if k:
                chunks.append(C.string_at(C.addressof(arr), k * sz))
                n += k
    buf = b"".join(chunks)
    out = (Unit * max(n, 1))()
    if n:
        C.memmove(out, buf, len(buf))
    return out, n


def make_units617(triples: Iterable[Tuple[int, int, int]]) -> "C.Array":
    """(6,1,7) Branch-A class-5 candidates (B, u = 14u', w = 6v')."""
    triples = list(triples)
    arr = (Unit * max(len(triples), 1))()
    for i, (B, u, w) in enumerate(triples):
        arr[i].cls, arr[i].kind, arr[i].B, arr[i].u, arr[i].w = S615_CLS_617, 0, B, u, w
    return arr, len(triples)


def make_plant617(base: int, d: int, lim: int, B: int = 0, u: int = 14, w: int = 6) -> Unit:
    """A planted (6,1,7) class-5 target (solve_617_v1.cu:1564-1582): base
    given, one x21 residue, fmax = d, c4 and c3 capped by lim."""
    x = Unit()
    x.cls, x.kind, x.B, x.u, x.w = S615_CLS_617, 1, B, u, w
    for i in range(3):
        x.base[i] = (base >> (64 * i)) & (2**64 - 1)
    x.fmax1, x.res_d, x.lim = d, d % 64, lim
    return x


def s615_hits_copy(ptr, n: int) -> np.ndarray:
    if n == 0:
        return np.zeros(0, dtype=HIT_DTYPE)
    raw = C.string_at(C.cast(ptr, C.c_void_p), n * C.sizeof(Hit))
    return np.frombuffer(raw, dtype=HIT_DTYPE).copy()


def hits_to_array(hits, n: int) -> np.ndarray:
    raw = np.frombuffer(C.string_at(C.addressof(hits), n * C.sizeof(Hit)), dtype=HIT_DTYPE)
    return raw.copy()


class Journal:
    """s615_journal_*: the restart journal of a campaign (append-only, one
    committed block per finished request or chunk)."""

    def __init__(self, path: str):
        self._j = C.c_void_p()
        _check(lib().s615_journal_open(path.encode(), C.byref(self._j)), "journal_open")

    def close(self) -> None:
        if self._j:
            _check(lib().s615_journal_close(self._j), "journal_close")
            self._j = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def has(self, unit: "Unit") -> bool:
        st = lib().s615_journal_has(self._j, C.byref(unit))
        if st < 0:
            _check(st, "journal_has")
        return st == 1

    def stats(self):
        u, h, s = C.c_size_t(0), C.c_size_t(0), C.c_size_t(0)
        _check(lib().s615_journal_stats(self._j, C.byref(u), C.byref(h), C.byref(s)), "journal_stats")
        return u.value, h.value, s.value

    def units(self):
        n = C.c_size_t(0)
        lib().s615_journal_units(self._j, None, 0, C.byref(n))
        arr = (Unit * max(n.value, 1))()
        _check(lib().s615_journal_units(self._j, C.cast(arr, C.c_void_p), n.value, C.byref(n)),
               "journal_units")
        return [arr[i] for i in range(n.value)]

    def solutions(self):
        n = C.c_size_t(0)
        lib().s615_journal_solutions(self._j, None, 0, C.byref(n))
        arr = (Solution * max(n.value, 1))()
        _check(lib().s615_journal_solutions(self._j, C.cast(arr, C.c_void_p), n.value, C.byref(n)),
               "journal_solutions")
        return [arr[i] for i in range(n.value)]

    def append(self, units, n: int, hits=None, sols=()) -> None:
        h = np.ascontiguousarray(hits if hits is not None else np.zeros(0, dtype=HIT_DTYPE))
        sarr = (Solution * max(len(sols), 1))(*sols)
        _check(lib().s615_journal_append(self._j, C.cast(units, C.c_void_p), n, _ptr(h), h.size,
                                         C.cast(sarr, C.c_void_p), len(sols)), "journal_append")


class Engine:
    """One device context (s615_open ... s615_close)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self._ctx = C.c_void_p()
        _check(lib().s615_open(device, hbm_budget, C.byref(self._ctx)), "s615_open")

    def close(self) -> None:
        if self._ctx:
            lib().s615_close(self._ctx)
            self._ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def launches(self) -> int:
        return int(lib().s615_launch_count(self._ctx))

    def check_flags(self) -> int:
        """S615_CHK_* bits the checked build's kernels set since the last call
        (0 in the default build)."""
        f = C.c_uint32(0)
        _check(lib().s615_check_flags(self._ctx, C.byref(f)), "check_flags")
        return f.value

    # ---- tables ----
    def load_table(self, path: str, expected_N: int = 0, layout: int = LAYOUT_AUTO) -> int:
        tid = C.c_int(0)
        _check(lib().s615_load_table(self._ctx, path.encode(), expected_N, layout, C.byref(tid)),
               f"load_table {path}")
        return tid.value

    def build_table(self, N: int, r: int, layout: int = LAYOUT_AUTO) -> int:
        tid = C.c_int(0)
        _check(lib().s615_build_table(self._ctx, N, r, layout, C.byref(tid)), "build_table")
        return tid.value

    def build_table_keys(self, keys, r: int, base_seed: int = 0x615615615615615,
                         layout: int = LAYOUT_AUTO) -> int:
        k = np.ascontiguousarray(np.asarray(keys, dtype=np.uint64))
        tid = C.c_int(0)
        _check(lib().s615_build_table_keys(self._ctx, _ptr(k), k.size, r, base_seed, layout,
                                           C.byref(tid)), "build_table_keys")
        return tid.value

    def save_table(self, tid: int, path: str) -> None:
        _check(lib().s615_save_table(self._ctx, tid, path.encode()), "save_table")

    def build_table_sharded(self, N: int, r: int, shards: int, layout: int = LAYOUT_AUTO) -> int:
        """A pair-space shard set: S xor tables, a probe queries its key's shard."""
        tid = C.c_int(0)
        _check(lib().s615_build_table_sharded(self._ctx, N, r, shards, layout, C.byref(tid)),
               "build_table_sharded")
        return tid.value

    def build_table_shard_range(self, N: int, r: int, shards: int, lo: int, hi: int,
                                layout: int = LAYOUT_AUTO) -> int:
        """Shards [lo, hi) of an S-shard set: one GPU's part of a set split over GPUs."""
        tid = C.c_int(0)
        _check(lib().s615_build_table_shard_range(self._ctx, N, r, shards, lo, hi, layout,
                                                  C.byref(tid)), "build_table_shard_range")
        return tid.value

    def load_table_shards(self, paths, expected_N: int = 0, layout: int = LAYOUT_AUTO) -> int:
        arr = (C.c_char_p * len(paths))(*[p.encode() for p in paths])
        tid = C.c_int(0)
        _check(lib().s615_load_table_shards(self._ctx, arr, len(paths), expected_N, layout,
                                            C.byref(tid)), "load_table_shards")
        return tid.value

    def autotune(self, tid: int, units, n: int, flags: int = 0):
        """s615_autotune: every trial (item_rows, blocks_per_sm, ms) and the chosen one."""
        table = (TuneEntry * 64)()
        k = C.c_size_t(0)
        best = TuneEntry()
        _check(lib().s615_autotune(self._ctx, tid, C.cast(units, C.c_void_p), n, flags,
                                   C.cast(table, C.c_void_p), 64, C.byref(k), C.byref(best)), "autotune")
        rows = [(table[i].item_rows, table[i].blocks_per_sm, table[i].ms) for i in range(k.value)]
        return rows, (best.item_rows, best.blocks_per_sm, best.ms)

    def tune_reset(self) -> None:
        _check(lib().s615_tune_reset(self._ctx), "tune_reset")

    def set_probe_groups(self, tid: int, groups: int) -> None:
        """Probe a shard set in `groups` passes (0: from its size)."""
        _check(lib().s615_set_probe_groups(self._ctx, tid, groups), "set_probe_groups")

    def save_table_shard(self, tid: int, shard: int, path: str) -> None:
        _check(lib().s615_save_table_shard(self._ctx, tid, shard, path.encode()), "save_table_shard")

    def export_table(self, tid: int):
        """(64 header bytes, packed cell bytes as uint8 ndarray)."""
        hdr = Header()
        n = C.c_size_t(0)
        _check(lib().s615_export_table(self._ctx, tid, C.byref(hdr), None, 0, C.byref(n)),
               "export_table")
        buf = np.zeros(n.value, dtype=np.uint8)
        _check(lib().s615_export_table(self._ctx, tid, C.byref(hdr), _ptr(buf), buf.size,
                                       C.byref(n)), "export_table")
        return bytes(hdr), buf

    def table_info(self, tid: int) -> TableInfo:
        info = TableInfo()
        _check(lib().s615_get_table_info(self._ctx, tid, C.byref(info)), "table_info")
        return info

    def free_table(self, tid: int) -> None:
        _check(lib().s615_free_table(self._ctx, tid), "free_table")

    def query(self, tid: int, keys) -> np.ndarray:
        k = np.ascontiguousarray(np.asarray(keys, dtype=np.uint64))
        out = np.zeros(k.size, dtype=np.uint8)
        _check(lib().s615_xor_query(self._ctx, tid, _ptr(k), k.size, _ptr(out)), "xor_query")
        return out

    # ---- peels (classes 2-5) ----
    def run(self, tid: int, units, n: int, flags: int = 0, hit_cap: int = 1 << 20,
            entry: str = "s615_run"):
        hits = (Hit * max(hit_cap, 1))()
        nh = C.c_size_t(0)
        ctr = Counters()
        st = getattr(lib(), entry)(self._ctx, tid, C.cast(units, C.c_void_p), n, flags,
                                   C.cast(hits, C.c_void_p), hit_cap, C.byref(nh), C.byref(ctr))
        _check(st, entry)
        return hits_to_array(hits, nh.value), ctr

    def run_band(self, tid: int, B_lo: int, B_hi: int, flags: int = 0, hit_cap: int = 1 << 20):
        """Stage-1 class-5 units of B in [B_lo, B_hi] generated on the device
        (s615_prepare_band), one run: (unit array, n, hits, counters)."""
        b = C.c_void_p()
        _check(lib().s615_prepare_band(self._ctx, B_lo, B_hi, C.byref(b)), "prepare_band")
        try:
            n = C.c_size_t(0)
            lib().s615_batch_units(self._ctx, b, None, 0, C.byref(n))
            units = (Unit * max(n.value, 1))()
            _check(lib().s615_batch_units(self._ctx, b, C.cast(units, C.c_void_p), n.value,
                                          C.byref(n)), "batch_units")
            _check(lib().s615_run_batch(self._ctx, tid, b, flags, None), "run_batch")
            hits = (Hit * max(hit_cap, 1))()
            nh = C.c_size_t(0)
            ctr = Counters()
            _check(lib().s615_batch_results(self._ctx, b, C.cast(hits, C.c_void_p), hit_cap,
                                            C.byref(nh), C.byref(ctr)), "batch_results")
            return units, n.value, hits_to_array(hits, nh.value), ctr
        finally:
            lib().s615_batch_free(self._ctx, b)

    def cls5_run(self, tid: int, units, n: int, flags: int = 0, hit_cap: int = 1 << 20):
        return self.run(tid, units, n, flags, hit_cap, entry="s615_cls5_run")

    # ---- serving (s615_serve_start / submit / poll / release / serve_stop)
    def serve_start(self, slots: int = 2, max_batch_units: int = 0) -> None:
        _check(lib().s615_serve_start(self._ctx, slots, max_batch_units), "serve_start")

    def submit(self, tid: int, units, n: int, flags: int = 0) -> int:
        t = C.c_uint64(0)
        _check(lib().s615_submit(self._ctx, tid, C.cast(units, C.c_void_p), n, flags, C.byref(t)),
               "submit")
        return t.value

    def poll(self, cap: int = 64, wait_ms: int = 100):
        """Finished requests: list of dicts with the hits and solutions copied
        out (the library's copies are released)."""
        out = (Result * cap)()
        n = C.c_size_t(0)
        _check(lib().s615_poll(self._ctx, C.cast(out, C.c_void_p), cap, C.byref(n), wait_ms), "poll")
        res = []
        for i in range(n.value):
            r = out[i]
            hits = (s615_hits_copy(r.hits, r.n_hits))
            sols = [Solution.from_buffer_copy(r.solutions[k]) for k in range(r.n_solutions)]
            res.append({"ticket": r.ticket, "status": r.status, "table_id": r.table_id,
                        "n_units": r.n_units, "hits": hits, "solutions": sols,
                        "counters": Counters.from_buffer_copy(r.counters),
                        "batch_requests": r.batch_requests, "queued_ms": r.queued_ms,
                        "latency_ms": r.latency_ms})
            _check(lib().s615_release(self._ctx, r.ticket), "release")
        return res

    def serve_stop(self) -> None:
        _check(lib().s615_serve_stop(self._ctx), "serve_stop")

    def verify(self, units, n_units: int, hits: np.ndarray, N: int, cap: int = 4096):
        h = np.ascontiguousarray(hits.astype(HIT_DTYPE))
        out = (Solution * cap)()
        no = C.c_size_t(0)
        _check(lib().s615_verify(self._ctx, C.cast(units, C.c_void_p), n_units, _ptr(h), h.size, N,
                                 C.cast(out, C.c_void_p), cap, C.byref(no)), "verify")
        return [out[i] for i in range(no.value)]


def solution_line(s: Solution) -> str:
    """The reference's SOLUTION line (fourcore_cls5_gpu_v4.cu:533-536,
    fourcore_find_v4.cu:450-453, solve_617_v1.cu:1101-1103; the (6,1,7)
    class-5 shape prints as cls=5 there); plants print a PLANT line."""
    if s.kind == 1:
        if s.cls == 5:
            return f"PLANT unit={s.unit} d={s.d} e={s.e} c1={s.c1} c2={s.c2}"
        if s.cls == S615_CLS_617:
            return (f"PLANT cls=7 unit={s.unit} d={s.d} c1={s.c1} c2={s.c2} c3={s.c3} "
                    f"c4={s.c4}")
        if s.cls == 1:
            return f"PLANT cls=1 unit={s.unit} c1={s.c1} c2={s.c2} c3={s.c3} c4={s.c4}"
        return f"PLANT cls={s.cls} unit={s.unit} d={s.d} c1={s.c1} c2={s.c2} c3={s.c3}"
    if s.kind == S615_KIND_JOB:   # an exact T match whose full identity does not hold
        return (f"EXACT cls={s.cls} unit={s.unit} d={s.d} e={s.e} c1={s.c1} c2={s.c2} "
                f"c3={s.c3} c4={s.c4}")
    a = list(s.a)
    if s.cls == S615_CLS_617_FIND4:   # the (6,1,7) class is in d
        terms = " ".join(f"a{i + 1}={a[i]}" for i in range(7))
        return (f"SOLUTION cls={s.d} B={s.B} {terms} (anchor={s.u}) gcd={s.gcd} "
                f"{'primitive' if s.gcd == 1 else 'NON-PRIMITIVE'}")
    if s.cls == S615_CLS_617:
        terms = " ".join(f"a{i + 1}={a[i]}" for i in range(7))
        return (f"SOLUTION cls=5 B={s.B} {terms} (anchor={s.u}) gcd={s.gcd} "
                f"{'primitive' if s.gcd == 1 else 'NON-PRIMITIVE'}")
    return (f"SOLUTION cls={s.cls} B={s.B} u={s.u} a1={a[0]} a2={a[1]} a3={a[2]} a4={a[3]} "
            f"a5={a[4]} gcd={s.gcd} {'primitive' if s.gcd == 1 else 'NON-PRIMITIVE'}")
