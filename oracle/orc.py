"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference leg.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


class OrcHeader(C.Structure):
    _fields_ = [("magic", C.c_uint32), ("version", C.c_uint32), ("kind", C.c_uint32),
                ("r", C.c_uint32), ("w", C.c_uint32), ("N", C.c_uint32),
                ("n_keys", C.c_uint64), ("m_cells", C.c_uint64), ("mix_seed", C.c_uint64),
                ("shard_count", C.c_uint32), ("shard_index", C.c_uint32),
                ("shard_mode", C.c_uint32), ("reserved", C.c_uint32)]


class OrcUnit5(C.Structure):
    _fields_ = [("B", C.c_uint64), ("u", C.c_uint64), ("base", C.c_uint64 * 3),
                ("lim", C.c_uint32), ("mod1", C.c_uint32), ("mod2", C.c_uint32),
                ("fmax1", C.c_uint32), ("fmax2", C.c_uint32), ("nres1", C.c_uint32),
                ("nres2", C.c_uint32), ("res", C.c_uint32 * 24), ("planted", C.c_uint32)]


class OrcHit(C.Structure):
    _fields_ = [("unit", C.c_uint32), ("a", C.c_uint32), ("b", C.c_uint32), ("d", C.c_uint32),
                ("e", C.c_uint32), ("fp", C.c_uint64)]


class OrcJob3(C.Structure):
    _fields_ = [("cls", C.c_uint32), ("lim", C.c_uint32), ("B", C.c_uint64), ("u", C.c_uint64),
                ("d", C.c_uint64), ("T", C.c_uint64 * 2), ("lo", C.c_uint32), ("hi", C.c_uint32)]


class OrcHit3(C.Structure):
    _fields_ = [("job", C.c_uint32), ("c3", C.c_uint32), ("fp", C.c_uint64)]


class OrcHit4(C.Structure):
    _fields_ = [("job", C.c_uint32), ("c3", C.c_uint32), ("c4", C.c_uint32), ("pad", C.c_uint32),
                ("fp", C.c_uint64)]


class OrcJob(C.Structure):
    _fields_ = [("cls", C.c_uint32), ("lim", C.c_uint32), ("B", C.c_uint64), ("u", C.c_uint64),
                ("free1", C.c_uint64), ("free2", C.c_uint64), ("T", C.c_uint64 * 2)]


class OrcJob617(C.Structure):
    _fields_ = [("Q4", C.c_uint64 * 2), ("B", C.c_uint32), ("u", C.c_uint32), ("w", C.c_uint32),
                ("cls", C.c_uint32), ("c5", C.c_uint32), ("lim", C.c_uint32), ("lo", C.c_uint32),
                ("hi", C.c_uint32)]


class OrcCand617(C.Structure):
    _fields_ = [("base", C.c_uint64 * 2), ("B", C.c_uint32), ("u", C.c_uint32), ("w", C.c_uint32),
                ("lim", C.c_uint32), ("mod1", C.c_uint32), ("fmax1", C.c_uint32),
                ("nres1", C.c_uint32), ("pad", C.c_uint32), ("res", C.c_uint32 * 24)]


class OrcHit617(C.Structure):
    _fields_ = [("cand", C.c_uint32), ("a", C.c_uint32), ("b", C.c_uint32), ("c", C.c_uint32),
                ("d", C.c_uint32), ("e", C.c_uint32), ("fp", C.c_uint64)]


assert C.sizeof(OrcUnit5) == 168 and C.sizeof(OrcHit) == 32
assert C.sizeof(OrcCand617) == 144 and C.sizeof(OrcHit617) == 32

_P = C.c_void_p
_SIG = {
    "orc_unit_candidates": (C.c_size_t, [C.c_uint64, C.c_int, _P, C.c_size_t]),
    "orc_seed_count": (C.c_size_t, [C.c_uint64, C.c_int]),
    "orc_pack_unit5": (C.c_int, [C.c_uint64, C.c_uint64, C.POINTER(OrcUnit5)]),
    "orc_pow6_192": (None, [C.c_uint32, _P]),
    "orc_T_peel2": (C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, _P]),
    "orc_funnel_fp": (C.c_uint64, [C.POINTER(OrcUnit5), C.c_uint32, C.c_uint32, C.POINTER(C.c_int)]),
    "orc_gate_tables": (None, [_P, _P]),
    "orc_mix64": (C.c_uint64, [C.c_uint64]),
    "orc_capacity_for": (C.c_size_t, [C.c_size_t]),
    "orc_packed_bytes": (C.c_size_t, [C.c_uint64, C.c_uint32]),
    "orc_build_xor": (_P, [_P, C.c_size_t, C.c_int, C.c_uint64, C.c_int]),
    "orc_build_pairs": (_P, [C.c_int, C.c_int]),
    "orc_build_pairs_shard": (_P, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64]),
    "orc_shard_set": (_P, [_P, C.c_int, C.c_uint64]),
    "orc_shard_of": (C.c_uint32, [C.c_uint64, C.c_uint64, C.c_uint32]),
    "orc_load": (_P, [C.c_char_p, C.c_int]),
    "orc_from_memory": (_P, [C.POINTER(OrcHeader), _P, C.c_size_t]),
    "orc_save": (C.c_int, [_P, C.c_char_p]),
    "orc_free": (None, [_P]),
    "orc_table_header": (None, [_P, C.POINTER(OrcHeader)]),
    "orc_table_bytes": (C.POINTER(C.c_uint8), [_P, C.POINTER(C.c_size_t)]),
    "orc_query": (None, [_P, _P, C.c_size_t, _P]),
    "orc_fpr_smoke": (C.c_int, [_P]),
    "orc_residue": (None, [_P, _P, C.c_size_t, _P]),
    "orc_mt64": (None, [C.c_uint64, C.c_size_t, _P]),
    "orc_cls5_run": (C.c_size_t, [_P, _P, C.c_size_t, C.c_int, C.c_int, _P, C.c_size_t, _P]),
    "orc_cls5_verify": (C.c_size_t, [_P, _P, C.c_size_t, C.c_int, C.c_int, C.c_char_p, C.c_size_t]),
    "orc_expand_cls234": (C.c_size_t, [C.c_uint64, C.c_uint64, C.c_int, _P, C.c_size_t]),
    "orc_find3_run": (C.c_size_t, [_P, _P, C.c_size_t, C.c_int, C.c_int, _P, C.c_size_t, _P]),
    "orc_expand_cls1": (C.c_size_t, [C.c_uint64, C.c_uint64, _P, C.c_size_t]),
    "orc_find4_run": (C.c_size_t, [_P, _P, C.c_size_t, C.c_int, C.c_int, C.c_int, _P, C.c_size_t,
                                   _P]),
    "orc_617_jobs": (C.c_size_t, [C.c_uint64, C.c_int, _P, C.c_size_t]),
    "orc_expand_unit": (C.c_size_t, [C.c_uint64, C.c_uint64, C.c_int, _P, C.c_size_t, _P]),
    "orc_jobs_run": (C.c_size_t, [_P, _P, C.c_size_t, C.c_int, C.c_int, C.c_int, _P, C.c_size_t,
                                  _P]),
    "orc_jobs_verify": (C.c_size_t, [_P, _P, C.c_size_t, C.c_int, C.c_char_p, C.c_size_t, _P]),
    "orc_617_find4_run": (C.c_size_t, [_P, _P, C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_int, _P,
                                       C.c_size_t, _P]),
    "orc_617_find4_verify": (C.c_size_t, [_P, _P, C.c_size_t, C.c_int, C.c_char_p, C.c_size_t, _P]),
    "orc_617_cands": (C.c_size_t, [C.c_uint64, _P, C.c_size_t]),
    "orc_617_run": (C.c_size_t, [_P, _P, C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_int, _P,
                                 C.c_size_t, _P]),
    "orc_617_verify": (C.c_size_t, [_P, _P, C.c_size_t, C.c_int, C.c_int, C.c_char_p, C.c_size_t,
                                    _P]),
}

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True,
                           stdout=subprocess.DEVNULL)
        L = C.CDLL(LIB)
        for k, (res, args) in _SIG.items():
            f = getattr(L, k)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


SHARD_SEED = 0x615615615615615   # the routing seed of pair-space shards


class Table:
    def __init__(self, handle):
        if not handle:
            raise RuntimeError("oracle table build/load failed")
        self.h = handle

    @classmethod
    def build_pairs(cls, N: int, r: int) -> "Table":
        return cls(lib().orc_build_pairs(N, r))

    @classmethod
    def build_pairs_shard(cls, N: int, r: int, S: int, s: int, seed: int = SHARD_SEED) -> "Table":
        """Shard s of S: the pair keys with mix64(key + seed) % S == s."""
        return cls(lib().orc_build_pairs_shard(N, r, S, s, seed))

    @classmethod
    def shard_set(cls, parts, seed: int = SHARD_SEED) -> "Table":
        """A table whose probes go to parts[mix64(key + seed) % S] (parts stay
        referenced; None marks a shard held elsewhere)."""
        arr = (C.c_void_p * len(parts))(*[p.h if p is not None else None for p in parts])
        t = cls(lib().orc_shard_set(arr, len(parts), seed))
        t.parts = [p for p in parts if p is not None]
        return t

    @classmethod
    def build_keys(cls, keys, r: int, base_seed: int = 0x615615615615615, tries: int = 64):
        k = np.ascontiguousarray(np.asarray(keys, dtype=np.uint64))
        return cls(lib().orc_build_xor(_ptr(k), k.size, r, base_seed, tries))

    @classmethod
    def load(cls, path: str, expected_N: int = 0) -> "Table":
        return cls(lib().orc_load(path.encode(), expected_N))

    @classmethod
    def from_memory(cls, header_bytes: bytes, packed: np.ndarray) -> "Table":
        h = OrcHeader.from_buffer_copy(header_bytes)
        p = np.ascontiguousarray(packed, dtype=np.uint8)
        return cls(lib().orc_from_memory(C.byref(h), _ptr(p), p.size))

    def save(self, path: str) -> None:
        if not lib().orc_save(self.h, path.encode()):
            raise RuntimeError("oracle save failed")

    @property
    def header(self) -> OrcHeader:
        h = OrcHeader()
        lib().orc_table_header(self.h, C.byref(h))
        return h

    def bytes(self) -> bytes:
        n = C.c_size_t(0)
        p = lib().orc_table_bytes(self.h, C.byref(n))
        return C.string_at(p, n.value)

    def query(self, keys) -> np.ndarray:
        k = np.ascontiguousarray(np.asarray(keys, dtype=np.uint64))
        out = np.zeros(k.size, dtype=np.uint8)
        lib().orc_query(self.h, _ptr(k), k.size, _ptr(out))
        return out

    def residue(self, keys) -> np.ndarray:
        """cell(i0) ^ cell(i1) ^ cell(i2) ^ fingerprint per key (0 iff "maybe")."""
        k = np.ascontiguousarray(np.asarray(keys, dtype=np.uint64))
        out = np.zeros(k.size, dtype=np.uint64)
        lib().orc_residue(self.h, _ptr(k), k.size, _ptr(out))
        return out

    def fpr_smoke(self) -> int:
        return lib().orc_fpr_smoke(self.h)

    def __del__(self):
        try:
            if self.h:
                lib().orc_free(self.h)
        except Exception:
            pass


def mt64(seed: int, n: int) -> np.ndarray:
    """n draws of std::mt19937_64(seed) (the reference FPR test's non-key stream)."""
    out = np.zeros(n, dtype=np.uint64)
    lib().orc_mt64(seed, n, _ptr(out))
    return out


def shard_of(key: int, S: int, seed: int = SHARD_SEED) -> int:
    """shard_of_key (spike/ribbon/shard.hpp:19-24)."""
    return lib().orc_shard_of(key, seed, S)


def pack_unit(B: int, u: int):
    U = OrcUnit5()
    ok = lib().orc_pack_unit5(B, u, C.byref(U))
    return U if ok else None


def plant_unit(base: int, e: int, d: int, lim: int, B: int = 0, u: int = 0) -> OrcUnit5:
    U = OrcUnit5()
    U.B, U.u = B, u
    for i in range(3):
        U.base[i] = (base >> (64 * i)) & (2**64 - 1)
    U.lim, U.mod1, U.mod2 = lim, 729, 64
    U.fmax1, U.fmax2, U.nres1, U.nres2 = e, d, 1, 1
    U.res[0], U.res[1] = e % 729, d % 64
    U.planted = 1
    return U


def units_array(units):
    arr = (OrcUnit5 * max(len(units), 1))()
    for i, U in enumerate(units):
        arr[i] = U
    return arr


HIT_DTYPE = np.dtype([("unit", "<u4"), ("a", "<u4"), ("b", "<u4"), ("d", "<u4"), ("e", "<u4"),
                      ("pad", "<u4"), ("fp", "<u8")])


def cls5_run(table: Table, units_arr, n: int, use_gate: bool = True, threads: int = 0,
             cap: int = 1 << 22):
    """k_cls5_192 semantics on the CPU: (hits ndarray, [calls, gated, probes])."""
    hits = (OrcHit * cap)()
    ctr = np.zeros(3, dtype=np.uint64)
    nh = lib().orc_cls5_run(table.h, C.cast(units_arr, C.c_void_p), n, 1 if use_gate else 0,
                            threads, C.cast(hits, C.c_void_p), cap, _ptr(ctr))
    if nh > cap:
        raise RuntimeError("oracle hit buffer overflow")
    raw = np.frombuffer(C.string_at(C.addressof(hits), nh * C.sizeof(OrcHit)), dtype=HIT_DTYPE)
    return raw.copy(), [int(x) for x in ctr]


def cls5_verify(units_arr, hits: np.ndarray, N: int, stop_first: bool = False):
    h = np.ascontiguousarray(hits.astype(HIT_DTYPE))
    buf = C.create_string_buffer(1 << 20)
    lib().orc_cls5_verify(C.cast(units_arr, C.c_void_p), _ptr(h), h.size, N,
                          1 if stop_first else 0, buf, len(buf))
    return [l for l in buf.value.decode().splitlines() if l]


def gate_tables():
    g504 = np.zeros(504, dtype=np.uint8)
    g247 = np.zeros(247, dtype=np.uint8)
    lib().orc_gate_tables(_ptr(g504), _ptr(g247))
    return g504, g247


def pow6_192(x: int) -> int:
    out = np.zeros(3, dtype=np.uint64)
    lib().orc_pow6_192(x, _ptr(out))
    return int(out[0]) | (int(out[1]) << 64) | (int(out[2]) << 128)


def unit_candidates(B: int, cls: int = 5):
    buf = np.zeros(8192, dtype=np.uint64)
    n = lib().orc_unit_candidates(B, cls, _ptr(buf), buf.size)
    return [int(x) for x in buf[:n]]


def seed_count(B: int, cls: int) -> int:
    return int(lib().orc_seed_count(B, cls))


HIT617_DTYPE = np.dtype([("cand", "<u4"), ("a", "<u4"), ("b", "<u4"), ("c", "<u4"), ("d", "<u4"),
                         ("e", "<u4"), ("fp", "<u8")])


def cands617(B: int):
    """gen_class_cands(cls=5) of solve_617_v1.cu:885-906 for one B (full u band)."""
    n = lib().orc_617_cands(B, None, 0)
    arr = (OrcCand617 * max(n, 1))()
    lib().orc_617_cands(B, C.cast(arr, C.c_void_p), n)
    return arr, n


def concat617(parts):
    """One candidate array from [(array, count), ...]."""
    n = sum(k for _, k in parts)
    out = (OrcCand617 * max(n, 1))()
    i = 0
    for arr, k in parts:
        C.memmove(C.byref(out, i * C.sizeof(OrcCand617)), arr, k * C.sizeof(OrcCand617))
        i += k
    return out, n


def run617(table: Table, cands, n: int, use_gate: bool = True, use_tri: bool = True,
           zmax: int = 1, threads: int = 0, cap: int = 1 << 20):
    """k_find4_cls5 semantics: (hits, [calls, gated, probes, tri_total, tri_skipped])."""
    hits = (OrcHit617 * cap)()
    ctr = np.zeros(5, dtype=np.uint64)
    nh = lib().orc_617_run(table.h, C.cast(cands, C.c_void_p), n, int(use_gate), int(use_tri),
                           zmax, threads, C.cast(hits, C.c_void_p), cap, _ptr(ctr))
    if nh > cap:
        raise RuntimeError("oracle hit buffer overflow")
    raw = np.frombuffer(C.string_at(C.addressof(hits), nh * C.sizeof(OrcHit617)),
                        dtype=HIT617_DTYPE)
    return raw.copy(), [int(x) for x in ctr]


def verify617(cands, hits: np.ndarray, N: int, planted: bool = False, stats: list = None):
    """SOLUTION (or PLANT617) lines; stats, if given, receives [exact, fp_false]."""
    h = np.ascontiguousarray(hits.astype(HIT617_DTYPE))
    buf = C.create_string_buffer(1 << 20)
    st = np.zeros(2, dtype=np.uint64)
    lib().orc_617_verify(C.cast(cands, C.c_void_p), _ptr(h), h.size, N, int(planted), buf, len(buf),
                         _ptr(st))
    if stats is not None:
        stats[:] = [int(st[0]), int(st[1])]
    return [l for l in buf.value.decode().splitlines() if l]


HIT4_DTYPE = np.dtype([("job", "<u4"), ("c3", "<u4"), ("c4", "<u4"), ("pad", "<u4"), ("fp", "<u8")])


def jobs_cls1(units):
    """expand_unit(cls 1) + make_cand(mode 4) for (B, u) pairs: (jobs, n, unit index per job)."""
    buf = (OrcJob3 * 1)()
    jobs, origin = [], []
    for k, (B, u) in enumerate(units):
        if lib().orc_expand_cls1(B, u, C.cast(buf, C.c_void_p), 1):
            jobs.append(OrcJob3.from_buffer_copy(buf[0]))
            origin.append(k)
    arr = (OrcJob3 * max(len(jobs), 1))()
    for i, J in enumerate(jobs):
        arr[i] = J
    return arr, len(jobs), origin


def run_find4(table: Table, jobs, n: int, use_gate: bool = True, ref_tiles: bool = False,
              threads: int = 0, cap: int = 1 << 20):
    """k_find4 semantics: (hits, [calls, gated, probes])."""
    hits = (OrcHit4 * cap)()
    ctr = np.zeros(3, dtype=np.uint64)
    nh = lib().orc_find4_run(table.h, C.cast(jobs, C.c_void_p), n, int(use_gate), int(ref_tiles),
                             threads, C.cast(hits, C.c_void_p), cap, _ptr(ctr))
    if nh > cap:
        raise RuntimeError("oracle hit buffer overflow")
    raw = np.frombuffer(C.string_at(C.addressof(hits), nh * C.sizeof(OrcHit4)), dtype=HIT4_DTYPE)
    return raw.copy(), [int(x) for x in ctr]


def expand_unit(B: int, u: int, cls: int):
    """expand_unit of fourcore_find_v4: (jobs, n, failT) of one Stage-1 unit."""
    fail = C.c_uint64(0)
    n = lib().orc_expand_unit(B, u, cls, None, 0, C.byref(fail))
    arr = (OrcJob * max(n, 1))()
    lib().orc_expand_unit(B, u, cls, C.cast(arr, C.c_void_p), n, C.byref(fail))
    return arr, n, fail.value


def concat_jobs(parts):
    """One OrcJob array from (array, n, ...) parts."""
    n = sum(p[1] for p in parts)
    out = (OrcJob * max(n, 1))()
    k = 0
    for p in parts:
        C.memmove(C.byref(out, k * C.sizeof(OrcJob)), p[0], p[1] * C.sizeof(OrcJob))
        k += p[1]
    return out, n


def run_jobs(table: Table, jobs, n: int, use_gate: bool = True, ref_tiles: bool = False,
             threads: int = 0, cap: int = 1 << 20):
    """run_batch over reduced-T jobs (find2/find3/find4 by class): (hits
    {job, c3, c4, fp}, [calls, gated, probes])."""
    hits = (OrcHit4 * cap)()
    ctr = np.zeros(3, dtype=np.uint64)
    nh = lib().orc_jobs_run(table.h, C.cast(jobs, C.c_void_p), n, int(use_gate), int(ref_tiles),
                            threads, C.cast(hits, C.c_void_p), cap, _ptr(ctr))
    if nh > cap:
        raise RuntimeError("oracle hit buffer overflow")
    raw = np.frombuffer(C.string_at(C.addressof(hits), nh * C.sizeof(OrcHit4)), dtype=HIT4_DTYPE)
    return raw.copy(), [int(x) for x in ctr]


def verify_jobs(jobs, hits: np.ndarray, N: int):
    """(exact matches, SOLUTION lines) of run_batch's filter + report_solution."""
    arr = (OrcHit4 * max(len(hits), 1))()
    for i, h in enumerate(hits):
        arr[i].job, arr[i].c3, arr[i].c4, arr[i].fp = int(h["job"]), int(h["c3"]), int(h["c4"]), int(h["fp"])
    buf = C.create_string_buffer(1 << 20)
    nl = C.c_size_t(0)
    exact = lib().orc_jobs_verify(C.cast(jobs, C.c_void_p), C.cast(arr, C.c_void_p), len(hits), N,
                                  buf, len(buf), C.byref(nl))
    return exact, [l for l in buf.value.decode().splitlines() if l]


def jobs617(B: int, cls: int):
    """gen_class_cands(cls in 1..4) of solve_617_v1.cu with the c5 expansion: find4 jobs."""
    n = lib().orc_617_jobs(B, cls, None, 0)
    arr = (OrcJob617 * max(n, 1))()
    lib().orc_617_jobs(B, cls, C.cast(arr, C.c_void_p), n)
    return arr, n


def concat_jobs617(parts):
    n = sum(k for _, k in parts)
    out = (OrcJob617 * max(n, 1))()
    i = 0
    for arr, k in parts:
        C.memmove(C.byref(out, i * C.sizeof(OrcJob617)), arr, k * C.sizeof(OrcJob617))
        i += k
    return out, n


def run617_find4(table: Table, jobs, n: int, use_gate: bool = True, use_tri: bool = True,
                 ymax: int = 1, threads: int = 0, cap: int = 1 << 20):
    hits = (OrcHit4 * cap)()
    ctr = np.zeros(5, dtype=np.uint64)
    nh = lib().orc_617_find4_run(table.h, C.cast(jobs, C.c_void_p), n, int(use_gate), int(use_tri),
                                 ymax, threads, C.cast(hits, C.c_void_p), cap, _ptr(ctr))
    if nh > cap:
        raise RuntimeError("oracle hit buffer overflow")
    raw = np.frombuffer(C.string_at(C.addressof(hits), nh * C.sizeof(OrcHit4)), dtype=HIT4_DTYPE)
    return raw.copy(), [int(x) for x in ctr]


def verify617_find4(jobs, hits: np.ndarray, N: int, stats: list = None):
    h = np.ascontiguousarray(hits.astype(HIT4_DTYPE))
    buf = C.create_string_buffer(1 << 20)
    st = np.zeros(2, dtype=np.uint64)
    lib().orc_617_find4_verify(C.cast(jobs, C.c_void_p), _ptr(h), h.size, N, buf, len(buf), _ptr(st))
    if stats is not None:
        stats[:] = [int(st[0]), int(st[1])]
    return [l for l in buf.value.decode().splitlines() if l]
