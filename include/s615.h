/*
 * s615.h -- C ABI of the B200 engine for the (6,1,5) class-5 meet-in-the-middle
 * search: 2-D (d,e) free peel, mod-124,488 residue gate, xor-filter probe and
 * exact verification, plus the device xor-filter builder the path consumes.
 *
 * Naming follows the reference (cavedave/six-one-five): e is the x14 free
 * term (residues mod 3^6, e <= (B-1)/14), d is the x21 free term (residues mod
 * 2^6, d <= (B-1)/21).  A unit is a Stage-1 pair (B,u); its grid point (e,d)
 * has R = B^6 - u^6 - (14e)^6 - (21d)^6 and T = R / 42^6.
 *
 * Conventions: every call returns an int status (S615_OK or a negative
 * S615_E_* code); nothing here calls exit().  Plain pointers and sizes only.
 * Host-buffer entry points copy in and out themselves; *_dev entry points take
 * device pointers and a cudaStream_t passed as void*.
 * A context is not thread-safe, except that s615_submit may be called from any
 * thread while one thread calls s615_poll (serving, below).
 */
#ifndef S615_H
#define S615_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define S615_OK 0
#define S615_E_ARG (-1)        /* bad argument */
#define S615_E_IO (-2)         /* cannot open / short read or write */
#define S615_E_FORMAT (-3)     /* bad header, kind, version, or unit shape */
#define S615_E_N_MISMATCH (-4) /* table file N != expected N */
#define S615_E_FPR_SMOKE (-5)  /* FPR smoke > 16 / 200k: refuse to search */
#define S615_E_OOM (-6)        /* device or HBM-budget allocation failed */
#define S615_E_DEVICE (-7)     /* CUDA error */
#define S615_E_TIMEOUT (-8)    /* a bounded device wait gave up */
#define S615_E_OVERFLOW (-9)   /* hit buffer too small (results incomplete) */
#define S615_E_BUILD (-10)     /* xor peel stalled for every seed */
#define S615_E_NOTABLE (-11)   /* unknown table id */
#define S615_E_BUSY (-12)      /* the context is serving: stop it first */

const char* s615_strerror(int status);

typedef struct s615_ctx s615_ctx;

/* Table layouts held in HBM.  PACKED is the file layout (r-bit cells);
 * WIDE stores one cell per aligned 4- or 8-byte word (one sector per cell). */
#define S615_LAYOUT_AUTO 0
#define S615_LAYOUT_PACKED 1
#define S615_LAYOUT_WIDE 2

/* Store header v2, byte-identical to the reference's StoreHeader
 * (spike/ribbon/store_header.hpp:23-37): 64 bytes, little-endian. */
typedef struct s615_header {
  uint32_t magic, version, kind, r, w, N;
  uint64_t n_keys, m_cells, mix_seed;
  uint32_t shard_count, shard_index, shard_mode, reserved;
} s615_header;

typedef struct s615_table_info {
  s615_header hdr;
  int layout;             /* S615_LAYOUT_PACKED or _WIDE */
  int cell_bytes;         /* 0 for PACKED, else 4 or 8 */
  uint64_t device_bytes;  /* HBM held by the table */
} s615_table_info;

/* Unit record.  cls 5: the 2-D (e,d) peel; cls 2, 3, 4: one free term d
 * (x14, x21, x7) and the find3 leaf over c3 (fourcore_find_v4.cu:165-205).
 * cls 1: the find4 unit of fourcore_find_v4 (expand_unit + make_cand mode 4
 * + k_find4, fourcore_find_v4.cu:165-176,406-420,287-338),
 * B^6 = u^6 + 42^6 (c1^6 + c2^6 + c3^6 + c4^6); a cls 1 plant has
 * base = 42^6 (c1^6 + .. + c4^6) and lim < 2^21.
 * cls 8 (S615_CLS_617_FIND4): one find4 job of the (6,1,7) Branch-A classes
 * 1-4 (gen_class_cands + push_find5_cand + set_window4_gen + k_find4,
 * solve_617_v1.cu:807-884,766-803,507-560), as s615_617_jobs makes them:
 * base[0..1] = Q4 = c1^6 + .. + c4^6 (the target after the c5 peel), B, u, w
 * (the sixth anchor term), lim, fmax2..fmax1 = the c4 window, res_e = c5 and
 * res_d = the (6,1,7) class (1-4).
 * cls 7 (S615_CLS_617): the (6,1,7) Branch-A class-5 candidate of
 * solve_617_v1.cu:885-906, B^6 = u^6 + w^6 + (21d)^6 + 42^6 (c1^6+..+c4^6)
 * with u = 14u', w = 6v', d over residues mod 2^6 (d <= (B-1)/21) and the
 * c4 / c3 windows of k_find4_cls5 (solve_617_v1.cu:563-657).
 * kind 0: a Stage-1 unit (B,u); the engine derives everything like
 * pack_unit5 (fourcore_cls5_gpu_v4.cu:169-184) / free_d_cls234
 * (fourcore_classes_v3.hpp:188-209).  kind 1: a planted target: base
 * (= target - u^6, 3 LE limbs) is taken as given with a single residue per
 * axis and fmax equal to the planted value (the reference's plant shape,
 * solve_516_v3.cu:1130-1170): cls 5 uses res_e/fmax1 and res_d/fmax2;
 * cls 2-4 and 7 use res_d/fmax1.  Classes 2-5: B <= 40,000,000 for kind 0,
 * and for kind 1 base < 2^152 with f * fmax <= 40,000,000 on each axis.  cls 7 kind 0 needs 14 | u, 6 | w,
 * u^6 = B^6 (mod 3^6), w^6 = B^6 (mod 7^6) and B <= 2,353,973 (B^6 < 2^127);
 * units with base <= 0 are dropped like the reference drops them.  A cls 7
 * plant (solve_617_v1.cu:1564-1582) has base < 2^127 and lim < 65536.
 * kind 2 (S615_KIND_JOB): a reduced-T job of fourcore_find_v4 (a .but line or
 * .bbj record, fourcore_job_bin.hpp:30-39, read by job_from_bin
 * fourcore_find_v4.cu:598-608): base[0..1] = T (base[2] = 0), B, u,
 * res_d = free1 (d), res_e = free2 (e, cls 5 only); lim is (B-1)/42.  cls 1:
 * find4 over T (make_cand mode 4); cls 2-4: one find3 row, c3 in
 * [least c with 3c^6 >= T, min(iroot6 T, lim)] (mode 3); cls 5: one gated
 * probe of key T (mode 2, k_find2 :233-252).  A job with an empty window
 * searches nothing, as run_batch drops it (:486); s615_unit_status reports
 * class 1 and out-of-range T (cls 2-4: T = 0 or T >= 2^121) as dropped. */
#define S615_CLS_617 7
#define S615_CLS_617_FIND4 8
#define S615_KIND_JOB 2
typedef struct s615_unit {
  uint32_t cls;      /* 1, 2, 3, 4, 5, 7 or 8 */
  uint32_t kind;     /* 0 = (B,u) or (B,u,w), 1 = planted base, 2 = reduced-T job */
  uint64_t B, u;
  uint64_t base[3];  /* kind 1; kind 2: T in base[0..1] */
  uint32_t fmax1, fmax2, res_e, res_d, lim; /* kind 1; kind 2: res_d, res_e */
  uint32_t w;        /* cls 7: the x6 anchor term 6v'; otherwise 0 */
} s615_unit;

/* Raw filter hit, same layout as the reference's Hit{unit,a,b,d,e,fp}
 * (fourcore_cls5_gpu_v4.cu:140); a=b=0, unit = index into the unit array.
 * cls 5: d is the x21 term and e the x14 term.  cls 2-4: d is the free term
 * and e carries c3 (the reference's find3 Hit puts c3 in its third field,
 * fourcore_find_device.cuh:70-77).  cls 1: d = 0, e carries c3 and c4 carries
 * c4 (k_find4's Hit holds them as c and d).  cls 7: d is the x21 term, e carries c3
 * and c4 carries c4 (the reference's Hit{cand,a,b,c,d,e} of
 * solve_617_v1.cu:364 holds them as e, c and d).  c4 is 0 for other classes
 * and sits in what is padding in the reference's record. */
typedef struct s615_hit {
  uint32_t unit, a, b, d, e, c4;
  uint64_t fp;
} s615_hit;

/* Counters with the reference's meaning (fourcore_cls5_gpu_v4.cu:382-409):
 * calls = in-range (e,d) points, gated = R>0 points stopped by the gate,
 * probes = xor probes issued; pos = R>0 points (= gated + probes).
 * cls 2-4 and 7 count c3 window points as calls and pos.  The (6,1,7)
 * counters of solve_617_v1.cu:985-995 are: its calls = probes, its gated =
 * gated, its probes = 3 * probes, and tri_total / tri_skipped = c4 values
 * that reached / failed the triple-sum gate (0 with S615_F_NO_TRI). */
typedef struct s615_counters {
  uint64_t calls, gated, probes, pos, hits;
  uint64_t tri_total, tri_skipped;
} s615_counters;

/* A verified identity with sorted distinct terms a[0..n-1] < B and their gcd
 * with B (the SOLUTION line of fourcore_cls5_gpu_v4.cu:524-536,
 * fourcore_find_v4.cu:427-457 and solve_617_v1.cu:1096-1106), or a recovered
 * plant (kind 1, a[] unused):
 *   cls 5  : B^6 = u^6 + (21d)^6 + (14e)^6 + 42^6 (c1^6 + c2^6)           n = 5
 *   cls 2-4: B^6 = u^6 + (f d)^6 + 42^6 (c1^6 + c2^6 + c3^6), f = 14, 21, 7 n = 5
 *   cls 7  : B^6 = u^6 + w^6 + (21d)^6 + 42^6 (c1^6 + .. + c4^6)         n = 7
 *   cls 8  : B^6 = u^6 + w^6 + 42^6 (c1^6 + .. + c4^6 + c5^6)            n = 7
 *            (d holds the (6,1,7) class 1-4 and e holds c5)
 * (for plants the left side is base + u^6, or base + u^6 + w^6).  cls 7
 * reports each distinct 7-tuple once per call, like the reference's reported
 * set (solve_617_v1.cu:1096). */
typedef struct s615_solution {
  uint32_t unit, kind, cls, c3;
  uint64_t B, u;
  uint32_t d, e, c1, c2;
  uint32_t c4, w;
  int64_t a[7];
  int64_t gcd;
} s615_solution;

/* ------------------------------------------------------------- context */
/* Open device `device` with an HBM admission budget (0 = all free memory).
 * s615_close frees every table, batch buffer and host staging buffer the
 * context holds (batches from s615_prepare are the caller's to free first). */
int s615_open(int device, size_t hbm_budget, s615_ctx** out);
int s615_close(s615_ctx* ctx);
/* Change the HBM admission budget of an open context (0 = all device memory):
 * allocations that would take the context's total above it fail with
 * S615_E_OOM (a serving loop then waits for running batches to finish). */
int s615_set_budget(s615_ctx* ctx, size_t hbm_budget);
/* Kernel launches the engine issued since open (all of its own kernels). */
uint64_t s615_launch_count(s615_ctx* ctx);

/* Checked build (lib/libs615_checked.so, `make checked`): its kernels compare
 * every table cell, work item, unit, shard and key index with its bound and,
 * when one is out of range, skip the access and set a bit of
 * S615_CHK_CELL / _ITEM / _HIT / _LIST instead.  s615_checked_build returns 1
 * in that build and 0 in the default one; s615_check_flags waits for the
 * device, returns the bits set since the last call in *flags and clears them
 * (always 0 in the default build). */
#define S615_CHK_CELL 1u   /* table cell index >= m, or shard index >= S */
#define S615_CHK_ITEM 2u   /* work item: unit, residue or job run out of range */
#define S615_CHK_HIT 4u    /* a hit's unit index out of range */
#define S615_CHK_LIST 8u   /* xor build: a cell, list entry or key index out of range */
int s615_checked_build(void);
int s615_check_flags(s615_ctx* ctx, uint32_t* flags);

/* -------------------------------------------------------------- tables */
/* xor_load_file (fourcore_xor_store.hpp:147-181) + xor_fpr_smoke (:54-65) +
 * upload: header v2 checks, exact N (expected_N <= 0 accepts any), smoke <=16
 * hits of 200k keys, then the table is resident in HBM. */
int s615_load_table(s615_ctx* ctx, const char* path, int expected_N, int layout,
                    int* table_id);
/* xor_build_pairs (fourcore_xor_store.hpp:67-119) on the device: keys
 * (i^6+j^6) mod 2^64 for 1<=i<=j<=N, the same capacity, seeds and header;
 * parallel peel (cell bytes differ from the host FIFO peel). */
int s615_build_table(s615_ctx* ctx, int N, int r, int layout, int* table_id);
/* build_xor (spike/ribbon/xor_filter.hpp:447-470) over arbitrary host keys. */
int s615_build_table_keys(s615_ctx* ctx, const uint64_t* keys, size_t n, int r,
                          uint64_t base_seed, int layout, int* table_id);
/* xor_save_file (fourcore_xor_store.hpp:126-143): header + packed cells. */
int s615_save_table(s615_ctx* ctx, int table_id, const char* path);
/* Pair-space shard sets (spike/ribbon/shard.hpp:19-24, the shard fields of
 * store_header.hpp:33-35): shard s of S is an xor table over the pair keys k
 * with mix64(k + 0x615615615615615) % S == s (shard_mode 0); a probe of k
 * queries only its own shard, so a set answers exactly like one table over
 * all keys (no false negatives, FPR 2^-r).  Each shard is built on the device
 * with scratch for its own keys only, so sets reach N that one build cannot
 * (the single-table cap is N <= 120,000).  A set's header has shard_count S,
 * the key and cell totals and the routing seed in mix_seed; 2 <= S <= 64.
 * s615_load_table refuses a file that is one shard of a set;
 * s615_load_table_shards takes the files in shard order; s615_save_table
 * and s615_export_table refuse a set, s615_save_table_shard writes one shard's
 * file.  Every run and query entry point takes a set's table id. */
int s615_build_table_sharded(s615_ctx* ctx, int N, int r, int shards, int layout, int* table_id);
/* Shards [lo, hi) of an S-shard set only (one GPU's part when the shards of
 * a set are split over GPUs, no counterpart in the reference): probes of keys
 * whose shard lies outside [lo, hi) find nothing here, so every GPU runs the
 * same units and the union of their hits is the whole set's; each GPU's
 * counters are the whole set's. */
int s615_build_table_shard_range(s615_ctx* ctx, int N, int r, int shards, int lo, int hi,
                                 int layout, int* table_id);
/* paths: consecutive shards k, k+1, .. of one set, in order (all S of them,
 * or a range as above). */
int s615_load_table_shards(s615_ctx* ctx, const char* const* paths, int n, int expected_N,
                           int layout, int* table_id);
int s615_save_table_shard(s615_ctx* ctx, int table_id, int shard, const char* path);
/* Probe passes over a shard set (no counterpart in the reference).  Random
 * reads lose ~3x of their rate once their footprint passes ~64 GiB (the
 * GPU's address-translation reach), so a larger set is probed in G passes:
 * pass g sieves the whole batch again but probes only keys of the g-th group
 * of shards.  Counters and hits are those of one pass over all shards.
 * groups = 0 (the default) picks G = ceil(set bytes / 56 GiB); 1..S forces
 * G.  S615_E_ARG for a single table. */
int s615_set_probe_groups(s615_ctx* ctx, int table_id, int groups);
/* The packed file bytes (after the 64-byte header) into a host buffer of
 * cap >= packed_bytes(m_cells, r) bytes; the in-memory form of the
 * reference's XorFilter::packed. *len receives the byte count. */
int s615_export_table(s615_ctx* ctx, int table_id, s615_header* hdr, uint8_t* buf, size_t cap,
                      size_t* len);
/* xor_fpr_smoke (fourcore_xor_store.hpp:54-65) on a resident table: hits
 * among 200,000 fixed non-member keys (the loaders refuse > 16; the (6,1,7)
 * solver refuses > 8, solve_617_v1.cu:1829-1833). */
int s615_fpr_smoke(s615_ctx* ctx, int table_id, int* hits);
int s615_get_table_info(s615_ctx* ctx, int table_id, s615_table_info* info);
int s615_free_table(s615_ctx* ctx, int table_id);
/* xor_might_contain (xor_filter.hpp:472-483) for n host keys -> out[i] 0/1. */
int s615_xor_query(s615_ctx* ctx, int table_id, const uint64_t* keys, size_t n,
                   uint8_t* out);
int s615_xor_query_dev(s615_ctx* ctx, int table_id, const uint64_t* d_keys, size_t n,
                       uint8_t* d_out, void* stream);

/* Free / total device memory of the context's GPU (cudaMemGetInfo). */
int s615_mem_info(s615_ctx* ctx, size_t* free_bytes, size_t* total_bytes);

/* --------------------------------------------------------------- units */
/* unit_candidates(rt,B,cls,0,1) (fourcore_classes_v3.hpp:137-154). */
int s615_unit_candidates(uint64_t B, int cls, uint64_t* out, size_t cap, size_t* n);
/* gen_class_cands(cls=5) of the (6,1,7) solver (solve_617_v1.cu:885-906) over
 * the full u band: the cls 7 units (B, u = 14u', w = 6v') with
 * u^6 + w^6 < B^6, u' over the 6 classes with (14u')^6 = B^6 (mod 3^6), v' over
 * the 6 classes with (6v')^6 = B^6 (mod 7^6), in the reference's order (u,
 * then w, ascending).  Writes min(cap, count) records; *n = count;
 * S615_E_OVERFLOW when cap is short; S615_E_ARG for B > 2,353,973. */
int s615_617_candidates(uint64_t B, s615_unit* out, size_t cap, size_t* n);
/* gen_class_cands(cls in 1..4) of the (6,1,7) solver with its c5 expansion
 * (solve_617_v1.cu:807-884 over the full u band, push_find5_cand and
 * set_window4_gen :766-803): the cls 8 find4 jobs of one B, in the
 * reference's order.  Same return rules as s615_617_candidates. */
int s615_617_jobs(uint64_t B, int cls, s615_unit* out, size_t cap, size_t* n);
/* expand_unit of fourcore_find_v4 (fourcore_find_v4.cu:164-205): the
 * reduced-T jobs (kind 2) of one Stage-1 unit (kind 0).  cls 1: one job,
 * T = (B^6 - u^6)/42^6; cls 2-4: one job per free term d of free_d_cls234
 * (residue order, then d ascending), T = (B^6 - u^6 - (f d)^6)/42^6; cls 5:
 * one job per (e, d) of free_de_cls5 (e outer), T = (B^6 - u^6 - (21d)^6 -
 * (14e)^6)/42^6.  A d or (e, d) whose difference is not positive, or not
 * divisible by 42^6, is counted in *fail_t (the reference's failT) and
 * skipped.  Writes min(cap, count) jobs; *n = count; S615_E_OVERFLOW when cap
 * is short.  B <= 40,000,000. */
int s615_expand_unit(const s615_unit* unit, s615_unit* out, size_t cap, size_t* n,
                     uint64_t* fail_t);

/* Job files (fourcore_job_bin.hpp; load_jobs_but fourcore_find_v4.cu:125-145).
 * A path ending in .bbj (any case) is the binary form: a 32-byte header
 * {magic 'FCJB', version 2, n_jobs, rec_bytes 36, min_B, max_B, pad} and
 * 36-byte records {u8 cls, 3 pad, u32 B, u, free1, free2, u64 T_lo, T_hi},
 * little-endian.  Any other path is text, one job per line:
 * "cls B u free1 free2 T_lo T_hi" (lines that do not parse are skipped and
 * counted).  The reader streams: s615_jobs_next returns up to cap jobs (kind
 * 2) and *n = 0 at the end. */
typedef struct s615_jobs_file s615_jobs_file;
typedef struct s615_jobs_info {
  uint64_t n_jobs;        /* .bbj: the header's count; text: 0 */
  uint32_t min_B, max_B;  /* .bbj: the header's range; text: 0 */
  uint32_t binary;        /* 1 for .bbj */
  uint32_t pad;
  uint64_t bad_lines;     /* text lines skipped so far */
} s615_jobs_info;
int s615_jobs_open(const char* path, s615_jobs_file** out, s615_jobs_info* info);
int s615_jobs_next(s615_jobs_file* f, s615_unit* out, size_t cap, size_t* n);
int s615_jobs_close(s615_jobs_file* f, s615_jobs_info* info);
/* Writes kind 2 units as a job file (.bbj header with n, min_B, max_B; or
 * text lines).  S615_E_ARG for other kinds or fields wider than the format. */
int s615_jobs_write(const char* path, const s615_unit* jobs, size_t n);

/* Autotuner (no counterpart in the reference).  Times one pass of the peel
 * over this batch of units under every candidate setting -- 16, 32 or 64 rows
 * per class 2-5 work item, times 1 .. the kernel's occupancy limit of blocks
 * per SM -- and keeps the fastest for later batches of the same size (units
 * in [2^k, 2^(k+1))) on this context: s615_prepare, s615_run and the serving
 * loop then use it.  Other sizes keep the default rule (64-row items, fewer
 * for small batches; the occupancy limit).  Results never depend on the
 * setting.  table receives every trial (S615_E_OVERFLOW when cap is short),
 * best the chosen one.  s615_tune_reset forgets every choice. */
typedef struct s615_tune_entry {
  uint32_t item_rows, blocks_per_sm;
  float ms;            /* one pass, CUDA events on the context's stream */
} s615_tune_entry;
int s615_autotune(s615_ctx* ctx, int table_id, const s615_unit* units, size_t n, unsigned flags,
                  s615_tune_entry* table, size_t cap, size_t* n_entries, s615_tune_entry* best);
int s615_tune_reset(s615_ctx* ctx);

/* What a run does with one unit: S615_OK = searched, 1 = dropped like
 * pack_unit5 drops it (u >= B or an empty residue class), S615_E_FORMAT =
 * rejected (outside the engine's exact-arithmetic range, or a planted base
 * whose grid points are not all divisible by 42^6). */
int s615_unit_status(const s615_unit* unit);

/* ---------------------------------------------------------- free peels */
#define S615_F_NO_GATE 1u     /* --no-gate: probe every R>0 point */
#define S615_F_PLAIN 2u       /* one unit per launch + sync (the plain form) */
#define S615_F_NO_TRI 4u      /* cls 7: --no-tri-gate, every c4 of the window */
/* Sharper sound gate (no counterpart in the reference): for every unit kind
 * the peel also requires the point value to be a sum of two sixth powers mod
 * 64, 27, 49, 31, 37 and 43.  Every true pair sum passes, so the verified
 * solutions are the same; the raw hits are a subset of the default run's
 * (the filter's false positives at rejected points are not probed) and
 * calls/gated/probes count the sharper gate.  Ignored with S615_F_NO_GATE. */
#define S615_F_SHARP 8u
/* Launch the peel kernels without their L2-persisting access window (no
 * counterpart in the reference).  By default a table whose cells fit the
 * device's persisting L2 set-aside is marked persisting for the launch, and a
 * larger table's launches mark the gate pattern block instead; results are
 * the same either way.  This flag exists to measure the window. */
#define S615_F_NO_L2_WINDOW 16u

/* The peel of a mixed batch of units (classes 2-5 and 7) in one persistent
 * launch per kernel: run_cls5_gpu's chunk loop (fourcore_cls5_gpu_v4.cu:
 * 472-512) for cls 5, run_batch mode 3 (fourcore_find_v4.cu:460-513) for
 * cls 2-4 and gpu_run (solve_617_v1.cu:924-1006) for cls 7, without the
 * verify step.  Class-7 units go to their own persistent kernel, launched
 * after the first on the same stream.  Host units in, raw hits + counters out (hits unordered).
 * Returns S615_E_OVERFLOW (*n_hits = the true count) when hit_cap is too
 * small; at most 2^24 units per call.  The context keeps the call's device
 * buffers for the next call; they count against the HBM budget and are given
 * back when a table is built or loaded, when another allocation runs out of
 * room, or on s615_close. */
int s615_run(s615_ctx* ctx, int table_id, const s615_unit* units, size_t n, unsigned flags,
             s615_hit* hits, size_t hit_cap, size_t* n_hits, s615_counters* counters);
/* run_cls5_gpu (fourcore_cls5_gpu_v4.cu:412-563) without the verify step:
 * s615_run restricted to class-5 units (S615_E_FORMAT for any other). */
int s615_cls5_run(s615_ctx* ctx, int table_id, const s615_unit* units, size_t n,
                  unsigned flags, s615_hit* hits, size_t hit_cap, size_t* n_hits,
                  s615_counters* counters);
/* Device-resident form: the units are packed and uploaded once
 * (s615_prepare); each s615_run_batch is one launch on the caller's stream
 * (NULL = the context's stream); results stay on the device until
 * s615_batch_results.  s615_batch_free first waits for the batch's last
 * s615_run_batch to finish (it may be called right after the launch, with no
 * sync), then hands the batch's device buffers to a pool on the context (up to
 * 8 GiB), from which later batches take buffers of a fitting size, so
 * prepare/free loops stop allocating device memory; pooled buffers count
 * against the HBM budget and are given back like s615_run's. */
typedef struct s615_batch s615_batch;
int s615_prepare(s615_ctx* ctx, const s615_unit* units, size_t n, s615_batch** out);
int s615_run_batch(s615_ctx* ctx, int table_id, s615_batch* b, unsigned flags, void* stream);
int s615_batch_results(s615_ctx* ctx, s615_batch* b, s615_hit* hits, size_t hit_cap,
                       size_t* n_hits, s615_counters* counters);
int s615_batch_free(s615_ctx* ctx, s615_batch* b);
/* Stage-1 on the device: the class-5 units of every eligible B in
 * [B_lo, B_hi] (gcd(B, 42) = 1; the rule of unit_candidates,
 * fourcore_classes_v3.hpp:114-154, as fourcore_hunt_v3.cpp:371-381 emits it)
 * generated and packed (pack_unit5, fourcore_cls5_gpu_v4.cu:169-184) by device
 * kernels straight into a batch, in the same order as s615_prepare on the
 * host list (B ascending, u ascending).  No unit records cross from the host.
 * B_hi <= 40,000,000 and B_hi - B_lo < 2^26. */
int s615_prepare_band(s615_ctx* ctx, uint64_t B_lo, uint64_t B_hi, s615_batch** out);
/* The (cls, B, u) records of a batch's units, in batch order (to verify or
 * report the hits of a device-generated batch). */
int s615_batch_units(s615_ctx* ctx, const s615_batch* b, s615_unit* out, size_t cap, size_t* n);
/* What s615_prepare copied to the device: unit records, work items and the
 * host-to-device bytes of both (no counterpart in the reference). */
int s615_batch_size(const s615_batch* b, size_t* n_units, size_t* n_items, size_t* h2d_bytes);

/* No counterpart in the reference.  s615_cls5_run for callers that cannot
 * allocate device memory when they search: their free HBM is owned by another
 * allocator, cudaMalloc's latency and implicit device synchronisation are not
 * acceptable on their thread, or their host forbids new device allocations.
 * It allocates no device memory: unit records, work items, counters, the
 * queue cursor and hits live in one fixed device array of the library
 * (about 1.9 MB, held by every GPU that loads the library until exit).
 * Limits: n <= 4096 units, <= 65536 work items (S615_E_ARG beyond either),
 * <= 16384 raw hits (S615_E_OVERFLOW beyond, *n_hits = true count); flags may
 * only hold S615_F_NO_GATE (S615_E_ARG otherwise); S615_E_BUSY while a serving
 * loop owns the context.  Work items are cut like s615_cls5_run's (the tuned
 * rows per item for this batch size, else 64 rows, or 32 / 16 for small
 * batches).  The first call on a device looks up the array's device address;
 * make that first call before any stream capture.  All calls and contexts on
 * a GPU share the array: calls that overlap on the GPU race; each call clears
 * the counters and cursor it needs and waits for its own results. */
int s615_cls5_run_noalloc(s615_ctx* ctx, int table_id, const s615_unit* units, size_t n,
                          unsigned flags, s615_hit* hits, size_t hit_cap, size_t* n_hits,
                          s615_counters* counters);

/* ------------------------------------------------------------- verify */
/* PairRecover + exact identity on the device for hits of any class
 * (fourcore_xor_store.hpp:23-51; fourcore_cls5_gpu_v4.cu:513-542;
 * fourcore_find_v4.cu:516-560): every pair c1 <= c2 with c1^6 + c2^6 equal to
 * the hit's exact remainder (cls 5: T, c2 <= min(N, lim); cls 2-4: T - c3^6,
 * c2 <= min(N, c3); cls 7: T - c4^6 - c3^6, c2 <= N as in expand_xor_hits,
 * solve_617_v1.cu:1019-1036), then the identity, distinct-term, < B and gcd
 * checks.  Solutions come sorted by (unit, e, d, c4, c1). */
int s615_verify(s615_ctx* ctx, const s615_unit* units, size_t n_units, const s615_hit* hits,
                size_t n_hits, int N, s615_solution* out, size_t cap, size_t* n_out);
/* s615_verify restricted to class-5 units (S615_E_FORMAT for any other). */
int s615_cls5_verify(s615_ctx* ctx, const s615_unit* units, size_t n_units,
                     const s615_hit* hits, size_t n_hits, int N, s615_solution* out,
                     size_t cap, size_t* n_out);

/* ------------------------------------------------------------ selftest */
/* Host-only checks of selftest_host (fourcore_cls5_gpu_v4.cu:186-263) plus the
 * engine's invariants (gate factorisation, exact remainder, row identity).
 * Needs no GPU.  Returns 0 on success, else the number of the failed check. */
int s615_selftest_host(void);

/* ------------------------------------------------------------- journal */
/* Restart journal of a campaign (no counterpart in the reference, whose
 * restarts redo the whole band, fourcore_runbook_v3.md:162-170): an
 * append-only text file of committed blocks, one per finished request or
 * chunk, holding the block's units, their raw hits and their verified
 * solutions (hit and solution unit indices refer to the block's units).  A
 * block counts only once its closing checksum line is complete, so a block
 * torn by a crash is ignored and its units are searched again; opening the
 * journal cuts such a tail off before anything is appended.
 * s615_journal_append flushes and fsyncs before it returns.  A journal
 * handle is not thread-safe. */
typedef struct s615_journal s615_journal;
int s615_journal_open(const char* path, s615_journal** out);   /* creates the file if missing */
/* 1 if the unit (every field equal) is in a committed block, else 0. */
int s615_journal_has(const s615_journal* j, const s615_unit* unit);
int s615_journal_stats(const s615_journal* j, size_t* units, size_t* hits, size_t* solutions);
/* Committed units in file order, and the recorded solutions with `unit`
 * indexing that list (to report them again after a restart). */
int s615_journal_units(const s615_journal* j, s615_unit* out, size_t cap, size_t* n);
int s615_journal_solutions(const s615_journal* j, s615_solution* out, size_t cap, size_t* n);
int s615_journal_append(s615_journal* j, const s615_unit* units, size_t n, const s615_hit* hits,
                        size_t n_hits, const s615_solution* sols, size_t n_sols);
int s615_journal_close(s615_journal* j);

/* ------------------------------------------------------------- serving */
/* A long-running request loop on one context (no counterpart in the
 * reference, which runs one campaign per process).  s615_submit queues a copy
 * of the caller's units and returns a ticket; a worker thread takes every
 * pending request for the same (table, flags) -- up to max_batch_units units
 * -- as one batch, launches it on one of `slots` streams as soon as a stream
 * is free and its buffers fit the HBM budget (requests that arrive meanwhile
 * join the next batch: continuous batching), verifies its hits and splits the
 * results back per request.  A request's hits and solutions are the same as
 * those of s615_run + s615_verify on its units alone.  While serving, calls
 * that allocate or launch on the context (s615_run, s615_prepare,
 * s615_verify, table loads/builds/frees) return S615_E_BUSY. */
typedef struct s615_result {
  uint64_t ticket;
  int32_t status;                  /* S615_OK or the batch's error status */
  int32_t table_id;
  uint64_t n_units;
  uint64_t n_hits, n_solutions;
  const s615_hit* hits;            /* unit = index into this request's units */
  const s615_solution* solutions;  /* both owned by the library until s615_release */
  s615_counters counters;          /* of the whole batch that carried the request */
  uint32_t batch_requests;         /* requests in that batch */
  uint32_t pad;
  double queued_ms;                /* submit -> launch */
  double latency_ms;               /* submit -> result ready (verified) */
} s615_result;
/* slots: batches in flight (1..16); max_batch_units: 0 = 2^20. */
int s615_serve_start(s615_ctx* ctx, int slots, size_t max_batch_units);
int s615_submit(s615_ctx* ctx, int table_id, const s615_unit* units, size_t n, unsigned flags,
                uint64_t* ticket);
/* Finished requests, oldest first; waits up to wait_ms for the first one. */
int s615_poll(s615_ctx* ctx, s615_result* out, size_t cap, size_t* n, int wait_ms);
int s615_release(s615_ctx* ctx, uint64_t ticket);
/* Stops accepting requests, finishes every submitted one, joins the worker;
 * finished results stay readable until released or s615_close. */
int s615_serve_stop(s615_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif
