/*
 * s615_oracle.h -- C API of the CPU oracle for the cls5 peel/gate/probe path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain CPU restatement of the
 * reference algorithm (cavedave/six-one-five) and is used exclusively as the
 * checker: by tests/, by __graft_entry__.smoke() and by bench.py's
 * cpu_baseline / reference leg.  The product (libs615) never links or calls it.
 *
 * Every function follows the reference file:line named beside it.  Naming
 * follows the reference: e is the x14 free term (residues mod 3^6), d is the
 * x21 free term (residues mod 2^6).
 */
#ifndef S615_ORACLE_H
#define S615_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Store header v2 (spike/ribbon/store_header.hpp:23-37), 64 bytes LE. */
typedef struct orc_header {
  uint32_t magic, version, kind, r, w, N;
  uint64_t n_keys, m_cells, mix_seed;
  uint32_t shard_count, shard_index, shard_mode, reserved;
} orc_header;

/* Unit5 (fourcore_cls5_gpu_v4.cu:143-151): base = B^6-u^6 as 3 LE limbs. */
typedef struct orc_unit5 {
  uint64_t B, u;
  uint64_t base[3];
  uint32_t lim, mod1, mod2, fmax1, fmax2, nres1, nres2;
  uint32_t res[24]; /* e residues then d residues */
  uint32_t planted; /* 1 = base set directly (plant), verify against base */
} orc_unit5;

/* Hit (fourcore_cls5_gpu_v4.cu:140). */
typedef struct orc_hit {
  uint32_t unit, a, b, d, e;
  uint64_t fp;
} orc_hit;

typedef struct orc_table orc_table;

/* ---- units (fourcore_classes_v3.hpp) ---- */
/* unit_candidates(rt,B,cls,0,1) -> sorted u list; returns count (<= cap written). */
size_t orc_unit_candidates(uint64_t B, int cls, uint64_t* out, size_t cap);
/* seeds_for_B count for a class (selftest KAT). */
size_t orc_seed_count(uint64_t B, int cls);
/* pack_unit5 (fourcore_cls5_gpu_v4.cu:169-184). 1 = ok. */
int orc_pack_unit5(uint64_t B, uint64_t u, orc_unit5* out);
/* free_d_cls234 (fourcore_classes_v3.hpp:188-209): residues, mod, fmax. */
int orc_free_d_cls234(uint64_t B, uint64_t u, int cls, uint32_t* res, uint32_t* nres,
                      uint64_t* mod, uint64_t* fmax);

/* ---- exact arithmetic KATs ---- */
void orc_pow6_192(uint32_t x, uint64_t out[3]);
/* T=(B^6-u^6-(21d)^6-(14e)^6)/42^6 (fourcore_gmp.hpp:55-62); 1 if ok. */
int orc_T_peel2(uint64_t B, uint64_t u, uint64_t d, uint64_t e, uint64_t T[2]);
/* funnel fingerprint of base-(14e)^6-(21d)^6 (cls5_gpu_v4.cu:266-268). */
uint64_t orc_funnel_fp(const orc_unit5* U, uint32_t d, uint32_t e, int* ok);
/* gate bitmaps (cls5_gpu_v4.cu:124-137): 504 + 247 flags. */
void orc_gate_tables(uint8_t g504[504], uint8_t g247[247]);

/* ---- xor filter (spike/ribbon/xor_filter.hpp, xor_pack.hpp, mix64.hpp) ---- */
uint64_t orc_mix64(uint64_t x);
size_t orc_capacity_for(size_t n);
size_t orc_packed_bytes(uint64_t m_cells, uint32_t r);
/* build_xor(keys, r, base_seed, max_tries) -> table (NULL on failure). */
orc_table* orc_build_xor(const uint64_t* keys, size_t n, int r, uint64_t base_seed,
                         int max_seed_tries);
/* xor_build_pairs(N, r) (fourcore_xor_store.hpp:67-119). */
orc_table* orc_build_pairs(int N, int r);
/* xor_load_file (fourcore_xor_store.hpp:147-181); expected_N<=0 accepts any. */
/* Pair-space shards (spike/ribbon/shard.hpp, store_header.hpp shard fields):
 * shard s of S holds the pair keys with mix64(key + seed) % S == s. */
orc_table* orc_build_pairs_shard(int N, int r, int S, int s, uint64_t seed);
orc_table* orc_shard_set(const orc_table* const* parts, int S, uint64_t seed);
uint32_t orc_shard_of(uint64_t key, uint64_t seed, uint32_t S);
orc_table* orc_load(const char* path, int expected_N);
orc_table* orc_from_memory(const orc_header* h, const uint8_t* bytes, size_t len);
int orc_save(const orc_table* t, const char* path);
void orc_free(orc_table* t);
void orc_table_header(const orc_table* t, orc_header* h);
const uint8_t* orc_table_bytes(const orc_table* t, size_t* n);
/* xor_might_contain (xor_filter.hpp:472-483) over n keys. */
void orc_query(const orc_table* t, const uint64_t* keys, size_t n, uint8_t* out);
/* xor_fpr_smoke (fourcore_xor_store.hpp:54-65). */
int orc_fpr_smoke(const orc_table* t);
void orc_residue(const orc_table* t, const uint64_t* keys, size_t n, uint64_t* out);
void orc_mt64(uint64_t seed, size_t n, uint64_t* out);

/* ---- cls5 peel (k_cls5_192, fourcore_cls5_gpu_v4.cu:353-410) ---- */
/* Runs every unit; hits (unit index, d, e, fp) appended up to cap; counters
 * calls/gated/probes; threads<=0 uses all OpenMP threads. Returns #hits found
 * (may exceed cap; only cap written). */
size_t orc_cls5_run(const orc_table* t, const orc_unit5* units, size_t n, int use_gate,
                    int threads, orc_hit* hits, size_t cap, uint64_t counters[3]);

/* ---- verify (cls5_gpu_v4.cu:513-542, fourcore_xor_store.hpp:23-51) ---- */
/* For each hit, PairRecover + exact verify.  Writes SOLUTION lines (or PLANT
 * lines for planted units) into buf; returns number of lines. */
size_t orc_cls5_verify(const orc_unit5* units, const orc_hit* hits, size_t nh, int N,
                       int stop_first, char* buf, size_t buflen);

/* ---- cls2-4 find3 leaf (fourcore_find_v4.cu:165-205,255-284,401-425) ---- */
typedef struct orc_job3 {
  uint32_t cls, lim;
  uint64_t B, u, d;     /* free term d (x14 / x21 / x7) */
  uint64_t T[2];        /* T=(B^6-u^6-(f d)^6)/42^6 */
  uint32_t lo, hi;      /* c3 window */
} orc_job3;
typedef struct orc_hit3 {
  uint32_t job, c3;
  uint64_t fp;
} orc_hit3;
/* Expand one unit into find3 jobs (expand_unit + make_cand mode 3). */
size_t orc_expand_cls234(uint64_t B, uint64_t u, int cls, orc_job3* out, size_t cap);
size_t orc_find3_run(const orc_table* t, const orc_job3* jobs, size_t n, int use_gate,
                     int threads, orc_hit3* hits, size_t cap, uint64_t counters[3]);

/* ---- cls1 find4 (fourcore_find_v4.cu:165-176,406-420,287-338) ---- */
typedef struct orc_hit4 {
  uint32_t job, c3, c4, pad;
  uint64_t fp;
} orc_hit4;
/* expand_unit(cls 1) + make_cand(mode 4): one job with T = (B^6-u^6)/42^6 and
 * the c4 window [lo, hi] (hi = min(iroot6(T), lim), lo least with 4 lo^6 >= T);
 * returns 0 when compute_T fails or the window is empty (run_batch drops it). */
size_t orc_expand_cls1(uint64_t B, uint64_t u, orc_job3* out, size_t cap);
/* k_find4: per c4 the c3 window [max(1, (u32)(0.8 hi3)), hi3], hi3 = min(iroot6(T - c4^6),
 * lim, c4); counters calls / gated / probes.  ref_tiles != 0 repeats each c4 as the
 * reference's y tiles of 2048 do (block y walks c4 >= lo + 2048 y to hi). */
size_t orc_find4_run(const orc_table* t, const orc_job3* jobs, size_t n, int use_gate,
                     int ref_tiles, int threads, orc_hit4* hits, size_t cap, uint64_t counters[3]);

/* ---- reduced-T jobs of fourcore_find_v4 (.but / .bbj; find2 / find3 / find4) ---- */
typedef struct orc_job {
  uint32_t cls, lim;    /* lim = (B-1)/42 (job_from_bin, fourcore_find_v4.cu:598-608) */
  uint64_t B, u, free1, free2;
  uint64_t T[2];
} orc_job;
/* expand_unit (fourcore_find_v4.cu:164-205) for cls 1-5: the jobs of one
 * Stage-1 unit in the reference's order; *fail_t counts the d or (e, d) whose
 * T cannot be formed (compute_T_*_gmp false). */
size_t orc_expand_unit(uint64_t B, uint64_t u, int cls, orc_job* out, size_t cap,
                       uint64_t* fail_t);
/* run_batch over jobs: make_cand (:401-425) then k_find2 (:233-252), k_find3
 * (:255-284) or k_find4 (:287-338) by class; empty find3/find4 windows are
 * dropped (:486).  Hits {job, c3, c4, fp} (c3 = c4 = 0 for find2, c4 = 0 for
 * find3); counters calls / gated / probes summed over the three modes. */
size_t orc_jobs_run(const orc_table* t, const orc_job* jobs, size_t n, int use_gate, int ref_tiles,
                    int threads, orc_hit4* hits, size_t cap, uint64_t counters[3]);
/* The exact filter of run_batch (:536-560) over PairRecover's pairs: returns
 * the exact matches (the reference's `sols`); the ones report_solution
 * (:427-457) prints go to buf as SOLUTION lines, *n_lines of them. */
size_t orc_jobs_verify(const orc_job* jobs, const orc_hit4* hits, size_t nh, int N, char* buf,
                       size_t buflen, size_t* n_lines);

/* ---- (6,1,7) Branch-A class 5 (solve_617_v1.cu) ---- */
typedef struct orc_cand617 {
  uint64_t base[2];        /* B^6 - u^6 - w^6 (i128; B <= 2,353,973) */
  uint32_t B, u, w, lim;   /* u = 14u', w = 6v' */
  uint32_t mod1, fmax1, nres1, pad;
  uint32_t res[24];        /* d residues mod 64 (the 21d term) */
} orc_cand617;
typedef struct orc_hit617 {
  uint32_t cand, a, b, c, d, e;   /* c = c3, d = c4, e = the x21 term */
  uint64_t fp;
} orc_hit617;
/* gen_class_cands(cls=5) (solve_617_v1.cu:885-906), full u band. */
size_t orc_617_cands(uint64_t B, orc_cand617* out, size_t cap);
/* k_find4_cls5 (solve_617_v1.cu:563-657): counters[0..4] = calls (post-gate
 * probes), gated, probes (3 slot reads per probe), tri_total, tri_skipped
 * (c4 values that reached / failed the triple-sum gate; the reference's own
 * tri counters are 32 times these, since each of the 32 threads of the warp
 * that walks a c4 counts it, :604-614).
 * zmax <= 1 visits every (d, c4, c3) once.  zmax > 1 restates the reference
 * launch with grid.z = zmax (gpu_run, solve_617_v1.cu:960-968): block z walks
 * c4 from lo4 + 2048 z to hi4, so c4 is visited min(zmax, (c4-lo4)/2048 + 1)
 * times and every count and hit is repeated that often. */
size_t orc_617_run(const orc_table* t, const orc_cand617* cands, size_t n, int use_gate,
                   int use_tri, int zmax, int threads, orc_hit617* hits, size_t cap,
                   uint64_t counters[5]);
/* expand_xor_hits + verify_hit (solve_617_v1.cu:1019-1110): SOLUTION lines
 * (distinct tuples only); plants (u=14, w=6 dummies) print PLANT617 lines.
 * stats (may be NULL) gets the campaign's exact / fp-false counts
 * (:1949-1950): expanded (hit, pair) records with / without the identity. */
size_t orc_617_verify(const orc_cand617* cands, const orc_hit617* hits, size_t nh, int N,
                      int planted, char* buf, size_t buflen, uint64_t stats[2]);

/* ---- (6,1,7) Branch-A classes 1-4: find5 by c5 expansion, then find4
 * (solve_617_v1.cu:807-884 gen_class_cands, :766-803 push_find5_cand /
 * set_window4_gen, :507-560 k_find4, :1040-1110 verify_hit) ---- */
typedef struct orc_job617 {
  uint64_t Q4[2];          /* Q - c5^6 = c1^6 + .. + c4^6 */
  uint32_t B, u, w, cls;   /* w: the sixth anchor term (42w', 14v', 21v' or 6v') */
  uint32_t c5, lim, lo, hi;/* c4 window [lo, hi] */
} orc_job617;
typedef struct orc_hit4x {
  uint32_t job, c3, c4, pad;
  uint64_t fp;
} orc_hit4x;
size_t orc_617_jobs(uint64_t B, int cls, orc_job617* out, size_t cap);
/* counters as orc_617_run; ymax > 1 repeats c4 as the reference's y tiles do
 * (block y walks c4 >= lo + 2048 y, ymax = the batch's tile count). */
size_t orc_617_find4_run(const orc_table* t, const orc_job617* jobs, size_t n, int use_gate,
                         int use_tri, int ymax, int threads, orc_hit4x* hits, size_t cap,
                         uint64_t counters[5]);
size_t orc_617_find4_verify(const orc_job617* jobs, const orc_hit4x* hits, size_t nh, int N,
                            char* buf, size_t buflen, uint64_t stats[2]);

#ifdef __cplusplus
}
#endif
#endif
