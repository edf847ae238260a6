// engine.hpp -- internal types of the B200 engine (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/s615.h"
#include "s615_common.hpp"

namespace s615 {

// An NVTX range over a host scope, so a profiler's timeline shows the
// engine's phases (prepare, run, results, verify, table build and load,
// serving batches); a no-op unless a profiler is attached.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// ------------------------------------------------------------ device unit
// One unit as the peel kernel consumes it.  Only base mod 2^128 is needed:
// every row quantity is an exact integer below 2^122 recovered from the low
// 128 bits with the 2-adic inverse of 21^6 (the host checks the
// divisibility this relies on).
//   cls 5  : rows are e = res1[i] + 729 j (e <= fmax1), columns
//            d = res2[k] + 64 t (d <= fmax2); row value V = (base-(14e)^6)/21^6.
//   cls 2-4: rows are d = res1[i] + mod1 j (d <= fmax1), free factor f; row
//            value T = (base-(f d)^6)/42^6, columns c3 over the find3 window.
//   cls 1  : the find4 unit (fourcore_find_v4.cu:287-338): base holds
//            T = (B^6-u^6)/42^6 itself, fmax2..fmax1 the c4 window [lo4, hi4];
//            items are chunks of kC4Chunk c4 values.
//   cls 8  : a (6,1,7) class 1-4 find4 job: base = Q4, fmax2..fmax1 the c4
//            window, pad1 = c5, pad2 = the (6,1,7) class; c4 chunks as cls 1.
//   cls 7  : the (6,1,7) class-5 shape: base = B^6-u^6-w^6 (< 2^127), rows
//            d = res1[i] + 64 j (d <= fmax1), f = 21; each row's c4 window
//            opens find3 rows T' = T - c4^6 over c3.
struct DevUnit {
  u64 base_lo, base_hi;
  u64 B, u;
  u32 cls, fmax1, fmax2, lim;
  u32 nres1, nres2, mod1, f;
  u32 id, w, pad1, pad2;
  u32 res1[24];
  u32 res2[12];
};
static_assert(sizeof(DevUnit) == 224, "DevUnit layout");

// Gate pattern tables.  For q in {9,7,13,19} and a,s in [0,q), bit i of word
// pat[base_q + a*q + s] says whether (W - x^6)/scale is an admissible pair sum
// mod q when W = a (mod q) and x = s + step*i (mod q).  Two sets: the cls5
// columns (step 64, scale 64) and the find3 columns (step 1, scale 1).
constexpr int kPatQ[4] = {9, 7, 13, 19};
constexpr int kPatBase[4] = {0, 81, 130, 299};
constexpr int kPatB9 = 0, kPatB7 = 81, kPatB13 = 130, kPatB19 = 299;  // usable in device code
constexpr int kPatWords = 660;

// Sharper sound gate (S615_F_SHARP, no counterpart in the reference): T must
// also be a sum of two sixth powers mod 64 (a 32-column mask per row), 27 and
// 49 (in place of 9 and 7), 13, 19, 31, 37 and 43 (pattern words as above).
// Pattern blocks per q in this order; 7,839 words per column shape.
constexpr int kSharpQ[7] = {27, 49, 13, 19, 31, 37, 43};
constexpr int kSharpBase[7] = {0, 729, 3130, 3299, 3660, 4621, 5990};
constexpr int kSB27 = 0, kSB49 = 729, kSB13 = 3130, kSB19 = 3299, kSB31 = 3660, kSB37 = 4621,
              kSB43 = 5990;
constexpr int kSharpWords = 7839;

// Triple-sum gate of solve_617_v1.cu:334-345 for the c4 step, as one
// 400-word block: bitmaps of {a^6+b^6+c^6 mod 504} (16 words) and mod 247
// (8 words), then c^6 mod 504 (504 u16) and c^6 mod 247 (247 u16).
constexpr int kTriT504 = 0, kTriT247 = 16, kTriP504 = 24, kTriWords = 400;

// Table resident in HBM.
// Pair-space shards (spike/ribbon/shard.hpp:19-24): shard s of S holds the
// pair keys k with mix64(k + kShardSeed) % S == s, and a probe of k queries
// only that shard.  The reference's helper takes the seed as a parameter;
// this store fixes it (every shard file of one set shares it).
constexpr u64 kShardSeed = 0x615615615615615ULL;

struct DevTable {
  s615_header hdr{};
  int layout = S615_LAYOUT_WIDE;
  int cell_bytes = 8;        // 4 or 8 for WIDE, 0 for PACKED
  void* d_cells = nullptr;
  size_t bytes = 0;
  u64 block = 0, recip = 0;
  std::vector<DevTable> parts;   // a shard set (hdr.shard_count > 1): its shards in order
  u32 shard_lo = 0;              // parts[i] is shard shard_lo + i of hdr.shard_count
  void* d_views = nullptr;       // one TableView per shard of the set in HBM (owned ones set)
  u32 groups = 0;                // probe passes over a set (0: from its size)
};

// Random reads keep their rate over footprints up to 64 GiB and lose ~3x at
// 110 GiB on a B200 (bin/randaccess_peak 2 8 29 64 110).  A shard set larger
// than this is probed in passes over groups of its shards, each pass
// touching at most this many bytes.
constexpr u64 kProbeGroupBytes = 56ull << 30;
// Internal launch flag: a pass after the first adds no counters (it repeats
// the first pass's points; only its probes differ).
constexpr unsigned kFlagNoCount = 1u << 30;

// Kernel-facing view of a table (or of a shard set: shards > 1, parts).
struct TableView {
  const void* cells;
  u64 block, recip, fpmask, seed;
  u32 r, layout, cell_bytes, shards;
  const TableView* parts;
  u64 shard_seed;
  u32 grp_lo, grp_hi;   // this pass probes keys of shards [grp_lo, grp_hi)
  u32 groups, pad;      // passes over the set
  u64 bytes;            // bytes of cells (a single table; 0 for a set)
};

struct Cls5Counters {  // device accumulators (u64 atomics)
  unsigned long long calls, probes, pos, hits;
  unsigned long long tri_total, tri_skipped;
};

// Work items: (unit, residue index, chunk of kItemRows rows) packed in a u64.
constexpr u32 kItemRows = 64;
// (6,1,7) rows carry a whole c4 window each: 8 rows per item, and each such
// chunk goes out as kParts617 items (chunk field = chunk * kParts617 + part) of
// which part p takes every kParts617-th 32-wide block of the rows' c4 windows,
// so that the heaviest rows are shared by several warps.
constexpr u32 kItemRows617 = 8;
constexpr u32 kParts617 = 8;
S615_HD u32 item_rows(u32 cls) { return cls == 7u ? kItemRows617 : kItemRows; }
constexpr u32 kC4Chunk = 128;   // cls 1: c4 values per work item
constexpr u32 kMaxBatchUnits = 1u << 24;
S615_HD u64 make_item(u32 unit, u32 ires, u32 chunk) {
  return ((u64)unit << 32) | ((u64)ires << 24) | chunk;
}
S615_HD u32 item_unit(u64 it) { return (u32)(it >> 32); }
S615_HD u32 item_res(u64 it) { return (u32)(it >> 24) & 255u; }
S615_HD u32 item_chunk(u64 it) { return (u32)it & 0xFFFFFFu; }
// Reduced-T jobs (kind 2) of classes 2-5 become one-row units of this
// internal class; consecutive ones share an item (first unit, kJobItemTag,
// count | kJobFind2 for the one-probe rows of class-5 jobs).
constexpr u32 kClsJobRow = 9;
constexpr u32 kJobRows = 64;
constexpr u32 kJobItemTag = 255;
constexpr u32 kJobFind2 = 1u << 8;
S615_HD u32 job_count(u64 it) { return (u32)it & 0xFFu; }
// Rows of one residue class: x = r0 + mod j for j in [jmin, jend), x <= fmax.
S615_HD void class_rows(u32 r0, u32 mod, u32 fmax, u32* jmin, u32* jend) {
  *jmin = (r0 == 0) ? 1u : 0u;
  *jend = (r0 <= fmax) ? (fmax - r0) / mod + 1u : 0u;
}

}  // namespace s615

namespace s615 {
struct Server;   // serve.cpp
}

struct s615_batch {
  size_t n_units = 0, n_items = 0;
  size_t n_main = 0;             // items [0, n_main) are classes 2-5, the rest cls 7
  s615::DevUnit* d_units = nullptr;
  s615::u64* d_items = nullptr;
  s615_hit* d_hits = nullptr;
  s615::u32 hit_cap = 0;
  size_t cap_units = 0, cap_items = 0;   // device capacity (a reused batch only grows)
  size_t units_bytes = 0, items_bytes = 0, ctr_bytes = 0, hits_bytes = 0;   // buffer sizes
  s615::Cls5Counters* d_ctr = nullptr;
  s615::u32* d_work = nullptr;   // persistent-queue cursors [classes 2-5, cls 7]
  s615::u32 item_rows = s615::kItemRows;   // rows per class 2-5 item (smaller for small batches)
  // items per class 2-4 row chunk, 1, 2 or 4 (chunk field = chunk * parts3 +
  // part): part p sieves every parts3-th 1024-column tile of the rows' c3 windows
  s615::u32 parts3 = 1;
  s615::u32 blocks_per_sm = 0;              // k_peel blocks per SM (0: the occupancy limit)
  cudaEvent_t done = nullptr;   // recorded after the last s615_run_batch's launches
  // host copy of the work items: grow-only and uninitialised, written in
  // place by the fill's threads
  std::unique_ptr<s615::u64[]> host_items;
  size_t host_items_cap = 0;
};

namespace s615 {
// A grow-only host buffer: pinned when the driver grants it, pageable if not.
struct HostStage {
  void* p = nullptr;
  size_t bytes = 0;
  bool pinned = false;
};
}  // namespace s615

struct s615_ctx {
  int device = 0;
  size_t budget = 0;
  // device bytes held against the budget; updated by the caller's threads and
  // the serving worker (dev_alloc reserves before it allocates)
  std::atomic<size_t> used{0};
  cudaStream_t stream = nullptr;
  std::map<int, s615::DevTable> tables;
  int next_table = 1;
  s615::u32* d_pat = nullptr;   // [gate cls5 | open cls5 | gate find3 | open find3]
  s615::u32* d_tri = nullptr;   // triple-sum gate block (kTriWords)
  s615::u32* d_sharp = nullptr; // sharp patterns [cls5 shape | find3 shape]
  unsigned long long p64 = 0;   // bit t: t is a sum of two sixth powers mod 64
  int num_sms = 0;
  unsigned long long launches = 0;
  std::mutex mu;
  s615::Server* server = nullptr;   // the serving loop, when started
  void* arena[4] = {};              // verify scratch, grow-only (units, hits, pairs, count)
  s615::u32* d_roots = nullptr;     // device Stage-1 root tables (stage1.cu)
  size_t roots_bytes = 0;
  size_t arena_cap[4] = {};
  // s615_autotune's choice per batch size (bucket k: 2^k <= units < 2^(k+1));
  // zero fields fall back to the occupancy rule.  force_* hold a trial's
  // setting while s615_autotune times it.
  struct Tune { s615::u32 item_rows = 0, blocks_per_sm = 0; } tune[40];
  s615::u32 force_rows = 0, force_bps = 0;
  // The unit records every fill_batch packs before its host-to-device copy
  // (reused, so a large batch is neither page-faulted nor copied from pageable
  // memory again), and s615_run's own batch, whose device buffers serve the
  // next call.  Both live until s615_close; the batch is also given back when a
  // device allocation runs out of room.
  s615::HostStage unit_stage;
  s615_batch* run_batch = nullptr;
  // device buffers of freed batches, reused by the next batch (capi.cu)
  std::vector<std::pair<void*, size_t>> pool;
  size_t pool_bytes = 0;
  std::mutex pool_mu;
  bool run_busy = false;
  // L2-persisting access windows (cudaDevAttrMaxPersistingL2CacheSize,
  // cudaDevAttrMaxAccessPolicyWindowSize) and the set-aside this context
  // has asked for (cudaLimitPersistingL2CacheSize, per process).
  size_t l2_persist_max = 0, l2_window_max = 0, l2_limit = 0;
};

namespace s615 {

// Status helpers.
int cuda_status(cudaError_t e);
#define S615_CU(x)                                   \
  do {                                               \
    cudaError_t _e = (x);                            \
    if (_e != cudaSuccess) return ::s615::cuda_status(_e); \
  } while (0)

// Serving: true when a request loop owns the context and the caller is not
// its worker thread (calls that allocate or launch then return S615_E_BUSY).
bool serving_blocks(s615_ctx* ctx);
void server_destroy(s615_ctx* ctx);   // stops the loop (draining it) and frees it

// Host staging (grow-only; nullptr if even a pageable buffer cannot be had).
void* stage_get(HostStage& s, size_t bytes);
void stage_free(HostStage& s);
// Frees s615_run's kept batch (unless a run is using it) and the pool of
// freed batch buffers; true if either held anything.
bool release_run_batch(s615_ctx* ctx);

// Budgeted device allocation.
int dev_alloc(s615_ctx* ctx, void** p, size_t bytes);
void dev_free(s615_ctx* ctx, void* p, size_t bytes);
// Batch buffers through the context's pool: pool_get hands out a pooled
// buffer of at least `bytes` (at most twice that) or a new one, with its size
// in *got; pool_put keeps a buffer for reuse (or frees it once the pool is
// full); pool_release frees every pooled buffer.
int pool_get(s615_ctx* ctx, size_t bytes, void** p, size_t* got);
void pool_put(s615_ctx* ctx, void* p, size_t bytes);
void pool_release(s615_ctx* ctx);
// The check words of the checked build (read and cleared; 0 in the default
// build), one per compiled file whose kernels check their indices.
unsigned check_take_peel();
unsigned check_take_peel617();
unsigned check_take_table();
unsigned check_take_xor_build();
// Grow-only scratch slot k of the context (no free, so no device-wide sync
// once it is large enough).
int arena_get(s615_ctx* ctx, int k, size_t bytes, void** p);
// Pack units into batch b (new or reused: its device buffers only grow) and
// copy them to the device.
int fill_batch(s615_ctx* ctx, const s615_unit* units, size_t n, s615_batch* b);

TableView view_of(const DevTable& t);

// The launch attribute for a peel kernel's L2-persisting access window: the
// table's cells when they fit the persisting set-aside (the window's lines
// stay in L2 while other traffic streams past), else the gate pattern block
// the kernels read.  Returns the number of attributes written (0 or 1); 0
// with S615_F_NO_L2_WINDOW or when the device offers no persisting L2.
int l2_window(s615_ctx* ctx, const TableView& tv, unsigned flags, cudaLaunchAttribute* attr);

// Kernel launchers (each returns a status and counts its launches).
// Launches k_peel over items [0, n_main) and, when present, the (6,1,7)
// kernel over [n_main, n_items), in that order on st.
int launch_peel(s615_ctx* ctx, const TableView& tv, s615_batch* b, unsigned flags,
                cudaStream_t st, int grid_blocks);
int launch_peel617(s615_ctx* ctx, const TableView& tv, s615_batch* b, unsigned flags,
                   cudaStream_t st, int grid_blocks);
int launch_xor_query(s615_ctx* ctx, const TableView& tv, const u64* d_keys, size_t n,
                     u8* d_out, cudaStream_t st);
int launch_unpack(s615_ctx* ctx, const u8* d_packed, u64 m, u32 r, void* d_wide, int cell_bytes,
                  cudaStream_t st);
int launch_pack(s615_ctx* ctx, const void* d_wide, int cell_bytes, u64 m, u32 r, u8* d_packed,
                u64 packed_len, cudaStream_t st);

// Device xor build over a unique-value source; see xor_build.cu.
int build_xor_device(s615_ctx* ctx, const u64* d_pair_vals, u64 n_vals, const u64* d_keys,
                     u64 n_keys, int r, const u64* seeds, int n_seeds, int N, int layout,
                     DevTable* out, u32 shards = 1, u32 shard = 0);

// Device verifier; see verify.cu.
int verify_device(s615_ctx* ctx, const s615_unit* units, size_t n_units, const s615_hit* hits,
                  size_t n_hits, int N, s615_solution* out, size_t cap, size_t* n_out);

// Host math shared by the C ABI and the CLI.
struct W3 { u64 l[3]; };
W3 pow6_w3(u64 x);
bool sub_w3(W3& a, const W3& b);   // a -= b, true on borrow
void add_w3(W3& a, const W3& b);
W3 mul_w3_u64(const W3& a, u64 m);
bool zero_w3(const W3& a);
bool eq_w3(const W3& a, const W3& b);
u64 divmod_w3(W3& a, u64 m);
u128 pow6_u128(u64 x);
u128 inv_2adic_u128(u128 a);  // a odd

// Residue classes (free-term rules of fourcore_classes_v3.hpp:156-219).
std::vector<u32> e_residues(u64 B);
std::vector<u32> d_residues(u64 B, u64 u);
std::vector<u32> d_residues_cls234(u64 B, u64 u, int cls, u32* mod, u32* fmax);
std::vector<u64> unit_candidates(u64 B, int cls);
void root_csr(int which, std::vector<u32>& off, std::vector<u32>& roots);
u32 inv_pow6_mod(u32 f, u32 m);   // (f^6)^-1 mod m
// (u, w) anchor pairs of the (6,1,7) class-5 candidates of one B.
std::vector<std::pair<u64, u64>> candidates617(u64 B);
// find4 jobs of the (6,1,7) classes 1-4 for one B (cls 8 unit records).
std::vector<s615_unit> jobs617(u64 B, int cls);
int free_factor(int cls);

// Build the device record of one caller unit; returns S615_OK (with *skip
// set for units the reference drops) or S615_E_FORMAT for units the engine
// cannot search exactly.
int make_dev_unit(const s615_unit& in, u32 id, DevUnit* out, bool* skip);
// Sinks for unit_items besides a std::vector<u64>: one that counts the items
// a pass would append (it keeps the last one, which a run of job rows
// extends), and one that appends into a window of a preallocated buffer.
struct ItemCount {
  size_t n = 0;
  u64 last = 0;
  bool empty() const { return n == 0; }
  u64& back() { return last; }
  void push_back(u64 it) { ++n; last = it; }
};
struct ItemWriter {
  u64* p = nullptr;
  size_t n = 0;
  bool empty() const { return n == 0; }
  u64& back() { return p[n - 1]; }
  void push_back(u64 it) { p[n++] = it; }
};

// Work items of one packed unit (appended to out).
// Job rows are grouped up to job_rows (<= kJobRows) per item; the row chunks
// of classes 2-5 have unit_rows (<= kItemRows) rows each.
template <class Out>
void unit_items(const DevUnit& d, u32 unit_index, Out& out, u32 job_rows = kJobRows,
                u32 unit_rows = kItemRows, u32 parts3 = 1) {
  if (d.cls == kClsJobRow) {   // runs of up to job_rows consecutive job rows of one kind
    const u32 kind = d.w != 0 ? kJobFind2 : 0u;
    // an item also starts at every multiple of job_rows, so a batch can be
    // itemised in ranges cut there and still give one pass's items
    if (!out.empty() && unit_index % job_rows != 0) {
      const u64 last = out.back();
      if (item_res(last) == kJobItemTag && (item_chunk(last) & kJobFind2) == kind &&
          item_unit(last) + job_count(last) == unit_index && job_count(last) < job_rows) {
        out.back() = last + 1;
        return;
      }
    }
    out.push_back(make_item(unit_index, kJobItemTag, kind | 1u));
    return;
  }
  if (d.cls == 1 || d.cls == S615_CLS_617_FIND4) {   // chunks of the c4 window
    const u32 n = (d.fmax1 - d.fmax2) / kC4Chunk + 1;
    for (u32 c = 0; c < n; ++c) out.push_back(make_item(unit_index, 0, c));
    return;
  }
  const bool c617 = d.cls == (u32)S615_CLS_617;
  const u32 per = c617 ? item_rows(d.cls) : unit_rows;
  const u32 parts = c617 ? kParts617 : (d.cls >= 2 && d.cls <= 4) ? std::max(parts3, 1u) : 1u;
  for (u32 ir = 0; ir < d.nres1; ++ir) {
    u32 jmin = 0, jend = 0;
    class_rows(d.res1[ir], d.mod1, d.fmax1, &jmin, &jend);
    const u32 rows = jend > jmin ? jend - jmin : 0;
    for (u32 c = 0; c * per < rows; ++c)
      for (u32 p = 0; p < parts; ++p) out.push_back(make_item(unit_index, ir, c * parts + p));
  }
}

void gate_patterns(bool gated, int shape, u32 out[kPatWords]);
void tri_tables(u32 out[kTriWords]);
void gate_patterns_sharp(int shape, u32 out[kSharpWords]);
u64 pair_sums_mask64();

}  // namespace s615
