// engine.hpp -- internal types of the B200 engine (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/s615.h"
#include "s615_common.hpp"

namespace s615 {

// ------------------------------------------------------------ device unit
// One class-5 unit as the sieve kernel consumes it.  Only base mod 2^128 is
// needed: every row quantity V(e) = (base - (14e)^6) / 21^6 is exact and
// below 2^112, so it is recovered from the low 128 bits by the 2-adic
// inverse of 21^6 (the host checks the divisibility this relies on).
struct DevUnit5 {
  u64 base_lo, base_hi;
  u64 B, u;
  u32 fmax1, fmax2, lim, nres1, nres2, id;
  u32 res1[12];
  u32 res2[12];
};
static_assert(sizeof(DevUnit5) == 152, "DevUnit5 layout");

// Gate pattern tables: for q in {9,7,13,19} and a,s in [0,q), bit i of word
// pat[base_q + a*q + s] says whether T = (V - x^6)/64 is an admissible pair
// sum mod q when V = a (mod q) and x = s + 64 i (mod q).
constexpr int kPatQ[4] = {9, 7, 13, 19};
constexpr int kPatBase[4] = {0, 81, 130, 299};
constexpr int kPatB9 = 0, kPatB7 = 81, kPatB13 = 130, kPatB19 = 299;  // usable in device code
constexpr int kPatWords = 660;

// Table resident in HBM.
struct DevTable {
  s615_header hdr{};
  int layout = S615_LAYOUT_WIDE;
  int cell_bytes = 8;        // 4 or 8 for WIDE, 0 for PACKED
  void* d_cells = nullptr;
  size_t bytes = 0;
  u64 block = 0, recip = 0;
};

// Kernel-facing view of a table.
struct TableView {
  const void* cells;
  u64 block, recip, fpmask, seed;
  u32 r, layout, cell_bytes, pad;
};

struct Cls5Counters {  // device accumulators (u64 atomics)
  unsigned long long calls, probes, pos, hits;
};

// Work items of the sieve: (unit, e residue, chunk of kItemRows e-rows),
// packed as unit << 12 | e-residue index << 8 | chunk.
constexpr u32 kItemRows = 64;
constexpr u32 kMaxBatchUnits = 1u << 20;
S615_HD u32 make_item(u32 unit, u32 ie, u32 chunk) { return (unit << 12) | (ie << 8) | chunk; }
S615_HD u32 item_unit(u32 it) { return it >> 12; }
S615_HD u32 item_eres(u32 it) { return (it >> 8) & 15u; }
S615_HD u32 item_chunk(u32 it) { return it & 255u; }
// e-rows of one residue: e = e0 + 729 j for j in [jmin, jend).
S615_HD void e_rows(u32 e0, u32 fmax1, u32* jmin, u32* jend) {
  *jmin = (e0 == 0) ? 1u : 0u;
  *jend = (e0 <= fmax1) ? (fmax1 - e0) / 729u + 1u : 0u;
}

}  // namespace s615

struct s615_batch {
  size_t n_units = 0, n_items = 0;
  s615::DevUnit5* d_units = nullptr;
  s615::u32* d_items = nullptr;
  s615_hit* d_hits = nullptr;
  s615::u32 hit_cap = 0;
  s615::Cls5Counters* d_ctr = nullptr;
  s615::u32* d_work = nullptr;   // persistent-queue cursor
  std::vector<s615::u32> unit_ids;
  std::vector<s615::u32> host_items;
};

struct s615_ctx {
  int device = 0;
  size_t budget = 0, used = 0;
  cudaStream_t stream = nullptr;
  std::map<int, s615::DevTable> tables;
  int next_table = 1;
  s615::u32* d_pat_gate = nullptr;
  s615::u32* d_pat_open = nullptr;
  int num_sms = 0;
  unsigned long long launches = 0;
  std::mutex mu;
};

namespace s615 {

// Status helpers.
int cuda_status(cudaError_t e);
#define S615_CU(x)                                   \
  do {                                               \
    cudaError_t _e = (x);                            \
    if (_e != cudaSuccess) return ::s615::cuda_status(_e); \
  } while (0)

// Budgeted device allocation.
int dev_alloc(s615_ctx* ctx, void** p, size_t bytes);
void dev_free(s615_ctx* ctx, void* p, size_t bytes);

TableView view_of(const DevTable& t);

// Kernel launchers (each returns a status and counts its launches).
int launch_cls5_sieve(s615_ctx* ctx, const TableView& tv, s615_batch* b, unsigned flags,
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
                     DevTable* out);

// Device verifier; see verify.cu.
int verify_cls5_device(s615_ctx* ctx, const s615_unit* units, size_t n_units,
                       const s615_hit* hits, size_t n_hits, int N, s615_solution* out,
                       size_t cap, size_t* n_out);

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
std::vector<u64> unit_candidates(u64 B, int cls);

// Build the device record of one caller unit; returns S615_OK, or
// S615_E_FORMAT when the unit cannot be searched (reference pack_unit5 drops
// it) -- *skip is set for units that are dropped rather than rejected.
int make_dev_unit(const s615_unit& in, u32 id, DevUnit5* out, bool* skip);

void gate_patterns(bool gated, u32 out[kPatWords]);

}  // namespace s615
