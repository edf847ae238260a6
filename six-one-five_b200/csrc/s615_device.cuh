// s615_device.cuh -- device-side building blocks: table cell loads for the
// three HBM layouts, the xor-filter membership test, exact 128-bit helpers.
#pragma once
#include <cuda_runtime.h>

#include "engine.hpp"

namespace s615 {

// Checked builds (-DS615_CHECKED, `make checked`: lib/libs615_checked.so).
// Every table cell index, work item, unit index and shard index a kernel
// uses is compared with its bound; a failed check sets a
// bit in this file's check word (kChk*) and the access is skipped, so a bug
// shows up as a flag the host reads (s615_check_flags), never as a trap or a
// stray access.  In the default build S615_CHECK is `true` and costs nothing.
// The word is per compiled file (no relocatable device code); each file
// defines its reader with S615_CHECK_TAKE_DEFINE.
constexpr unsigned kChkCell = 1u;      // table cell index >= m (or shard >= S)
constexpr unsigned kChkItem = 2u;      // work item's unit / residue / job run out of range
constexpr unsigned kChkHit = 4u;       // a hit's unit index out of range
constexpr unsigned kChkList = 8u;      // a builder cell index (list entry, key's cells) out of range
#ifdef S615_CHECKED
static __device__ unsigned g_check_word;
#define S615_CHECK(cond, bit) \
  ((cond) ? true : (atomicOr(&::s615::g_check_word, (unsigned)(bit)), false))
#define S615_CHECK_TAKE_DEFINE(name)                                          \
  unsigned name() {                                                           \
    unsigned v = 0;                                                           \
    const unsigned z = 0;                                                     \
    if (cudaMemcpyFromSymbol(&v, ::s615::g_check_word, sizeof v) != cudaSuccess || \
        cudaMemcpyToSymbol(::s615::g_check_word, &z, sizeof z) != cudaSuccess) { \
      cudaGetLastError();                                                     \
      return 0;                                                               \
    }                                                                         \
    return v;                                                                 \
  }
#else
#define S615_CHECK(cond, bit) true
#define S615_CHECK_TAKE_DEFINE(name) \
  unsigned name() { return 0; }
#endif

// Read one r-bit cell.  WIDE layouts hold one cell per aligned word, so a
// cell is one load from one 32-byte sector.  PACKED is the file layout:
// cell i starts at bit i*r; it is assembled from at most two aligned 64-bit
// words (the device buffer is padded so word w+1 always exists).
// Table reads are random and never reused: they skip L1 (.cg) and cap the
// L2 miss fill at 64 bytes (.L2::64B).  Without the cap every miss fills a
// 128-byte line from DRAM; random-access throughput is bound by the HBM
// access rate either way, so the cap halves DRAM bytes at the same speed.
__device__ __forceinline__ u64 ld_cell64(const unsigned long long* p) {
  u64 v;
  asm("ld.global.cg.L2::64B.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ u32 ld_cell32(const unsigned int* p) {
  u32 v;
  asm("ld.global.cg.L2::64B.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

__device__ __forceinline__ u64 load_cell_at(const void* cells, u32 layout, u32 cell_bytes, u32 r,
                                             u64 fpmask, u64 i) {
  if (layout == S615_LAYOUT_WIDE) {
    if (cell_bytes == 8) return ld_cell64(static_cast<const unsigned long long*>(cells) + i);
    return (u64)ld_cell32(static_cast<const unsigned int*>(cells) + i);
  }
  const unsigned long long* p = static_cast<const unsigned long long*>(cells);
  const u64 bit = i * (u64)r;
  const u64 w = bit >> 6;
  const u32 o = (u32)(bit & 63);
  u64 v = ld_cell64(p + w) >> o;
  if (o + r > 64) v |= ld_cell64(p + w + 1) << (64 - o);
  return v & fpmask;
}

__device__ __forceinline__ u64 load_cell(const TableView& t, u64 i) {
  return load_cell_at(t.cells, t.layout, t.cell_bytes, t.r, t.fpmask, i);
}

// xor_might_contain: h = mix64(key + seed), three cells, compare with the
// low r bits of h.
__device__ __forceinline__ bool might_contain_one(const TableView& t, u64 key) {
  if (t.block == 0) return false;
  const u64 h = mix64(key + t.seed);
  u64 c[3];
  cell_indices(h, t.block, t.recip, c);
  if (!S615_CHECK(c[0] < 3 * t.block && c[1] < 3 * t.block && c[2] < 3 * t.block, kChkCell))
    return false;
  const u64 a = load_cell(t, c[0]);
  const u64 b = load_cell(t, c[1]);
  const u64 d = load_cell(t, c[2]);
  return (a ^ b ^ d) == (h & t.fpmask);
}

// A shard set sends the probe to the key's own shard, mix64(key + seed) % S
// (residue-steered probing: one query per probe, as for one table); a set's
// view keeps S and its reciprocal in block / recip.  The hot kernels are
// compiled once per case (kSet), so a single table's probe is unchanged.
// A key whose shard is outside the pass's group [grp_lo, grp_hi) is left to
// the pass that owns that group.
template <bool kSet>
__device__ __forceinline__ bool probe_table(const TableView& t, u64 key) {
  if constexpr (kSet) {
    const u32 s = (u32)fast_mod(mix64(key + t.shard_seed), t.block, t.recip);
    if (!S615_CHECK(s < t.block, kChkCell)) return false;
    if (s - t.grp_lo >= t.grp_hi - t.grp_lo) return false;
    return might_contain_one(t.parts[s], key);
  } else {
    return might_contain_one(t, key);
  }
}

__device__ __forceinline__ bool might_contain(const TableView& t, u64 key) {
  return t.shards > 1 ? probe_table<true>(t, key) : probe_table<false>(t, key);
}

// x^6, exact for x <= 2,642,245 (the largest x with x^3 < 2^64; x^6 < 2^128).
__device__ __forceinline__ u128 pow6_small(u64 x) {
  const u64 x3 = x * x * x;
  return (u128)x3 * x3;
}

// floor(v^(1/6)) for 0 <= v < 2^127 (root < 2,413,000): double estimate, off by at
// most one, then exact fix-up.  The clamp keeps pow6_small(r + 1) exact; it is
// above every root of the domain, so the fix-up takes a step or two.  (A class-5
// row at B = 40,000,000 has V ~ 2^125 and D(e) up to 1.9M.)
__device__ __forceinline__ u32 iroot6_u128(u128 v) {
  if (v == 0) return 0;
  const double x = (double)(u64)(v >> 64) * 18446744073709551616.0 + (double)(u64)v;
  u64 r = (u64)cbrt(sqrt(x));
  if (r > 2642244ull) r = 2642244ull;
  while (r > 0 && pow6_small(r) > v) --r;
  while (pow6_small(r + 1) <= v) ++r;
  return (u32)r;
}

}  // namespace s615
