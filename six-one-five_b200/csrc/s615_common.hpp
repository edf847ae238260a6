// s615_common.hpp -- constants and small helpers shared by host and device code.
//
// Everything here states a fact of the reference's formats: the mixer
// (spike/ribbon/mix64.hpp:13-25), the cell-index derivation
// (spike/ribbon/xor_filter.hpp:53-60), the packed r-bit cell layout
// (spike/ribbon/xor_pack.hpp:14-23) and the table capacity rule
// (spike/ribbon/xor_filter.hpp:185-192).
#pragma once
#include <cstddef>
#include <cstdint>

#ifdef __CUDACC__
#define S615_HD __host__ __device__ __forceinline__
#else
#define S615_HD inline
#endif

namespace s615 {

using u8 = std::uint8_t;
using u16 = std::uint16_t;
using u32 = std::uint32_t;
using u64 = std::uint64_t;
using i64 = std::int64_t;
using u128 = unsigned __int128;

constexpr u64 kM42 = 5489031744ULL;   // 42^6 = 2^6 * 21^6
constexpr u64 kM21 = 85766121ULL;     // 21^6
constexpr u32 kModE = 729;            // 3^6: e residues
constexpr u32 kModD = 64;             // 2^6: d residues
constexpr u64 kPhi = 0x9E3779B97F4A7C15ULL;
constexpr u64 kSalt2 = 0xBF58476D1CE4E5B9ULL;
constexpr u64 kSeedBase = 0x615615615615615ULL;  // xor_filter.hpp:448
constexpr u32 kMagic = 0x53353136u;              // store_header.hpp:151
constexpr u32 kVersion = 2;
constexpr int kNSoftMax = 120000;                 // fourcore_xor_store.hpp:122

// The reference's 64-bit finaliser (three xor-shift / multiply rounds).
S615_HD u64 mix64(u64 x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33;
  return x;
}

S615_HD u64 fp_mask(u32 r) { return r >= 64 ? ~0ULL : ((1ULL << r) - 1ULL); }

// Packed file layout: m cells of r bits, then 8 pad bytes.
S615_HD u64 packed_bytes(u64 m, u32 r) {
  if (m == 0 || r == 0) return 0;
  return (m * (u64)r + 7) / 8 + 8;
}

// Cells = 1.23 n + 32, rounded up, then up to a multiple of 3.  Computed in
// double exactly as the reference does so that m_cells matches bit for bit.
inline u64 capacity_for(u64 n) {
  const double need = 32.0 + 1.23 * (double)n;
  u64 cap = (u64)(need + 0.999);
  if (cap < 3) cap = 3;
  return (cap + 2) / 3 * 3;
}

// Reciprocal for the exact 64-bit remainder used by every probe: for
// block >= 2, q = umulhi(h, floor((2^64-1)/block)) undershoots h/block by at
// most 2, so two conditional subtractions give h % block exactly.
inline u64 mod_recip(u64 block) { return block >= 2 ? (~0ULL) / block : 0; }

S615_HD u64 mulhi64(u64 a, u64 b) {
#ifdef __CUDA_ARCH__
  return __umul64hi(a, b);
#else
  return (u64)(((u128)a * b) >> 64);
#endif
}

S615_HD u64 fast_mod(u64 h, u64 block, u64 recip) {
  u64 r = h - mulhi64(h, recip) * block;
  if (r >= block) r -= block;
  if (r >= block) r -= block;
  return r;
}

// The three cell indices of a hashed key: one per third of the table.
S615_HD void cell_indices(u64 h, u64 block, u64 recip, u64 out[3]) {
  out[0] = fast_mod(h, block, recip);
  out[1] = fast_mod(mix64(h ^ kPhi), block, recip) + block;
  out[2] = fast_mod(mix64(h ^ kSalt2), block, recip) + 2 * block;
}

}  // namespace s615
