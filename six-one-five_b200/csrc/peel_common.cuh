// peel_common.cuh -- pieces shared by the peel kernels: the row record, the
// residue-gate pattern lookup and small warp and modular helpers.
#pragma once
#include <cuda_runtime.h>

#include "s615_device.cuh"

namespace s615 {

// One sieve row.  cls5: W = V(e); cls2-4: W = T(d); (6,1,7): W = T(d) - c4^6.
struct __align__(16) RowRec {
  u64 wlo, whi;   // row value W mod 2^128
  u32 a;          // cls5: D = iroot6(V-1);   find3 rows: window start lo
  u32 b;          // cls5: V mod 512 or kNoRow; find3 rows: window length | m4 << 28
  u16 off[4];     // pattern-table word offset per q for W mod q
};

__device__ __forceinline__ u32 lanemask_lt() {
  u32 m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// (hi * 2^64 + lo) mod Q for a small constant Q.
constexpr u32 two64_mod(u32 q) {
  u64 r = 1;
  for (int i = 0; i < 64; ++i) r = (r * 2) % q;
  return (u32)r;
}
template <u32 Q>
__device__ __forceinline__ u32 mod_small(u64 hi, u64 lo) {
  return (u32)(((hi % Q) * two64_mod(Q) + lo % Q) % Q);
}

__device__ __forceinline__ void set_offsets(RowRec& R) {
  R.off[0] = (u16)(kPatB9 + 9 * mod_small<9>(R.whi, R.wlo));
  R.off[1] = (u16)(kPatB7 + 7 * mod_small<7>(R.whi, R.wlo));
  R.off[2] = (u16)(kPatB13 + 13 * mod_small<13>(R.whi, R.wlo));
  R.off[3] = (u16)(kPatB19 + 19 * mod_small<19>(R.whi, R.wlo));
}

// Sharp gate offsets: q = 27, 49, 13, 19 in the row record, 31, 37, 43 in offx.
__device__ __forceinline__ void set_offsets_sharp(RowRec& R, u16* offx) {
  R.off[0] = (u16)(kSB27 + 27 * mod_small<27>(R.whi, R.wlo));
  R.off[1] = (u16)(kSB49 + 49 * mod_small<49>(R.whi, R.wlo));
  R.off[2] = (u16)(kSB13 + 13 * mod_small<13>(R.whi, R.wlo));
  R.off[3] = (u16)(kSB19 + 19 * mod_small<19>(R.whi, R.wlo));
  offx[0] = (u16)(kSB31 + 31 * mod_small<31>(R.whi, R.wlo));
  offx[1] = (u16)(kSB37 + 37 * mod_small<37>(R.whi, R.wlo));
  offx[2] = (u16)(kSB43 + 43 * mod_small<43>(R.whi, R.wlo));
}

// The three extra sharp words of one lane.
__device__ __forceinline__ u32 gate_word3(const u32* pat, const u16* offx, u32 s31, u32 s37,
                                          u32 s43) {
  return pat[offx[0] + s31] & pat[offx[1] + s37] & pat[offx[2] + s43];
}

// x^6 mod 4096 (and so mod 64) for x < 2^32.
__device__ __forceinline__ u32 pow6_mod4096(u32 x) {
  x &= 4095u;
  const u32 x2 = (x * x) & 4095u;
  const u32 x3 = (x2 * x) & 4095u;
  return (x3 * x3) & 4095u;
}

// The gate word of one lane: bits for 32 consecutive columns.
__device__ __forceinline__ u32 gate_word(const u32* pat, const RowRec& R, u32 s9, u32 s7, u32 s13,
                                         u32 s19) {
  const uint2 offs = *reinterpret_cast<const uint2*>(&R.off[0]);
  return pat[(offs.x & 0xFFFFu) + s9] & pat[(offs.x >> 16) + s7] & pat[(offs.y & 0xFFFFu) + s13] &
         pat[(offs.y >> 16) + s19];
}

// Least c >= 1 with 3 c^6 >= T, for 1 <= T < 2^127 (min_c_fix,
// solve_617_v1.cu:430-436, and the window start of make_cand mode 3,
// fourcore_find_v4.cu:411-416): a double estimate, then an exact fix-up.  The
// answer is below 1.95M; the clamp at 2^21 keeps 3 c^6 < 2^128.
__device__ __forceinline__ u32 least_c_3c6(u128 T) {
  const double x = ((double)(u64)(T >> 64) * 18446744073709551616.0 + (double)(u64)T) / 3.0;
  u64 c = (u64)cbrt(sqrt(x));
  if (c < 1) c = 1;
  if (c > (1ULL << 21)) c = 1ULL << 21;
  while (3 * pow6_small(c) < T) ++c;
  while (c > 1 && 3 * pow6_small(c - 1) >= T) --c;
  return (u32)c;
}

}  // namespace s615
