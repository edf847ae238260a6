// xor_build.cu -- device construction of the 3-hash xor filter.
//
// Produces a table with the reference's header (n_keys, m_cells, mix_seed,
// seed schedule: spike/ribbon/xor_filter.hpp:185-192,256-470 and
// fourcore_xor_store.hpp:67-119) from the same key set, built on the GPU:
//
//  1. Key set.  Pair mode enumerates unordered pairs of the DISTINCT values
//     of i^6 mod 2^64 (1<=i<=N); many i share a value (every multiple of 2048
//     has i^6 = 0 mod 2^64), so this already removes most duplicate keys.
//     Remaining duplicates are removed by an open-addressing hash set in HBM
//     (the reference sorts + uniques).  The survivors are the unique keys.
//  2. Incidence: every cell is one 64-bit word, count << 42 | sum of the
//     indices of its keys, and each key adds (1 << 42) + index to its three
//     cells (binned by L2-sized cell slice when HBM allows).
//  3. Peel in rounds.  A cell with count 1 holds exactly one key, named by
//     its index; in round r every such key is claimed by the lowest of its
//     count-1 cells (so a key is claimed once), then removed from its other
//     two cells.  The 2-core is unique, so peeling succeeds for exactly the
//     seeds for which the reference's FIFO peel succeeds.
//  4. Fill in reverse round order, in place: the claimed cell of a round-r key
//     becomes fp(h) ^ cell(c1) ^ cell(c2).  Its other cells were never claimed
//     in rounds <= r (a count-1 cell cannot hold a second unpeeled key), so
//     they are final already and a round needs no ordering inside it.
// Cells then hold exactly the reference's cell relation (FN = 0, same FPR);
// which key owns which cell differs from the FIFO order, so bytes differ.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "s615_device.cuh"

namespace s615 {

namespace {

namespace cg = cooperative_groups;

constexpr u64 kEmpty = ~0ULL;

// Bytes the context's HBM budget still allows (one read of the shared count).
size_t budget_room(const s615_ctx* ctx) {
  const size_t u = ctx->used.load();
  return ctx->budget > u ? ctx->budget - u : 0;
}

int grid_for(s615_ctx* ctx, u64 n, int threads) {
  const u64 want = (n + threads - 1) / threads;
  const u64 cap = (u64)ctx->num_sms * 16;
  return (int)(want < cap ? (want ? want : 1) : cap);
}

__device__ __forceinline__ void hset_insert(unsigned long long* table, u64 tmask, u64 key,
                                            u32* has_empty_key) {
  if (key == kEmpty) { *has_empty_key = 1; return; }
  u64 pos = mix64(key ^ 0x5bd1e9955bd1e995ULL) & tmask;
  for (u64 probe = 0; probe <= tmask; ++probe) {
    const unsigned long long old = atomicCAS(table + pos, (unsigned long long)kEmpty,
                                             (unsigned long long)key);
    if (old == kEmpty || old == key) return;
    pos = (pos + 1) & tmask;
  }
}

// Which keys this build takes: the memory partition (top bits of mix64(key))
// and, for one shard of a set, mix64(key + kShardSeed) % shards == shard.
struct KeyFilter {
  u32 part_bits, part, shards, shard;
  u64 srecip;
  __device__ __forceinline__ bool take(u64 key) const {
    if (part_bits && (mix64(key) >> (64 - part_bits)) != part) return false;
    return shards <= 1 || fast_mod(mix64(key + kShardSeed), shards, srecip) == shard;
  }
};

// Pair keys u[a] + u[b], a <= b, one block-stride row per a.
__global__ void k_insert_pairs(const u64* __restrict__ vals, u64 nv, unsigned long long* table,
                               u64 tmask, KeyFilter kf, u32* has_empty_key) {
  for (u64 a = blockIdx.x; a < nv; a += gridDim.x) {
    const u64 va = vals[a];
    for (u64 b = a + threadIdx.x; b < nv; b += blockDim.x) {
      const u64 key = va + vals[b];
      if (kf.take(key)) hset_insert(table, tmask, key, has_empty_key);
    }
  }
}

__global__ void k_insert_keys(const u64* __restrict__ keys, u64 n, unsigned long long* table,
                              u64 tmask, KeyFilter kf, u32* has_empty_key) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n;
       i += (u64)gridDim.x * blockDim.x) {
    const u64 key = keys[i];
    if (kf.take(key)) hset_insert(table, tmask, key, has_empty_key);
  }
}

// Append occupied slots to out (order irrelevant); slots past cap are
// counted, not written.
// The flagged threads' positions in a list whose length is *count, with ONE
// global atomic per block (a shared-memory scan of the warps' counts): the
// lists' counters are single addresses, and per-warp atomics on them
// serialise in their L2 slice.  Every thread of the block calls this (it
// synchronises the block); ~0 for a thread that takes nothing.
__device__ __forceinline__ u64 block_reserve(bool take, unsigned long long* count) {
  __shared__ u32 s_cnt[32];
  __shared__ unsigned long long s_base;
  const u32 lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  const u32 b = __ballot_sync(0xFFFFFFFFu, take);
  __syncthreads();   // the previous call's offsets have been read
  if (lane == 0) s_cnt[wid] = __popc(b);
  __syncthreads();
  if (threadIdx.x == 0) {
    u32 tot = 0;
    for (u32 w = 0; w < nw; ++w) {
      const u32 k = s_cnt[w];
      s_cnt[w] = tot;
      tot += k;
    }
    s_base = tot ? atomicAdd(count, (unsigned long long)tot) : 0ull;
  }
  __syncthreads();
  return take ? s_base + s_cnt[wid] + __popc(b & ((1u << lane) - 1u)) : ~0ull;
}

__global__ void k_compact(const unsigned long long* __restrict__ table, u64 tsize,
                          u64* __restrict__ out, u64 cap, unsigned long long* n_out) {
  for (u64 i0 = blockIdx.x * (u64)blockDim.x; i0 < tsize; i0 += (u64)gridDim.x * blockDim.x) {
    const u64 i = i0 + threadIdx.x;
    const bool occ = i < tsize && table[i] != kEmpty;
    const u64 k = block_reserve(occ, n_out);   // every thread of the block, every pass
    if (occ && k < cap) out[k] = table[i];
  }
}

// ---- cell words -------------------------------------------------------------
// During the build every cell is one 64-bit word: the number of unpeeled keys
// in the cell above bit 42 and the sum of their key indices below it.  An
// update of a cell is then one atomic add (the reference's incidence keeps an
// xor of hashes and a count: two arrays, two read-modify-writes per update),
// and a cell of count 1 names its key directly; the key's hash is
// recomputed from the key array.  Indices are below 2^34 and a count above
// 255 fails the build, so the sum never reaches bit 42.  After the peel the
// word array is filled in place with the final r-bit cells.
constexpr int kCntShift = 42;
constexpr u64 kSumMask = (1ull << kCntShift) - 1;
constexpr u64 kMaxKeys = 1ull << 34;
__device__ __forceinline__ u64 cnt_of(u64 w) { return w >> kCntShift; }
__device__ __forceinline__ u64 upd(u64 idx) { return (1ull << kCntShift) + idx; }

// Checked builds: the key and cell counts of the build in flight, set before
// the incidence, bound every key index a kernel decodes (from a loop or from a
// cell word's index sum) and the cells of the binned apply.  One build at a
// time per process in such a build.
#ifdef S615_CHECKED
static __device__ u64 g_check_nkeys, g_check_ncells;
#define S615_KEY_OK(idx) S615_CHECK((idx) < g_check_nkeys, kChkList)
#define S615_CELL_OK(c) S615_CHECK((c) < g_check_ncells, kChkList)
#else
#define S615_KEY_OK(idx) true
#define S615_CELL_OK(c) true
#endif

__device__ __forceinline__ u64 key_hash(const u64* keys, u64 idx, u64 seed) {
  if (!S615_KEY_OK(idx)) return 0;
  return mix64(keys[idx] + seed);
}

// Checked builds: all three cells of a key lie in [0, 3 * block).
__device__ __forceinline__ bool cells_ok(const u64* c, u64 block) {
  return S615_CHECK(c[0] < 3 * block && c[1] < 3 * block && c[2] < 3 * block, kChkList);
}

__global__ void k_incidence(const u64* __restrict__ keys, u64 n, u64 seed, u64 block, u64 recip,
                            unsigned long long* W) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n;
       i += (u64)gridDim.x * blockDim.x) {
    u64 c[3];
    cell_indices(key_hash(keys, i, seed), block, recip, c);
    if (!cells_ok(c, block)) continue;
#pragma unroll
    for (int t = 0; t < 3; ++t) atomicAdd(W + c[t], (unsigned long long)upd(i));
  }
}

// The largest count of any cell (a count above 255 fails the build).
__global__ void k_max_count(const unsigned long long* __restrict__ W, u64 m, unsigned* mx) {
  unsigned local = 0;
  for (u64 c = blockIdx.x * (u64)blockDim.x + threadIdx.x; c < m; c += (u64)gridDim.x * blockDim.x)
    { const u64 k = cnt_of(W[c]); local = max(local, k > 0xFFFFFFFFull ? 0xFFFFFFFFu : (unsigned)k); }
#pragma unroll
  for (int o = 16; o; o >>= 1) local = max(local, __shfl_xor_sync(0xFFFFFFFFu, local, o));
  if ((threadIdx.x & 31) == 0 && local) atomicMax(mx, local);
}

// ---- incidence through shared-memory radix bins ---------------------------
// The cells are cut into slices of 2^sbits cells (16 MB of cell words:
// L2-sized).  Each block takes a fixed range of keys.  k_bin_count counts the
// block's updates per slice in a shared-memory histogram; a host scan over
// (slice, block) gives every block its own output range per slice;
// k_bin_scatter bins the updates through shared-memory cursors into those
// ranges (slice-local cell offset and key index, 8 B), so the updates of a
// slice lie together; k_bin_apply walks them slice by slice with the whole
// grid, and its atomic adds land on a slice that is resident in L2.
constexpr u32 kMaxSlices = 4608;
constexpr int kBinThreads = 256;

__global__ void k_bin_count(const u64* __restrict__ keys, u64 k0, u64 per, u64 k1, u64 seed,
                            u64 block, u64 recip, u32 sbits, u32 S, u32* __restrict__ bhist) {
  extern __shared__ u32 hist[];
  for (u32 i = threadIdx.x; i < S; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  const u64 lo = k0 + blockIdx.x * per, hi = min(k1, lo + per);
  for (u64 i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    u64 c[3];
    cell_indices(key_hash(keys, i, seed), block, recip, c);
    if (!cells_ok(c, block) || !S615_CHECK(((3 * block - 1) >> sbits) < S, kChkList)) continue;
#pragma unroll
    for (int t = 0; t < 3; ++t) atomicAdd(&hist[(u32)(c[t] >> sbits)], 1u);
  }
  __syncthreads();
  for (u32 i = threadIdx.x; i < S; i += blockDim.x) bhist[(u64)blockIdx.x * S + i] = hist[i];
}

__global__ void k_bin_scatter(const u64* __restrict__ keys, u64 k0, u64 per, u64 k1, u64 seed,
                              u64 block, u64 recip, u32 sbits, u32 S,
                              const unsigned long long* __restrict__ bbase,
                              unsigned long long* __restrict__ ent) {
  extern __shared__ unsigned long long cur[];
  for (u32 i = threadIdx.x; i < S; i += blockDim.x) cur[i] = bbase[(u64)blockIdx.x * S + i];
  __syncthreads();
  const u64 lo = k0 + blockIdx.x * per, hi = min(k1, lo + per);
  const u64 lmask = (1ull << sbits) - 1;
  for (u64 i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    u64 c[3];
    cell_indices(key_hash(keys, i, seed), block, recip, c);
    if (!cells_ok(c, block) || !S615_CHECK(((3 * block - 1) >> sbits) < S, kChkList)) continue;
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      const unsigned long long pos = atomicAdd(&cur[(u32)(c[t] >> sbits)], 1ull);
      ent[pos] = ((u64)(i - k0) << 32) | (c[t] & lmask);   // one 8-byte store per update
    }
  }
}

// A cooperative grid walks the slices in order and splits each slice's
// entries over all its threads, with a grid-wide sync after every slice, so
// the whole GPU works on one slice (16 MB) at a time and its atomic adds hit
// in L2.  (Without the syncs, blocks drift apart over the walk and the slices
// in use outgrow L2.)
// kSync = false is the same walk without the syncs, for a device or setting
// where a cooperative launch is refused (the result is the same; only the L2
// hit rate suffers).
template <bool kSync>
__global__ void k_bin_apply(const unsigned long long* __restrict__ ent, u64 k0,
                            const unsigned long long* __restrict__ soff, u32 sbits, u32 S,
                            unsigned long long* W) {
  const u64 nt = (u64)gridDim.x * blockDim.x, tid = blockIdx.x * (u64)blockDim.x + threadIdx.x;
  for (u32 sl = 0; sl < S; ++sl) {
    unsigned long long* base = W + ((u64)sl << sbits);
    const u64 e1 = soff[sl + 1];
    for (u64 i = soff[sl] + tid; i < e1; i += nt) {
      const u64 e = ent[i];
      const u32 off = (u32)e, idx = (u32)(e >> 32);
      if (S615_KEY_OK(k0 + idx) && S615_CELL_OK(((u64)sl << sbits) + off))
        atomicAdd(base + off, (unsigned long long)upd(k0 + idx));
    }
    if constexpr (kSync) cg::this_grid().sync();
  }
}

// ---- peel ------------------------------------------------------------------
// Round r claims every key whose lowest count-1 cell is a count-1 cell (so a
// key is claimed once), then removes each claimed key from its two other
// cells; a claimed cell keeps its key's index with count 0.  Every count-1
// cell at the start of round r > 1 got its count 1 while round r-1 removed
// keys (a count-1 cell of round r-1 either claimed its key or lost it to a
// lower cell of the same key), so after a full scan in round 1 each round
// visits only the cells whose count went from 2 to 1 in the round before.
// Claimed cells are appended in round order (as offsets within their third
// of the table), and the fill walks that list backwards.  Without room for
// the lists every round scans all cells and tags its claims with the round.

// A list of cells, each entry a u32 offset within its third of the table and
// the third (0, 1, 2) in a byte: a cell index needs more than 32 bits once m
// passes 2^32, an offset within a third does not (block < 2^32 for every
// single table).
struct CellList {
  u32* off;
  u8* third;
  __host__ __device__ CellList at(u64 k) const { return CellList{off + k, third + k}; }
  __device__ __forceinline__ u64 cell(u64 k, u64 block) const { return third[k] * block + off[k]; }
};

// Append up to two flagged cells per thread with ONE global atomic per block:
// each warp's count goes to shared memory, thread 0 reserves the block's
// total, and every lane writes at its offset.  All appends of a list go
// through one counter, so per-warp atomics on it serialise in its L2 slice:
// at ~1.7e8 such atomics/s they bound the round's apply (ncu: DRAM 11%, L2 5%,
// 578 long-scoreboard stall cycles per issue); per block they are 8x fewer.
// Every thread of the block calls this (it synchronises the block); it
// returns the first entry's position, or ~0 when not taken or over capacity.
__device__ __forceinline__ u64 block_append(bool take0, u64 c0, bool take1, u64 c1, u64 block,
                                            CellList list, unsigned long long* count, u64 cap,
                                            u32* over) {
  __shared__ u32 s_cnt[32];
  __shared__ unsigned long long s_base;
  const u32 lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  const u32 b0 = __ballot_sync(0xFFFFFFFFu, take0), b1 = __ballot_sync(0xFFFFFFFFu, take1);
  __syncthreads();   // the previous call's offsets have been read
  if (lane == 0) s_cnt[wid] = __popc(b0) + __popc(b1);
  __syncthreads();
  if (threadIdx.x == 0) {
    u32 tot = 0;
    for (u32 w = 0; w < nw; ++w) {
      const u32 k = s_cnt[w];
      s_cnt[w] = tot;
      tot += k;
    }
    s_base = tot ? atomicAdd(count, (unsigned long long)tot) : 0ull;
  }
  __syncthreads();
  const u64 at0 = s_base + s_cnt[wid] + __popc(b0 & ((1u << lane) - 1u));
  const u64 at1 = s_base + s_cnt[wid] + __popc(b0) + __popc(b1 & ((1u << lane) - 1u));
  u64 first = ~0ull;
  if (take0) {
    if (at0 < cap) {
      const u32 t = c0 >= 2 * block ? 2u : c0 >= block ? 1u : 0u;
      list.off[at0] = (u32)(c0 - t * block);
      list.third[at0] = (u8)t;
      first = at0;
    } else {
      *over = 1;
    }
  }
  if (take1) {
    if (at1 < cap) {
      const u32 t = c1 >= 2 * block ? 2u : c1 >= block ? 1u : 0u;
      list.off[at1] = (u32)(c1 - t * block);
      list.third[at1] = (u8)t;
    } else {
      *over = 1;
    }
  }
  return first;
}

// The claimed cells of the peel, in round order.  With idx and hash set
// (HBM permitting: they reuse the incidence's entry buffers) the claim also
// records each claimed key's index and hash, so the apply and the fill read
// them in order instead of fetching the cell word and the key again.
struct ClaimList {
  CellList cells;
  u32* idx;                    // null: read from the cell word
  unsigned long long* hash;    // null: recomputed from the key array
  __host__ __device__ ClaimList at(u64 k) const {
    return ClaimList{cells.at(k), idx ? idx + k : nullptr, hash ? hash + k : nullptr};
  }
};

// Does cell c (count 1) claim its key?  The key's lower count-1 cells win.
__device__ __forceinline__ bool claims(const unsigned long long* W, const u64* keys, u64 seed,
                                       u64 block, u64 recip, u64 c, u64 w, u64& h) {
  h = key_hash(keys, w & kSumMask, seed);
  u64 cs[3];
  cell_indices(h, block, recip, cs);
  if (!cells_ok(cs, block)) return false;
#pragma unroll
  for (int t = 0; t < 3; ++t)
    if (cs[t] < c && cnt_of(W[cs[t]]) == 1) return false;
  return true;
}

// Claims among the candidate cells [0, ncand), or among every cell when the
// candidate list is null.
__global__ void k_claim_list(CellList cand, u64 ncand, const unsigned long long* __restrict__ W,
                             const u64* __restrict__ keys, u64 seed, u64 block, u64 recip,
                             ClaimList out, unsigned long long* n_order, u64 order_cap, u32* over) {
  for (u64 base = blockIdx.x * (u64)blockDim.x; base < ncand; base += (u64)gridDim.x * blockDim.x) {
    const u64 i = base + threadIdx.x;
    bool claim = false;
    u64 c = 0, w = 0, h = 0;
    if (i < ncand) {
      c = cand.off ? cand.cell(i, block) : i;
      if (S615_CHECK(c < 3 * block, kChkList)) {
        w = W[c];
        claim = cnt_of(w) == 1 && claims(W, keys, seed, block, recip, c, w, h);
      }
    }
    const u64 k = block_append(claim, c, false, 0, block, out.cells, n_order, order_cap, over);
    if (k != ~0ull && out.hash) {
      out.idx[k] = (u32)(w & kSumMask);
      out.hash[k] = h;
    }
  }
}

// Claimed keys a thread applies per pass of k_apply_list: their eight atomics
// are in flight together, and the block synchronises (in the append) once
// per pass instead of once per key.
constexpr int kApplyPer = 4;

// block_append for K cells per thread (flags take[k], cells c[k]), one global
// atomic per block; every thread of the block calls it.
template <int K>
__device__ __forceinline__ void block_append_n(const bool (&take)[K], const u64 (&c)[K], u64 block,
                                               CellList list, unsigned long long* count, u64 cap,
                                               u32* over) {
  __shared__ u32 s_cnt[32];
  __shared__ unsigned long long s_base;
  const u32 lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  u32 b[K];
  u32 wtot = 0;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    b[k] = __ballot_sync(0xFFFFFFFFu, take[k]);
    wtot += __popc(b[k]);
  }
  __syncthreads();   // the previous call's offsets have been read
  if (lane == 0) s_cnt[wid] = wtot;
  __syncthreads();
  if (threadIdx.x == 0) {
    u32 tot = 0;
    for (u32 w = 0; w < nw; ++w) {
      const u32 n = s_cnt[w];
      s_cnt[w] = tot;
      tot += n;
    }
    s_base = tot ? atomicAdd(count, (unsigned long long)tot) : 0ull;
  }
  __syncthreads();
  u64 at = s_base + s_cnt[wid];
  const u32 below = (1u << lane) - 1u;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (take[k]) {
      const u64 pos = at + __popc(b[k] & below);
      if (pos < cap) {
        const u32 t = c[k] >= 2 * block ? 2u : c[k] >= block ? 1u : 0u;
        list.off[pos] = (u32)(c[k] - t * block);
        list.third[pos] = (u8)t;
      } else {
        *over = 1;
      }
    }
    at += __popc(b[k]);
  }
}

__global__ void k_apply_list(ClaimList in, u64 L, unsigned long long* W,
                             const u64* __restrict__ keys, u64 seed, u64 block, u64 recip,
                             CellList next, unsigned long long* n_next, u64 next_cap, u32* over) {
  const u64 span = (u64)blockDim.x * kApplyPer;
  for (u64 base = blockIdx.x * span; base < L; base += (u64)gridDim.x * span) {
    bool to[2 * kApplyPer];
    u64 nc[2 * kApplyPer];
    u64 old[2 * kApplyPer];
#pragma unroll
    for (int q = 0; q < kApplyPer; ++q) {
      to[2 * q] = to[2 * q + 1] = false;
      nc[2 * q] = nc[2 * q + 1] = 0;
      old[2 * q] = old[2 * q + 1] = 0;
      const u64 i = base + (u64)q * blockDim.x + threadIdx.x;   // coalesced over the block
      if (i < L && S615_CHECK(in.cells.cell(i, block) < 3 * block, kChkList)) {
        const u64 c = in.cells.cell(i, block);
        u64 idx, h;
        if (in.hash) {
          idx = in.idx[i];
          h = in.hash[i];
        } else {
          idx = W[c] & kSumMask;
          h = key_hash(keys, idx, seed);
        }
        // remove the key from its two other cells (results read below, so the
        // atomics of all kApplyPer keys are in flight together)
        u64 cs[3];
        cell_indices(h, block, recip, cs);
        if (cells_ok(cs, block) && S615_KEY_OK(idx)) {   // always true in the default build
          const int own = cs[0] == c ? 0 : cs[1] == c ? 1 : 2;
          nc[2 * q] = cs[own == 0 ? 1 : 0];
          nc[2 * q + 1] = cs[own == 2 ? 1 : 2];
          old[2 * q] = atomicAdd(W + nc[2 * q], (unsigned long long)(0 - upd(idx)));
          old[2 * q + 1] = atomicAdd(W + nc[2 * q + 1], (unsigned long long)(0 - upd(idx)));
          to[2 * q] = to[2 * q + 1] = true;   // pending: the count check follows
          // count 0; without the recorded index the word keeps it for the fill
          W[c] = in.hash ? 0ull : idx;
        }
      }
    }
    // a cell whose count went from 2 to 1 is a candidate of the next round
#pragma unroll
    for (int k = 0; k < 2 * kApplyPer; ++k) to[k] = to[k] && cnt_of(old[k]) == 2;
    // every thread of the block reaches the append (it synchronises the block)
    block_append_n<2 * kApplyPer>(to, nc, block, next, n_next, next_cap, over);
  }
}

// Reverse fill of claimed cell c: fingerprint of its key xor its two other
// cells, which are final already (filled in a later round, or never claimed
// and 0).
__device__ __forceinline__ void fill_cell(unsigned long long* W, u64 h, u64 block, u64 recip,
                                          u64 mask, u64 c) {
  u64 cs[3];
  cell_indices(h, block, recip, cs);
  if (!cells_ok(cs, block) || !S615_CHECK(c < 3 * block, kChkList)) return;
  u64 v = h & mask;
#pragma unroll
  for (int t = 0; t < 3; ++t)
    if (cs[t] != c) v ^= W[cs[t]];
  W[c] = v & mask;
}

__global__ void k_fill_list(ClaimList in, u64 L, unsigned long long* W,
                            const u64* __restrict__ keys, u64 seed, u64 block, u64 recip, u64 mask) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < L;
       i += (u64)gridDim.x * blockDim.x) {
    const u64 c = in.cells.cell(i, block);
    const u64 h = in.hash ? (u64)in.hash[i] : key_hash(keys, W[c], seed);
    fill_cell(W, h, block, recip, mask, c);
  }
}

// remove_key for the scan form (index and hash from the cell word and keys).
__device__ __forceinline__ void remove_key_scan(unsigned long long* W, const u64* keys, u64 seed,
                                                u64 block, u64 recip, u64 c) {
  const u64 idx = W[c] & kSumMask;
  u64 cs[3];
  cell_indices(key_hash(keys, idx, seed), block, recip, cs);
  if (!cells_ok(cs, block) || !S615_KEY_OK(idx)) return;
#pragma unroll
  for (int t = 0; t < 3; ++t)
    if (cs[t] != c) atomicAdd(W + cs[t], (unsigned long long)(0 - upd(idx)));
  W[c] = idx;   // count 0; the index stays for the fill
}

// The scan form: claims of round r tagged in round[], apply and fill by tag.
__global__ void k_claim_scan(const unsigned long long* __restrict__ W, const u64* __restrict__ keys,
                             u64 seed, u16* __restrict__ round, u64 m, u64 block, u64 recip, u16 r,
                             unsigned long long* n_claimed) {
  for (u64 c0 = blockIdx.x * (u64)blockDim.x; c0 < m; c0 += (u64)gridDim.x * blockDim.x) {
    const u64 c = c0 + threadIdx.x;
    bool claim = false;
    if (c < m) {
      const u64 w = W[c];
      u64 h;
      claim = cnt_of(w) == 1 && claims(W, keys, seed, block, recip, c, w, h);
      if (claim) round[c] = r;
    }
    block_reserve(claim, n_claimed);   // counts the claims (every thread, every pass)
  }
}

__global__ void k_apply_scan(unsigned long long* W, const u64* __restrict__ keys, u64 seed,
                             const u16* __restrict__ round, u64 m, u64 block, u64 recip, u16 r) {
  for (u64 c = blockIdx.x * (u64)blockDim.x + threadIdx.x; c < m;
       c += (u64)gridDim.x * blockDim.x) {
    if (round[c] == r) remove_key_scan(W, keys, seed, block, recip, c);
  }
}

__global__ void k_fill_scan(unsigned long long* W, const u64* __restrict__ keys, u64 seed,
                            const u16* __restrict__ round, u64 m, u64 block, u64 recip, u16 r,
                            u64 mask) {
  for (u64 c = blockIdx.x * (u64)blockDim.x + threadIdx.x; c < m;
       c += (u64)gridDim.x * blockDim.x)
    if (round[c] == r) fill_cell(W, key_hash(keys, W[c], seed), block, recip, mask, c);
}

__global__ void k_narrow(const u64* __restrict__ in, u32* __restrict__ out, u64 m) {
  for (u64 c = blockIdx.x * (u64)blockDim.x + threadIdx.x; c < m;
       c += (u64)gridDim.x * blockDim.x)
    out[c] = (u32)in[c];
}

struct Buf {
  s615_ctx* ctx;
  void* p = nullptr;
  size_t n = 0;
  explicit Buf(s615_ctx* c) : ctx(c) {}
  int alloc(size_t bytes) { n = bytes; return dev_alloc(ctx, &p, bytes); }
  void release() { if (p) dev_free(ctx, p, n); p = nullptr; n = 0; }
  ~Buf() { release(); }
};

u64 pow2_at_least(u64 x) { u64 p = 1; while (p < x) p <<= 1; return p; }

// Incidence of keys [0, n) for one seed through the slice bins, in chunks of
// keys whose updates fit the entry buffers (ent_cap updates).
int incidence_binned(s615_ctx* ctx, const u64* keys, u64 n, u64 seed, u64 m, u64 block, u64 recip,
                     unsigned long long* ent, u64 ent_cap, unsigned long long* W, u32* bhist,
                     unsigned long long* bbase, cudaStream_t st) {
  u32 sbits = 21;
  while (((m + (1ull << sbits) - 1) >> sbits) > kMaxSlices) ++sbits;
  const u32 S = (u32)((m + (1ull << sbits) - 1) >> sbits);
  const int G = ctx->num_sms * 2;
  const u64 chunk = std::max<u64>(1, std::min<u64>(ent_cap / 3, 1ull << 32));
  std::vector<u32> h_hist((size_t)G * S);
  std::vector<unsigned long long> h_base((size_t)G * S), h_soff(S + 1);
  for (u64 k0 = 0; k0 < n; k0 += chunk) {
    const u64 k1 = std::min(n, k0 + chunk);
    const u64 per = (k1 - k0 + G - 1) / G;
    k_bin_count<<<G, kBinThreads, S * sizeof(u32), st>>>(keys, k0, per, k1, seed, block, recip, sbits,
                                                         S, bhist);
    ctx->launches++;
    S615_CU(cudaGetLastError());
    S615_CU(cudaMemcpyAsync(h_hist.data(), bhist, h_hist.size() * sizeof(u32), cudaMemcpyDeviceToHost, st));
    S615_CU(cudaStreamSynchronize(st));
    // exclusive scan in (slice, block) order: slice s's updates are contiguous
    unsigned long long run = 0;
    for (u32 sl = 0; sl < S; ++sl) {
      h_soff[sl] = run;
      for (int b = 0; b < G; ++b) {
        h_base[(size_t)b * S + sl] = run;
        run += h_hist[(size_t)b * S + sl];
      }
    }
    h_soff[S] = run;
    if (run != 3 * (k1 - k0)) return S615_E_DEVICE;
    S615_CU(cudaMemcpyAsync(bbase, h_base.data(), h_base.size() * sizeof(unsigned long long),
                            cudaMemcpyHostToDevice, st));
    k_bin_scatter<<<G, kBinThreads, S * sizeof(unsigned long long), st>>>(
        keys, k0, per, k1, seed, block, recip, sbits, S, bbase, ent);
    ctx->launches++;
    S615_CU(cudaGetLastError());
    // the slice starts go where the block bases were (read by the apply kernel)
    S615_CU(cudaMemcpyAsync(bbase, h_soff.data(), (S + 1) * sizeof(unsigned long long),
                            cudaMemcpyHostToDevice, st));
    int per_sm = 0;
    S615_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bin_apply<true>, 256, 0));
    const dim3 grid(ctx->num_sms * std::max(per_sm, 1));
    {   // cooperative: every block resident at once (the launch is refused otherwise)
      const unsigned long long* a_ent = ent;
      const unsigned long long* a_soff = bbase;
      u64 a_k0 = k0;
      u32 a_sbits = sbits, a_S = S;
      void* args[] = {(void*)&a_ent, (void*)&a_k0, (void*)&a_soff, (void*)&a_sbits, (void*)&a_S,
                      (void*)&W};
      if (cudaLaunchCooperativeKernel((const void*)k_bin_apply<true>, grid, dim3(256), args, 0, st) !=
          cudaSuccess) {
        cudaGetLastError();
        k_bin_apply<false><<<grid, 256, 0, st>>>(ent, k0, bbase, sbits, S, W);
      }
    }
    ctx->launches++;
    S615_CU(cudaGetLastError());
    S615_CU(cudaStreamSynchronize(st));   // h_base / h_soff are reused by the next chunk
  }
  return S615_OK;
}

// S615_TRACE: per-phase device times of a build on stderr (CUDA events on
// the build stream).
struct PhaseTrace {
  bool on = std::getenv("S615_TRACE") != nullptr;
  cudaStream_t st;
  std::vector<std::pair<const char*, cudaEvent_t>> marks;
  explicit PhaseTrace(cudaStream_t s) : st(s) {}
  void mark(const char* name) {
    nvtxMarkA(name);   // the phase boundary on a profiler's timeline
    if (!on) return;
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); return; }
    cudaEventRecord(e, st);
    marks.emplace_back(name, e);
  }
  void report(u64 n, u64 m, int rounds) {
    if (!on || marks.size() < 2) return;
    cudaEventSynchronize(marks.back().second);
    std::fprintf(stderr, "[xor-build] keys=%llu cells=%llu rounds=%d", (unsigned long long)n,
                 (unsigned long long)m, rounds);
    for (size_t i = 1; i < marks.size(); ++i) {
      float ms = 0;
      cudaEventElapsedTime(&ms, marks[i - 1].second, marks[i].second);
      std::fprintf(stderr, " %s=%.1fms", marks[i].first, ms);
    }
    std::fprintf(stderr, "\n");
  }
  ~PhaseTrace() {
    for (auto& m : marks) cudaEventDestroy(m.second);
  }
};

}  // namespace

int build_xor_device(s615_ctx* ctx, const u64* d_pair_vals, u64 n_vals, const u64* d_keys,
                     u64 n_keys, int r, const u64* seeds, int n_seeds, int N, int layout,
                     DevTable* out, u32 shards, u32 shard) {
  cudaStream_t st = ctx->stream;
  const bool pairs = d_pair_vals != nullptr;
  if (shards < 1) shards = 1;
  if (shard >= shards) return S615_E_ARG;
  const u64 n_all = pairs ? n_vals * (n_vals + 1) / 2 : n_keys;
  // one shard's share of the keys, with room for the binomial spread
  const u64 n_raw = shards == 1 ? n_all
                                : std::min<u64>(n_all, n_all / shards +
                                                           8 * (u64)std::sqrt((double)n_all) + 4096);

  PhaseTrace trace(st);
  trace.mark("start");
  // ---- 1. unique keys ----
  Buf keys(ctx);
  u64 n = 0;
  {
    // +1: the all-ones key is kept out of the hash set and appended last
    int s = keys.alloc((n_raw + 1) * sizeof(u64));
    if (s) return s;
    // Hash set sized for load <= 1/2 per partition; partitions by the top bits
    // of mix64(key) bound the table when HBM is short.
    release_run_batch(ctx);   // a table needs the room more than s615_run's kept buffers
    size_t free_b = 0, total_b = 0;
    S615_CU(cudaMemGetInfo(&free_b, &total_b));
    size_t avail = std::min(free_b, budget_room(ctx));
    if (avail > ((size_t)2 << 30)) avail -= (size_t)2 << 30;
    u32 part_bits = 0;
    u64 tsize = pow2_at_least(std::max<u64>(2 * n_raw, 1024));
    while (tsize * sizeof(u64) > avail && part_bits < 8) {
      ++part_bits;
      tsize = pow2_at_least(std::max<u64>((2 * n_raw >> part_bits) + (n_raw >> (part_bits + 3)) + 1024, 1024));
    }
    Buf table(ctx), scratch(ctx);
    s = table.alloc(tsize * sizeof(u64));
    if (s) return s;
    s = scratch.alloc(64);
    if (s) return s;
    u32* d_flag = static_cast<u32*>(scratch.p);
    unsigned long long* d_n = reinterpret_cast<unsigned long long*>(static_cast<char*>(scratch.p) + 8);
    S615_CU(cudaMemsetAsync(scratch.p, 0, 64, st));
    for (u32 part = 0; part < (1u << part_bits); ++part) {
      S615_CU(cudaMemsetAsync(table.p, 0xFF, tsize * sizeof(u64), st));
      const KeyFilter kf{part_bits, part, shards, shard, mod_recip(shards)};
      if (pairs) {
        const int grid = (int)std::min<u64>(n_vals ? n_vals : 1, (u64)ctx->num_sms * 32);
        k_insert_pairs<<<grid, 256, 0, st>>>(d_pair_vals, n_vals,
                                             static_cast<unsigned long long*>(table.p), tsize - 1,
                                             kf, d_flag);
      } else {
        k_insert_keys<<<grid_for(ctx, n_keys, 256), 256, 0, st>>>(
            d_keys, n_keys, static_cast<unsigned long long*>(table.p), tsize - 1, kf, d_flag);
      }
      ctx->launches++;
      S615_CU(cudaGetLastError());
      k_compact<<<grid_for(ctx, tsize, 256), 256, 0, st>>>(
          static_cast<const unsigned long long*>(table.p), tsize, static_cast<u64*>(keys.p), n_raw,
          d_n);
      ctx->launches++;
      S615_CU(cudaGetLastError());
    }
    u32 h_flag = 0;
    unsigned long long h_n = 0;
    S615_CU(cudaMemcpyAsync(&h_flag, d_flag, 4, cudaMemcpyDeviceToHost, st));
    S615_CU(cudaMemcpyAsync(&h_n, d_n, 8, cudaMemcpyDeviceToHost, st));
    S615_CU(cudaStreamSynchronize(st));
    n = h_n;
    if (n > n_raw) return S615_E_BUILD;   // more keys in this shard than its buffer holds
    if (h_flag) {
      const u64 e = kEmpty;
      S615_CU(cudaMemcpy(static_cast<u64*>(keys.p) + n, &e, 8, cudaMemcpyHostToDevice));
      ++n;
    }
  }

  std::memset(&out->hdr, 0, sizeof out->hdr);
  out->hdr.magic = kMagic; out->hdr.version = kVersion; out->hdr.kind = 1;
  out->hdr.r = (u32)r; out->hdr.N = (u32)(N > 0 ? N : 0);
  out->hdr.shard_count = shards;
  out->hdr.shard_index = shard;
  if (n == 0) {
    out->hdr.mix_seed = seeds[0];
    out->layout = S615_LAYOUT_WIDE; out->cell_bytes = 8;
    out->d_cells = nullptr; out->bytes = 0;
    return S615_OK;
  }

  trace.mark("unique");
  // ---- 2-4. per seed: incidence, peel, fill ----
  const u64 m = capacity_for(n);
  const u64 block = m / 3, recip = mod_recip(block);
  if (n > kMaxKeys) return S615_E_BUILD;   // key indices must stay below 2^34
#ifdef S615_CHECKED
  S615_CU(cudaMemcpyToSymbolAsync(g_check_nkeys, &n, sizeof n, 0, cudaMemcpyHostToDevice, st));
  S615_CU(cudaMemcpyToSymbolAsync(g_check_ncells, &m, sizeof m, 0, cudaMemcpyHostToDevice, st));
#endif
  Buf cells(ctx), rounds(ctx), scratch(ctx), order(ctx), front(ctx);
  int s = cells.alloc(m * sizeof(u64));
  if (s) return s;
  // Peel over lists (claimed cells in round order, two candidate lists of
  // m/8 cells each; a round whose candidates overflow scans every cell), or,
  // without room for the lists, over full scans by round tag.
  // Candidate lists: two of m/8 entries (5 bytes each: offset + third).
  const u64 fcap = std::max<u64>(4096, m / 8);
  bool lists = block < (1ull << 32);
  if (lists && front.alloc(2 * fcap * 5)) {
    front.release();
    lists = false;
  }
  if ((s = scratch.alloc(64))) return s;
  auto* W = static_cast<unsigned long long*>(cells.p);
  const u64* K = static_cast<const u64*>(keys.p);
  // scratch: [0] max count, [4] list overflow, [8] n_order / n_claimed, [16] n_next
  u32* d_max = static_cast<u32*>(scratch.p);
  u32* d_lover = reinterpret_cast<u32*>(static_cast<char*>(scratch.p) + 4);
  auto* d_norder = reinterpret_cast<unsigned long long*>(static_cast<char*>(scratch.p) + 8);
  auto* d_nnext = reinterpret_cast<unsigned long long*>(static_cast<char*>(scratch.p) + 16);
  const int g = grid_for(ctx, m, 256);
  // Entry buffers of the binned incidence: all 3n updates when HBM allows,
  // else chunks of keys; with no room for a useful chunk the incidence adds
  // directly into the cell words (k_incidence).  The peel's own buffers come
  // first: the round tags of the scan form, or (when the entry buffers will
  // not hold 2n entries for the recorded claim list) the claimed-cell list.
  auto avail_now = [&]() -> size_t {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) { cudaGetLastError(); return 0; }
    size_t a = std::min(free_b, budget_room(ctx));
    const size_t margin = (size_t)2 << 30;
    return a > margin ? a - margin : 0;
  };
  const size_t bin_bytes = (size_t)ctx->num_sms * 2 * kMaxSlices * (4 + 8) + 64;
  // the recorded claim list needs 17 bytes per key in the entry buffers
  // (offset, third, u32 index, hash) and n < 2^32; otherwise the claimed
  // cells alone (5 bytes per key) are taken now, before the entry buffers
  const bool rich_possible = n < (1ull << 32);
  if (lists && (!rich_possible || avail_now() < bin_bytes + 24 * n) && order.alloc(n * 5)) {
    order.release(); front.release();
    lists = false;
  }
  if (!lists && (s = rounds.alloc(m * sizeof(u16)))) return s;
  Buf ent(ctx), bins(ctx);   // ent: one 8-byte word per update (index << 32 | slice offset)
  u64 ent_cap = 0;
  {
    const size_t avail = avail_now();
    if (avail > bin_bytes) {
      ent_cap = std::min<u64>(3 * n, (avail - bin_bytes) / 8);
      ent_cap = ent_cap / 3 * 3;
    }
    if (ent_cap >= std::min<u64>(3 * n, 3ull << 20)) {
      if ((s = ent.alloc(ent_cap * 8)) || (s = bins.alloc(bin_bytes))) {
        ent.release(); bins.release();
        ent_cap = 0;
      }
    } else {
      ent_cap = 0;
    }
  }
  // The claim list: in the entry buffer (idle after the incidence) with each
  // key's index and hash when it has room, else cells only.  Its layout:
  // offsets (4n bytes), indices (4n), thirds (n), then the hashes (8n) from
  // the next 8-byte boundary.
  ClaimList claim_list{{nullptr, nullptr}, nullptr, nullptr};
  const u64 hash_at = (9 * n + 7) / 8 * 8;
  if (lists && rich_possible && ent_cap * 8 >= hash_at + 8 * n && !order.p) {
    u32* o = static_cast<u32*>(ent.p);
    claim_list = ClaimList{{o, reinterpret_cast<u8*>(o + 2 * n)}, o + n,
                           reinterpret_cast<unsigned long long*>(static_cast<char*>(ent.p) + hash_at)};
  } else if (lists && (order.p || !order.alloc(n * 5))) {
    u32* o = static_cast<u32*>(order.p);
    claim_list.cells = CellList{o, reinterpret_cast<u8*>(o + n)};
  } else if (lists) {   // no room for any list: scan, with round tags in the entry buffers' place
    order.release(); front.release();
    ent.release(); bins.release();
    ent_cap = 0;
    lists = false;
    if ((s = rounds.alloc(m * sizeof(u16)))) return s;
  }
  bool built = false;
  u64 used_seed = 0;
  int trace_rounds = 0;
  for (int si = 0; si < n_seeds && !built; ++si) {
    const u64 seed = seeds[si];
    S615_CU(cudaMemsetAsync(W, 0, m * sizeof(u64), st));
    if (!lists) S615_CU(cudaMemsetAsync(rounds.p, 0, m * sizeof(u16), st));
    S615_CU(cudaMemsetAsync(scratch.p, 0, 64, st));
    if (ent_cap) {
      const size_t G = (size_t)ctx->num_sms * 2;
      u32* bhist = static_cast<u32*>(bins.p);
      auto* bbase = reinterpret_cast<unsigned long long*>(static_cast<char*>(bins.p) +
                                                          (G * kMaxSlices * 4 + 7) / 8 * 8);
      if ((s = incidence_binned(ctx, K, n, seed, m, block, recip,
                                static_cast<unsigned long long*>(ent.p), ent_cap, W, bhist, bbase,
                                st)))
        return s;
    } else {
      k_incidence<<<grid_for(ctx, n, 256), 256, 0, st>>>(K, n, seed, block, recip, W);
      ctx->launches++;
      S615_CU(cudaGetLastError());
    }
    k_max_count<<<g, 256, 0, st>>>(W, m, d_max);
    ctx->launches++;
    u32 mx = 0;
    S615_CU(cudaMemcpyAsync(&mx, d_max, 4, cudaMemcpyDeviceToHost, st));
    S615_CU(cudaStreamSynchronize(st));
    if (mx > 255) return S615_E_BUILD;   // the index sums could reach the count bits
    trace.mark("incidence");
    const u64 mask = fp_mask((u32)r);
    if (lists) {

      u32* fo = static_cast<u32*>(front.p);
      u8* ft = reinterpret_cast<u8*>(fo + 2 * fcap);
      const CellList fr[2] = {CellList{fo, ft}, CellList{fo + fcap, ft + fcap}};
      std::vector<u64> off{0};
      u64 total = 0, ncand = m;
      CellList cand{nullptr, nullptr};   // round 1 scans every cell
      int cur = 0;
      // S615_TRACE: per round, the candidates, the keys claimed and the host
      // time of its claim and apply (each ends in a sync here anyway)
      using TClock = std::chrono::steady_clock;
      const auto ms_since = [](TClock::time_point a) {
        return std::chrono::duration<double, std::milli>(TClock::now() - a).count();
      };
      std::vector<std::array<double, 4>> rounds_trace;
      while (off.size() <= 0xFFFE) {
        const auto t_claim = TClock::now();
        k_claim_list<<<grid_for(ctx, ncand, 256), 256, 0, st>>>(cand, ncand, W, K, seed, block,
                                                                recip, claim_list, d_norder, n,
                                                                d_lover);
        ctx->launches++;
        unsigned long long h_n[2] = {0, 0};
        u32 h_lover = 0;
        S615_CU(cudaMemcpyAsync(&h_n[0], d_norder, 8, cudaMemcpyDeviceToHost, st));
        S615_CU(cudaStreamSynchronize(st));
        const u64 L = h_n[0] - total;
        const double claim_ms = trace.on ? ms_since(t_claim) : 0.0;
        const auto t_apply = TClock::now();
        if (L == 0) break;
        S615_CU(cudaMemsetAsync(d_nnext, 0, 8, st));
        S615_CU(cudaMemsetAsync(d_lover, 0, 4, st));
        k_apply_list<<<grid_for(ctx, (L + kApplyPer - 1) / kApplyPer, 256), 256, 0, st>>>(
            claim_list.at(total), L, W, K, seed,
                                                            block, recip,
                                                            fr[cur ^ 1], d_nnext, fcap, d_lover);
        ctx->launches++;
        S615_CU(cudaGetLastError());
        S615_CU(cudaMemcpyAsync(&h_n[1], d_nnext, 8, cudaMemcpyDeviceToHost, st));
        S615_CU(cudaMemcpyAsync(&h_lover, d_lover, 4, cudaMemcpyDeviceToHost, st));
        S615_CU(cudaStreamSynchronize(st));
        if (trace.on) rounds_trace.push_back({(double)ncand, (double)L, claim_ms, ms_since(t_apply)});
        total += L;
        off.push_back(total);
        cur ^= 1;
        if (h_lover) {   // candidates overflowed: the next round scans every cell
          cand = CellList{nullptr, nullptr};
          ncand = m;
          S615_CU(cudaMemsetAsync(d_lover, 0, 4, st));
        } else {
          cand = fr[cur];
          ncand = h_n[1];
          if (ncand == 0) break;   // nothing became count 1: the peel is over
        }
      }
      if (trace.on)
        for (size_t q = 0; q < rounds_trace.size(); ++q)
          std::fprintf(stderr, "[xor-build] round %zu: candidates=%.0f claimed=%.0f claim=%.2fms apply=%.2fms\n",
                       q + 1, rounds_trace[q][0], rounds_trace[q][1], rounds_trace[q][2],
                       rounds_trace[q][3]);
      if (total != n) continue;   // 2-core not empty: next seed
      trace.mark("peel");
      for (size_t q = off.size() - 1; q >= 1; --q) {
        const u64 L = off[q] - off[q - 1];
        k_fill_list<<<grid_for(ctx, L, 256), 256, 0, st>>>(claim_list.at(off[q - 1]), L, W, K,
                                                           seed, block, recip, mask);
        ctx->launches++;
      }
      trace_rounds = (int)off.size() - 1;
    } else {
      u16* rt = static_cast<u16*>(rounds.p);
      u64 peeled = 0;
      u16 rr = 0;
      for (;;) {
        if (rr == 0xFFFE) break;
        ++rr;
        S615_CU(cudaMemsetAsync(d_norder, 0, 8, st));
        k_claim_scan<<<g, 256, 0, st>>>(W, K, seed, rt, m, block, recip, rr, d_norder);
        ctx->launches++;
        k_apply_scan<<<g, 256, 0, st>>>(W, K, seed, rt, m, block, recip, rr);
        ctx->launches++;
        S615_CU(cudaGetLastError());
        unsigned long long c = 0;
        S615_CU(cudaMemcpyAsync(&c, d_norder, 8, cudaMemcpyDeviceToHost, st));
        S615_CU(cudaStreamSynchronize(st));
        if (c == 0) { --rr; break; }
        peeled += c;
      }
      if (peeled != n) continue;   // 2-core not empty: next seed
      trace.mark("peel");
      for (u16 q = rr; q >= 1; --q) {
        k_fill_scan<<<g, 256, 0, st>>>(W, K, seed, rt, m, block, recip, q, mask);
        ctx->launches++;
      }
      trace_rounds = rr;
    }
    S615_CU(cudaGetLastError());
    trace.mark("fill");
    built = true;
    used_seed = seed;
  }
  if (!built) return S615_E_BUILD;
  S615_CU(cudaStreamSynchronize(st));
  trace.mark("sync");
  keys.release(); rounds.release(); order.release(); front.release();
  trace.mark("free_keys");
  ent.release(); bins.release();
  trace.mark("free_bins");

  out->hdr.n_keys = n;
  out->hdr.m_cells = m;
  out->hdr.mix_seed = used_seed;
  // ---- 5. final HBM layout ----
  if (layout == S615_LAYOUT_PACKED) {
    const u64 len = packed_bytes(m, (u32)r);
    const size_t bytes = ((len + 7) / 8 + 1) * 8;
    void* p = nullptr;
    if ((s = dev_alloc(ctx, &p, bytes))) return s;
    S615_CU(cudaMemsetAsync(p, 0, bytes, st));
    if ((s = launch_pack(ctx, cells.p, 8, m, (u32)r, static_cast<u8*>(p), len, st))) {
      dev_free(ctx, p, bytes);
      return s;
    }
    out->layout = S615_LAYOUT_PACKED; out->cell_bytes = 0;
    out->d_cells = p; out->bytes = bytes;
  } else if (r <= 32) {
    void* p = nullptr;
    const size_t bytes = m * sizeof(u32);
    if ((s = dev_alloc(ctx, &p, bytes))) return s;
    k_narrow<<<g, 256, 0, st>>>(static_cast<const u64*>(cells.p), static_cast<u32*>(p), m);
    ctx->launches++;
    out->layout = S615_LAYOUT_WIDE; out->cell_bytes = 4;
    out->d_cells = p; out->bytes = bytes;
  } else {
    out->layout = S615_LAYOUT_WIDE; out->cell_bytes = 8;
    out->d_cells = cells.p; out->bytes = cells.n;
    cells.p = nullptr; cells.n = 0;   // ownership moves to the table
  }
  trace.mark("layout");
  trace.report(n, m, trace_rounds);
  S615_CU(cudaStreamSynchronize(st));
  S615_CU(cudaGetLastError());
  return S615_OK;
}

S615_CHECK_TAKE_DEFINE(check_take_xor_build)

}  // namespace s615
