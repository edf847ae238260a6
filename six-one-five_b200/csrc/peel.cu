// peel.cu -- the free peels of classes 2-5: exact row set-up, the residue
// gate as a sieve, compaction and the xor probe, in one persistent kernel.
//
// Class 5 replaces k_cls5_192 (fourcore_cls5_gpu_v4.cu:353-410); classes 2-4
// replace the find3 leaf (expand_unit + make_cand mode 3 + k_find3,
// fourcore_find_v4.cu:165-205,401-425,255-284).  Both give the reference's
// raw hits and calls/gated/probes counters.
//
//  * Exact rows, no per-point big integers.
//      cls5 row e:   V(e) = (base - (14e)^6) / 21^6 (exact, < 2^126 for B <= 40M);
//                    at column d, T = (V - d^6) / 64, and R > 0 <=> d <= D(e)
//                    with D(e) = iroot6(V - 1).
//      cls2-4 row d: T(d) = (base - (f d)^6) / 42^6 (exact, < 2^122); the
//                    column c3 runs over [lo, hi] with 3 lo^6 >= T and
//                    hi = min(iroot6(T), lim); the point value is T - c3^6.
//    Row values come from base mod 2^128 and the 2-adic inverse of 21^6.
//  * The gate as a sieve.  The reference keeps a value iff it is a sum of
//    two sixth powers mod 504 and mod 247.  Those sets are products over
//    8, 9, 7, 13, 19, and along a row each factor is periodic in the column,
//    so a lane evaluates 32 consecutive columns at once: one row constant for
//    mod 8 AND four 32-bit pattern words from shared memory.
//  * Compaction: gate survivors go to a per-warp ring; each full batch of 32
//    is probed by all lanes together (three L2-only cell loads per lane).
//  * Warps are independent workers pulling (unit, residue, 64-row chunk)
//    items from one device-wide queue; nothing waits at a block barrier.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <type_traits>

#include "peel_common.cuh"

namespace s615 {

namespace {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr u32 kRows = kItemRows;  // rows per item (64)
constexpr u32 kMaxD = 4;          // cls5 d residues per pass
constexpr u32 kQ = 64;            // warp ring capacity (power of two)
constexpr u32 kNoRow = 0xFFFFFFFFu;
constexpr u32 kLenMask = 0x0FFFFFFFu;

struct WarpSmem {                 // one warp's private slice
  RowRec rows[kRows];
  u16 K[kMaxD][kRows];            // cls5: in-row d limit per d residue
  u8 M4[kMaxD][kRows];            // cls5: mod-8 admissibility of k mod 4
  u32 ring[kQ];
  u32 d0s[kMaxD];                 // cls5: d residues of the current pass
  u32 part, nparts;               // class 2-4 items: this item's share of the window tiles
};

// With the sharp gate a cls5 row also carries the offsets for 31, 37, 43 and
// a 32-column mod-64 mask per d residue (T mod 64 has period 32 in k).
struct WarpSmemSharp : WarpSmem {
  u16 offx[kRows][4];
  u32 M32[kMaxD][kRows];
};
template <bool kSharp>
using WarpT = typename std::conditional<kSharp, WarpSmemSharp, WarpSmem>::type;

struct PeelParams {
  TableView tv;
  const DevUnit* units;
  const u64* items;
  u32 n_items;
  u32 n_units;             // unit records (bound of every item's unit index)
  u32* work;
  s615_hit* hits;
  u32 hit_cap;
  Cls5Counters* ctr;
  const u32* pat5;         // cls5 column patterns (step 64, scale 64)
  const u32* pat3;         // find3 column patterns (step 1, scale 1)
  const u32* pat3s;        // sharp gate: find3 column patterns in HBM (read through L1)
  u64 inv21_lo, inv21_hi;  // (21^6)^-1 mod 2^128
  u32 s8;                  // admissible values mod 8, as a bitmask
  u64 p64;                 // sharp gate: admissible values mod 64, as a bitmask
  u32 count;               // add this launch's counters (0 for a repeat pass over a set)
  u32 item_rows;           // rows per item of the batch (<= kRows)
  u32 parts3_log2;         // log2 of the items per class 2-4 row chunk (1 or 4 items)
};

// cls5 pattern words (sharp or not) then the find3 ones, then the warp slices
// (which start on a 16-byte boundary: the row records are 16-byte aligned).
template <bool kSharp>
constexpr size_t smem_pat() {
  return ((size_t)((kSharp ? kSharpWords : kPatWords) + kPatWords) * sizeof(u32) + 15) / 16 * 16;
}
template <bool kSharp>
constexpr size_t smem_total() { return smem_pat<kSharp>() + kWarps * sizeof(WarpT<kSharp>); }

// x^6 mod 512 for small x.
__device__ __forceinline__ u32 pow6_mod512(u32 x) {
  x &= 511;
  const u32 x2 = (x * x) & 511;
  const u32 x3 = (x2 * x) & 511;
  return (x3 * x3) & 511;
}

// Ring entry: column k (18 bits) | row (6 bits) << 18 | pass slot (2 bits) << 24.
__device__ __forceinline__ u32 entry(u32 di, u32 r, u32 k) { return (di << 24) | (r << 18) | k; }

struct ItemCtx {
  u32 cls, unit_id, r0, mod, j0, f;   // job items: unit_id = index of the first unit
};

// Probe the ring entries [head, head+cnt) (one per lane).
template <bool kSet>
__device__ __forceinline__ void probe_batch(const PeelParams& P, const WarpSmem& W, u32 head,
                                            u32 cnt, const ItemCtx& I, u32 lane) {
  if (lane >= cnt) return;
  const u32 ent = W.ring[(head + lane) & (kQ - 1)];
  const u32 k = ent & 0x3FFFFu, r = (ent >> 18) & 63u, di = ent >> 24;
  const RowRec& R = W.rows[r];
  const u128 Wv = ((u128)R.whi << 64) | R.wlo;
  u64 key, x;
  u32 rowval;
  if (I.cls == 5) {
    x = (u64)W.d0s[di] + 64ull * k;                 // d
    key = (u64)((Wv - pow6_small(x)) >> 6);         // T = (V - d^6)/64
    rowval = I.r0 + I.mod * (I.j0 + r);             // e
  } else {
    x = (u64)R.a + k;                               // c3
    key = R.wlo - (u64)pow6_small(x);               // T - c3^6 mod 2^64
    rowval = I.r0 + I.mod * (I.j0 + r);             // d
  }
  if (probe_table<kSet>(P.tv, key)) {
    const unsigned long long idx = atomicAdd(&P.ctr->hits, 1ull);
    if (idx < P.hit_cap) {
      s615_hit h;
      h.unit = I.unit_id; h.a = 0; h.b = 0; h.c4 = 0;
      if (I.cls == 5) { h.d = (u32)x; h.e = rowval; }
      else { h.d = rowval; h.e = (u32)x; }
      if (I.cls == kClsJobRow) {   // row r is unit unit_id + r (hits are rare: one load)
        if (!S615_CHECK(I.unit_id + r < P.n_units, kChkHit)) return;
        h.unit = P.units[I.unit_id + r].id;
        h.d = 0;
      }
      h.fp = key;
      P.hits[idx] = h;
    }
  }
}

// Push the set bits of m into the ring; probe every full batch of 32.
template <bool kSet>
__device__ __forceinline__ void push_bits(const PeelParams& P, WarpSmem& W, u32 m, u32 di, u32 r,
                                          u32 kbase, u32& head, u32& qlen, const ItemCtx& I,
                                          u32 lane) {
  while (__any_sync(0xFFFFFFFFu, m != 0)) {
    const bool has = m != 0;
    const u32 bit = has ? (u32)(__ffs(m) - 1) : 0u;
    m &= m - 1u;
    const u32 ballot = __ballot_sync(0xFFFFFFFFu, has);
    if (has) W.ring[(head + qlen + __popc(ballot & lanemask_lt())) & (kQ - 1)] = entry(di, r, kbase + bit);
    qlen += __popc(ballot);
    if (qlen >= 32u) {
      __syncwarp();
      probe_batch<kSet>(P, W, head, 32u, I, lane);
      __syncwarp();
      head = (head + 32u) & (kQ - 1);
      qlen -= 32u;
    }
  }
}

template <bool kSharp, bool kSet>
__global__ void __launch_bounds__(kThreads, kSharp ? 3 : 5) k_peel(PeelParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr u32 kP5 = kSharp ? (u32)kSharpWords : (u32)kPatWords;
  u32* s_pat5 = reinterpret_cast<u32*>(smem);
  u32* s_pat3 = s_pat5 + kP5;
  const u32 tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  WarpT<kSharp>& W = reinterpret_cast<WarpT<kSharp>*>(smem + smem_pat<kSharp>())[warp];
  for (u32 i = tid; i < kP5; i += kThreads) s_pat5[i] = P.pat5[i];
  for (u32 i = tid; i < (u32)kPatWords; i += kThreads) s_pat3[i] = P.pat3[i];
  __syncthreads();   // the only block barrier: pattern tables are shared

  const u128 inv21 = ((u128)P.inv21_hi << 64) | P.inv21_lo;
  u64 my_calls = 0, my_pos = 0, my_probes = 0;

  for (;;) {
    u32 it = 0;
    if (lane == 0) it = atomicAdd(P.work, 1u);
    it = __shfl_sync(0xFFFFFFFFu, it, 0);
    if (it >= P.n_items) break;
    const u64 packed = P.items[it];
    if (!S615_CHECK(item_unit(packed) < P.n_units, kChkItem)) continue;   // warp-uniform
    const DevUnit* U = P.units + item_unit(packed);
    ItemCtx I;
    I.cls = U->cls;
    I.unit_id = I.cls == kClsJobRow ? item_unit(packed) : U->id;
    I.f = U->f;
    u32 nrows;
    if (I.cls == kClsJobRow) {   // job_count consecutive one-row units; row r is unit u0 + r
      I.r0 = 0;
      I.mod = 1;
      I.j0 = 0;
      nrows = job_count(packed);
      if (!S615_CHECK(item_unit(packed) + nrows <= P.n_units, kChkItem)) continue;
    } else {
      if (!S615_CHECK(item_res(packed) < U->nres1 && U->nres1 <= 24, kChkItem)) continue;
      I.r0 = U->res1[item_res(packed)];
      I.mod = U->mod1;
      u32 jmin, jend;
      class_rows(I.r0, I.mod, U->fmax1, &jmin, &jend);
      u32 ch = item_chunk(packed);
      if (I.cls != 5) {   // kept in the warp's slice: the find3 loop reads them there
        if (lane == 0) { W.part = ch & ((1u << P.parts3_log2) - 1u); W.nparts = 1u << P.parts3_log2; }
        ch >>= P.parts3_log2;
      }
      I.j0 = jmin + ch * P.item_rows;
      nrows = min(P.item_rows, jend - I.j0);
    }
    if (I.cls == kClsJobRow && lane == 0) { W.part = 0; W.nparts = 1; }
    u32 head = 0, qlen = 0;
    __syncwarp();

    if (I.cls == 5) {
      // ---- cls5 rows: V, D and the residues of V (two rows per lane) ----
      const u128 base = ((u128)U->base_hi << 64) | U->base_lo;
      for (u32 r = lane; r < nrows; r += 32) {
        const u64 x = 14ull * ((u64)I.r0 + (u64)I.mod * (I.j0 + r));
        const u128 x3 = (u128)(x * x) * x;           // (14e)^3 < 2^78
        const u128 V = (base - x3 * x3) * inv21;    // exact mod 2^128
        RowRec R;
        R.wlo = (u64)V; R.whi = (u64)(V >> 64);
        if ((R.whi >> 63) || V == 0) {
          R.a = 0; R.b = kNoRow;
          R.off[0] = R.off[1] = R.off[2] = R.off[3] = 0;
        } else {
          R.a = iroot6_u128(V - 1);
          R.b = (u32)(R.wlo & 511u);
          if constexpr (kSharp) set_offsets_sharp(R, W.offx[r]);
          else set_offsets(R);
        }
        W.rows[r] = R;
      }
      const u32 fmax2 = U->fmax2, nres2 = U->nres2;
      for (u32 dg = 0; dg < nres2; dg += kMaxD) {
        const u32 nd = min(kMaxD, nres2 - dg);
        __syncwarp();
        if (lane < kMaxD) W.d0s[lane] = lane < nd ? U->res2[dg + lane] : 0u;
        __syncwarp();
        // per (row, d residue): in-row limit and the mod-8 row mask
        u32 kmax = 0;
        for (u32 idx = lane; idx < nd * nrows; idx += 32) {   // the item's rows only
          const u32 di = idx / nrows, r = idx - di * nrows;
          const u32 d0 = W.d0s[di];
          const RowRec& R = W.rows[r];
          const u32 kcap = (d0 <= fmax2) ? (fmax2 - d0) / 64u + 1u : 0u;
          const u32 kpos = (R.b != kNoRow && R.a >= d0) ? (R.a - d0) / 64u + 1u : 0u;
          const u32 kend = min(kcap, kpos);
          const u32 kmin = (d0 == 0) ? 1u : 0u;
          if (kend > kmin) my_pos += kend - kmin;
          if (r == 0) my_calls += (u64)nrows * (kcap > kmin ? kcap - kmin : 0u);
          kmax = max(kmax, kend);
          if constexpr (kSharp) {
            // T = (V - d^6)/64 mod 64 from (V - d^6) mod 4096, d = d0 + 64 i
            u32 m32 = 0;
            if (R.b != kNoRow) {
              const u32 v12 = (u32)R.wlo & 4095u;
              for (u32 i = 0; i < 32; ++i) {
                const u32 t = ((v12 - pow6_mod4096(d0 + 64u * i)) & 4095u) >> 6;
                m32 |= (u32)((P.p64 >> t) & 1ull) << i;
              }
            }
            W.M32[di][r] = m32;
          } else {
            u32 m4 = 0;
            if (R.b != kNoRow) {
#pragma unroll
              for (u32 i = 0; i < 4; ++i) {
                const u32 t8 = ((R.b - pow6_mod512(d0 + 64u * i)) & 511u) >> 6;
                m4 |= ((P.s8 >> t8) & 1u) << i;
              }
            }
            W.M4[di][r] = (u8)m4;
          }
          W.K[di][r] = (u16)kend;
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) kmax = max(kmax, __shfl_xor_sync(0xFFFFFFFFu, kmax, o));
        __syncwarp();
        const u32 ntiles = (kmax + 1023u) / 1024u;
        for (u32 di = 0; di < nd; ++di) {
          const u32 d0 = W.d0s[di];
          const u32 lowmask0 = (d0 == 0) ? ~1u : ~0u;
          for (u32 wt = 0; wt < ntiles; ++wt) {
            const u32 kbase = (wt * 32u + lane) * 32u;
            const u64 dstart = (u64)d0 + 64ull * kbase;
            const u32 s9 = (u32)(dstart % (kSharp ? 27 : 9)), s7 = (u32)(dstart % (kSharp ? 49 : 7));
            const u32 s13 = (u32)(dstart % 13), s19 = (u32)(dstart % 19);
            u32 s31 = 0, s37 = 0, s43 = 0;
            if constexpr (kSharp) {
              s31 = (u32)(dstart % 31); s37 = (u32)(dstart % 37); s43 = (u32)(dstart % 43);
            }
            const u32 lowmask = (kbase == 0) ? lowmask0 : ~0u;
            for (u32 r = 0; r < nrows; ++r) {
              const u32 kend = W.K[di][r];
              if (kend <= wt * 1024u) break;          // rows shorten as e grows
              u32 m = 0;
              if (kbase < kend) {
                if constexpr (kSharp)
                  m = W.M32[di][r] & gate_word(s_pat5, W.rows[r], s9, s7, s13, s19) &
                      gate_word3(s_pat5, W.offx[r], s31, s37, s43);
                else
                  m = ((u32)W.M4[di][r] * 0x11111111u) & gate_word(s_pat5, W.rows[r], s9, s7, s13, s19);
                const u32 n = kend - kbase;
                if (n < 32u) m &= (1u << n) - 1u;
                m &= lowmask;
              }
              my_probes += __popc(m);
              push_bits<kSet>(P, W, m, di, r, kbase, head, qlen, I, lane);
            }
          }
        }
        __syncwarp();
        probe_batch<kSet>(P, W, head, qlen, I, lane);   // drain before d0s change
        head = 0;
        qlen = 0;
        __syncwarp();
      }
    } else {
      // ---- cls2-4 rows: T(d) and its find3 window [lo, hi]; job rows: T given ----
      const bool job = I.cls == kClsJobRow;
      const bool find2 = job && U->w != 0;
      for (u32 r = lane; r < nrows; r += 32) {
        const DevUnit* Ur = job ? U + r : U;   // a job item's row r is its own unit
        const u64 x = (u64)I.f * ((u64)I.r0 + (u64)I.mod * (I.j0 + r));
        const u128 x3 = (u128)(x * x) * x;
        const u128 Rm = (((u128)Ur->base_hi << 64) | Ur->base_lo) - x3 * x3;
        const u128 T = ((Rm >> 6) * inv21) & ((~(u128)0) >> 6);  // T mod 2^122
        const u32 rlim = Ur->lim;
        RowRec R;
        R.wlo = (u64)T; R.whi = (u64)(T >> 64);
        R.a = 0; R.b = 0;
        R.off[0] = R.off[1] = R.off[2] = R.off[3] = 0;
        if (T != 0 && (T >> 121) == 0) {
          const u32 hi = find2 ? 1u : min(iroot6_u128(T), rlim);
          const u128 third = T / 3 + ((T % 3) ? 1 : 0);         // ceil(T/3) >= 1
          const u32 lo = find2 ? 1u : iroot6_u128(third - 1) + 1;  // least c with 3 c^6 >= T
          if (lo <= hi) {
            const u32 len = hi - lo + 1;
            u32 m4 = 0;
#pragma unroll
            for (u32 i = 0; i < 4; ++i) {
              const u32 odd = (lo + i) & 1u;                    // c^6 mod 8 = c odd ? 1 : 0
              const u32 t8 = ((u32)R.wlo - odd) & 7u;
              m4 |= ((P.s8 >> t8) & 1u) << i;
            }
            R.a = lo;
            R.b = len | (m4 << 28);
            if constexpr (kSharp) {   // q = 27, 49, 13, 19, 31, 37, 43 and T - c^6 mod 64
              set_offsets_sharp(R, W.offx[r]);
              u32 m32 = 0;
              for (u32 i = 0; i < 32; ++i) {
                const u32 t = ((u32)R.wlo - pow6_mod4096(lo + i)) & 63u;
                m32 |= (u32)((P.p64 >> t) & 1ull) << i;
              }
              W.M32[0][r] = m32;
            } else {
              set_offsets(R);
            }
            if (W.part == 0) {   // a row's window is counted once
              my_calls += len;
              my_pos += len;
            }
          }
        }
        W.rows[r] = R;
      }
      __syncwarp();
      // Sieve steps: a row's window in tiles of 1024 columns (lane = 32
      // columns), or for find2 items 32 one-column rows at once (lane = row).
      u32 r = 0, wt = W.part;
      while (r < nrows) {
        const u32 rr = find2 ? r + lane : r;
        const u32 kbase = find2 ? 0u : (wt * 32u + lane) * 32u;
        u32 m = 0, len = 0;
        if (rr < nrows) {
          const RowRec& R = W.rows[rr];
          len = R.b & kLenMask;
          if (kbase < len) {
            const u32 xs = R.a + kbase;
            if constexpr (kSharp)   // T - c^6 mod 64 has period 32 in c: one mask per row
              m = W.M32[0][rr] & gate_word(P.pat3s, R, xs % 27, xs % 49, xs % 13, xs % 19) &
                  gate_word3(P.pat3s, W.offx[rr], xs % 31, xs % 37, xs % 43);
            else
              m = ((R.b >> 28) * 0x11111111u) & gate_word(s_pat3, R, xs % 9, xs % 7, xs % 13, xs % 19);
            const u32 n = len - kbase;
            if (n < 32u) m &= (1u << n) - 1u;
          }
        }
        my_probes += __popc(m);
        push_bits<kSet>(P, W, m, 0, rr & 63u, kbase, head, qlen, I, lane);
        if (find2) {
          r += 32;
        } else if ((wt += W.nparts) >= (len + 1023u) / 1024u) {   // len: the same in every lane
          wt = W.part;
          ++r;
        }
      }
      __syncwarp();
      probe_batch<kSet>(P, W, head, qlen, I, lane);
      __syncwarp();
    }
  }

  // ---- counters: warp reduce, one atomic per warp ----
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    my_calls += __shfl_xor_sync(0xFFFFFFFFu, my_calls, o);
    my_pos += __shfl_xor_sync(0xFFFFFFFFu, my_pos, o);
    my_probes += __shfl_xor_sync(0xFFFFFFFFu, my_probes, o);
  }
  if (lane == 0 && P.count) {
    atomicAdd(&P.ctr->calls, (unsigned long long)my_calls);
    atomicAdd(&P.ctr->pos, (unsigned long long)my_pos);
    atomicAdd(&P.ctr->probes, (unsigned long long)my_probes);
  }
}

// k_peel over items [0, n) of the batch.
template <bool kSharp, bool kSet>
int launch_main(s615_ctx* ctx, const TableView& tv, const s615_batch* b, size_t n,
                unsigned flags, cudaStream_t st, int grid_blocks) {
  // the shared-memory attribute belongs to each device's context: one bit per device
  static std::atomic<unsigned long long> attr_set{0};
  constexpr size_t kSmemTotal = smem_total<kSharp>();
  const unsigned long long dev_bit = 1ull << (ctx->device & 63);
  if (!(attr_set.load() & dev_bit)) {
    S615_CU(cudaFuncSetAttribute(k_peel<kSharp, kSet>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSmemTotal));
    attr_set.fetch_or(dev_bit);
  }
  PeelParams P{};
  P.tv = tv;
  P.units = b->d_units;
  P.items = b->d_items;
  P.n_items = (u32)n;
  P.n_units = (u32)b->n_units;
  P.work = b->d_work;
  P.hits = b->d_hits;
  P.hit_cap = b->hit_cap;
  P.ctr = b->d_ctr;
  const bool gated = !(flags & S615_F_NO_GATE);
  // ctx->d_pat = [gate cls5 | open cls5 | gate find3 | open find3]
  P.pat5 = kSharp ? ctx->d_sharp : ctx->d_pat + (gated ? 0 : kPatWords);
  P.p64 = ctx->p64;
  P.count = (flags & kFlagNoCount) ? 0u : 1u;
  P.item_rows = b->item_rows ? std::min(b->item_rows, kRows) : kRows;
  P.parts3_log2 = b->parts3 >= 4 ? 2u : b->parts3 >= 2 ? 1u : 0u;
  P.pat3 = ctx->d_pat + 2 * kPatWords + (gated ? 0 : kPatWords);
  P.pat3s = ctx->d_sharp + kSharpWords;
  const u128 inv = inv_2adic_u128((u128)kM21);
  P.inv21_lo = (u64)inv;
  P.inv21_hi = (u64)(inv >> 64);
  P.s8 = gated ? 0x7u : 0xFFu;
  if (n == 0) return S615_OK;
  int grid = grid_blocks;
  if (grid <= 0) {
    int per_sm = 0;
    S615_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_peel<kSharp, kSet>, kThreads, kSmemTotal));
    if (b->blocks_per_sm && (int)b->blocks_per_sm < per_sm) per_sm = (int)b->blocks_per_sm;
    grid = ctx->num_sms * (per_sm > 0 ? per_sm : 1);
  }
  const size_t need = (n + kWarps - 1) / kWarps;
  if ((size_t)grid > need) grid = (int)need;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = kSmemTotal;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  cfg.attrs = attr;
  cfg.numAttrs = (unsigned)l2_window(ctx, tv, flags, attr);
  S615_CU(cudaLaunchKernelEx(&cfg, k_peel<kSharp, kSet>, P));
  ctx->launches++;
  S615_CU(cudaGetLastError());
  return S615_OK;
}

}  // namespace

static int launch_pass(s615_ctx* ctx, const TableView& tv, s615_batch* b, unsigned flags,
                       cudaStream_t st, int grid_blocks) {
  if (b->n_main) {
    const bool sharp = (flags & S615_F_SHARP) && !(flags & S615_F_NO_GATE);
    const bool set = tv.shards > 1;
    const int s =
        set ? (sharp ? launch_main<true, true>(ctx, tv, b, b->n_main, flags, st, grid_blocks)
                     : launch_main<false, true>(ctx, tv, b, b->n_main, flags, st, grid_blocks))
            : (sharp ? launch_main<true, false>(ctx, tv, b, b->n_main, flags, st, grid_blocks)
                     : launch_main<false, false>(ctx, tv, b, b->n_main, flags, st, grid_blocks));
    if (s) return s;
  }
  if (b->n_items > b->n_main) return launch_peel617(ctx, tv, b, flags, st, grid_blocks);
  return S615_OK;
}

// One pass, or for a shard set of G probe groups G passes: pass g probes only
// the keys of its group's shards; passes after the first restart the work
// queues and add no counters, and every pass appends to the same hit list.
int launch_peel(s615_ctx* ctx, const TableView& tv, s615_batch* b, unsigned flags,
                cudaStream_t st, int grid_blocks) {
  const u32 G = tv.shards > 1 ? std::max(1u, tv.groups) : 1u;
  for (u32 g = 0; g < G; ++g) {
    TableView v = tv;
    if (G > 1) {   // the g-th slice of the shards this set holds
      const u64 n = tv.grp_hi - tv.grp_lo;
      v.grp_lo = tv.grp_lo + (u32)(n * g / G);
      v.grp_hi = tv.grp_lo + (u32)(n * (g + 1) / G);
    }
    if (g > 0) S615_CU(cudaMemsetAsync(b->d_work, 0, 8, st));
    const int s = launch_pass(ctx, v, b, g > 0 ? flags | kFlagNoCount : flags, st, grid_blocks);
    if (s) return s;
  }
  return S615_OK;
}

S615_CHECK_TAKE_DEFINE(check_take_peel)

}  // namespace s615
