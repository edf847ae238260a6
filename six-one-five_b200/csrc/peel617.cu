// peel617.cu -- the (6,1,7) Branch-A class-5 search as one persistent kernel.
//
// Replaces k_find4_cls5 (solve_617_v1.cu:563-657), which gpu_run (:924-1006)
// launches with one block per (candidate, d) and c4 tiles of 2048, and gives
// its raw hits and its calls / gated / tri_total / tri_skipped counters.
//
//  * Rows d (the x21 term, one lane each, 8 per work item; items are handed
//    out smallest d first, where T and both windows are largest):
//      T = (base - (21d)^6) / 42^6, exact (< 2^95) from base mod 2^128 and
//      the 2-adic inverse of 21^6; the c4 window [lo4, hi4] with
//      hi4 = min(iroot6(T), lim) and lo4 the least c with 3 c^6 >= T
//      (iroot6_fix / min_c_fix, :416-437, on R = 42^6 T).
//  * c4 step: the warp walks one window 32 c4 at a time; the triple-sum gate
//    (T - c4^6 mod 504 and mod 247 must be a sum of three sixth powers,
//    :530-541) reads its tables from shared memory; survivors queue as
//    (lane of the row, c4).
//  * find3 rows: 32 queued c4 at a time, one per lane: T' = T - c4^6, the c3
//    window [lo3, hi3] with hi3 = min(iroot6(T'), lim, c4) and lo3 the least
//    c with 3 c^6 >= T' (:622-628), the mod-8 mask and pattern offsets of T'.
//    Rows collect in a 64-row buffer per warp.
//  * Sieve: the 32-column chunks of all buffered rows are dealt to the lanes
//    (a prefix over rows and a binary search), so short windows do not idle
//    the warp.  A lane's 32 gate bits are one mod-8 mask AND four pattern
//    words; survivors pass through the per-warp ring to the batched xor
//    probe with key = T' - c3^6 mod 2^64 (funnel_fp - pow6_64, :635-647).
//  * Every c4 is visited once.  The reference's c4 tiles re-walk c4 >=
//    lo4 + 2048 z in block z, which only happens for windows wider than 2048
//    (B above about 514,000); its counters and raw hits then repeat those c4.
#include <cuda_runtime.h>

#include <atomic>
#include <type_traits>

#include "peel_common.cuh"

namespace s615 {

namespace {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr u32 kBuf = 64;            // find3 rows buffered per warp
constexpr u32 kQ = 64;              // probe ring capacity (power of two)
constexpr u32 kCQ = 64;             // c4 queue capacity (power of two)
constexpr u32 kLenMask = 0x0FFFFFFFu;
constexpr u32 kFull = 0xFFFFFFFFu;
constexpr u32 kC4Bits = 21;         // c4 <= lim < 2^21 (B <= 40,000,000)
constexpr u32 kC4Mask = (1u << kC4Bits) - 1u;

struct WarpSmem617 {
  RowRec rows[kBuf];     // W = T', a = lo3, b = len | m4 << 28
  u32 aux[kBuf];         // c4 | (row index in the item) << kC4Bits
  u32 pre[kBuf + 1];     // first 32-column chunk of each buffered row
  u32 cq[kCQ];           // c4 queue: c4 | (lane holding the row) << kC4Bits
  u32 ring[kQ];          // probe ring: column (18 bits) | buffer row << 18
};

// With the sharp gate a row also carries the offsets for 31, 37, 43 and a
// 32-column mod-64 mask (c^6 mod 64 has period 32 in c).
struct WarpSmem617Sharp : WarpSmem617 {
  u16 offx[kBuf][4];
  u32 m32[kBuf];
};
template <bool kSharp>
using Warp617T = typename std::conditional<kSharp, WarpSmem617Sharp, WarpSmem617>::type;

struct Peel617Params {
  TableView tv;
  const DevUnit* units;
  const u64* items;
  u32 n_items;
  u32 n_units;   // unit records (bound of every item's unit index)
  u32* work;
  s615_hit* hits;
  u32 hit_cap;
  Cls5Counters* ctr;
  const u32* pat3;         // find3 column patterns (step 1, scale 1)
  const u32* tri;          // triple-sum gate block
  u64 inv21_lo, inv21_hi;  // (21^6)^-1 mod 2^128
  u32 s8;                  // admissible values mod 8, as a bitmask
  u32 use_tri;
  u64 p64;                 // sharp gate: admissible values mod 64, as a bitmask
  u32 count;               // add this launch's counters (0 for a repeat pass over a set)
};

// Pattern words, the triple-sum block, then the warp slices (16-byte aligned:
// the row records are).
template <bool kSharp>
constexpr size_t smem_pat617() {
  return ((size_t)(kSharp ? kSharpWords : kPatWords) * sizeof(u32) + 15) / 16 * 16;
}
constexpr size_t kSmemTri = kTriWords * sizeof(u32);
static_assert(kSmemTri % 16 == 0, "warp slices must start 16-byte aligned");
template <bool kSharp>
constexpr size_t smem_total617() { return smem_pat617<kSharp>() + kSmemTri + kWarps * sizeof(Warp617T<kSharp>); }

struct Item617 {
  u32 unit_id, r0, mod, j0, lim, cls;
};

// Per-warp state carried through one item.
struct State617 {
  u32 nbuf;        // rows in the buffer
  u32 head, qlen;  // probe ring
  u64 pos, probes;
};

template <bool kSet>
__device__ __forceinline__ void probe_batch(const Peel617Params& P, const WarpSmem617& W,
                                            u32 head, u32 cnt, const Item617& I, u32 lane) {
  if (lane >= cnt) return;
  const u32 ent = W.ring[(head + lane) & (kQ - 1)];
  const u32 k = ent & 0x3FFFFu, r = ent >> 18;
  const RowRec& R = W.rows[r];
  const u32 c3 = R.a + k;
  const u64 c33 = (u64)c3 * c3 * c3;
  const u64 key = R.wlo - c33 * c33;                // T' - c3^6 mod 2^64
  if (probe_table<kSet>(P.tv, key)) {
    const unsigned long long idx = atomicAdd(&P.ctr->hits, 1ull);
    if (idx < P.hit_cap) {
      const u32 aux = W.aux[r];
      s615_hit h;
      h.unit = I.unit_id; h.a = 0; h.b = 0;
      h.d = I.r0 + I.mod * (I.j0 + (aux >> kC4Bits));   // the x21 term (0 for cls 1)
      h.e = c3;
      h.c4 = aux & kC4Mask;
      h.fp = key;
      P.hits[idx] = h;
    }
  }
}

// Sieve every buffered row, probe the survivors, empty the buffer.
template <bool kSharp, bool kSet>
__device__ __forceinline__ void flush_rows(const Peel617Params& P, Warp617T<kSharp>& W,
                                           const u32* s_pat, State617& S, const Item617& I,
                                           u32 lane) {
  const u32 nbuf = S.nbuf;
  if (nbuf == 0) return;
  // chunk prefix over the rows (two rows per lane)
  const u32 n0 = lane < nbuf ? ((W.rows[lane].b & kLenMask) + 31u) >> 5 : 0u;
  const u32 n1 = lane + 32u < nbuf ? ((W.rows[lane + 32u].b & kLenMask) + 31u) >> 5 : 0u;
  u32 s0 = n0, s1 = n1;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const u32 t0 = __shfl_up_sync(kFull, s0, o), t1 = __shfl_up_sync(kFull, s1, o);
    if (lane >= (u32)o) { s0 += t0; s1 += t1; }
  }
  const u32 tot0 = __shfl_sync(kFull, s0, 31);
  const u32 total = tot0 + __shfl_sync(kFull, s1, 31);
  W.pre[lane] = s0 - n0;
  W.pre[lane + 32u] = tot0 + s1 - n1;
  __syncwarp();
  for (u32 g0 = 0; g0 < total; g0 += 32u) {
    const u32 g = g0 + lane;
    u32 m = 0, r = 0, kbase = 0;
    if (g < total) {
      u32 lo = 0, hi = nbuf - 1u;   // the last row starting at or before chunk g
      while (lo < hi) {
        const u32 mid = (lo + hi + 1u) >> 1;
        if (W.pre[mid] <= g) lo = mid; else hi = mid - 1u;
      }
      r = lo;
      const RowRec& R = W.rows[r];
      kbase = (g - W.pre[r]) << 5;
      const u32 len = R.b & kLenMask;
      const u32 xs = R.a + kbase;
      if constexpr (kSharp)
        m = W.m32[r] & gate_word(s_pat, R, xs % 27u, xs % 49u, xs % 13u, xs % 19u) &
            gate_word3(s_pat, W.offx[r], xs % 31u, xs % 37u, xs % 43u);
      else
        m = ((R.b >> 28) * 0x11111111u) & gate_word(s_pat, R, xs % 9u, xs % 7u, xs % 13u, xs % 19u);
      const u32 n = len - kbase;
      if (n < 32u) m &= (1u << n) - 1u;
    }
    S.probes += __popc(m);
    // push the set bits into the ring; probe every full batch of 32
    while (__any_sync(kFull, m != 0)) {
      const bool has = m != 0;
      const u32 bit = has ? (u32)(__ffs(m) - 1) : 0u;
      m &= m - 1u;
      const u32 ballot = __ballot_sync(kFull, has);
      if (has) W.ring[(S.head + S.qlen + __popc(ballot & lanemask_lt())) & (kQ - 1)] = (r << 18) | (kbase + bit);
      S.qlen += __popc(ballot);
      if (S.qlen >= 32u) {
        __syncwarp();
        probe_batch<kSet>(P, W, S.head, 32u, I, lane);
        __syncwarp();
        S.head = (S.head + 32u) & (kQ - 1);
        S.qlen -= 32u;
      }
    }
  }
  __syncwarp();
  probe_batch<kSet>(P, W, S.head, S.qlen, I, lane);   // drain before the rows change
  __syncwarp();
  S.head = 0;
  S.qlen = 0;
  S.nbuf = 0;
}

// Turn cnt queued c4 (from cq[ch]) into find3 rows, one per lane.
template <bool kSharp, bool kSet>
__device__ __forceinline__ void make_rows(const Peel617Params& P, Warp617T<kSharp>& W,
                                          const u32* s_pat, State617& S, const Item617& I,
                                          u32 lane, u32 ch, u32 cnt, u32 h, u64 tl, u64 th) {
  const bool act = lane < cnt;
  const u32 e = W.cq[(ch + lane) & (kCQ - 1)];
  const u32 src = act ? (e >> kC4Bits) & 31u : 0u;
  const u32 c4 = e & kC4Mask;
  const u64 Tl = __shfl_sync(kFull, tl, src), Th = __shfl_sync(kFull, th, src);
  RowRec R;
  u16 offx[4] = {0, 0, 0, 0};
  u32 m32 = 0;
  bool ok = false;
  u32 len = 0;
  if (act) {
    const u128 T = ((u128)Th << 64) | Tl;
    const u128 c6 = pow6_small(c4);
    if (T > c6) {
      const u128 T2 = T - c6;
      const u32 hi3 = min(min(iroot6_u128(T2), I.lim), c4);
      if (hi3 >= 1) {
        // cls 7: least c with 3 c^6 >= T' (min_c_fix); cls 1: (u32)(0.8 hi3), at
        // least 1 (k_find4, fourcore_find_v4.cu:312-314; 0.8 hi3 never lands within
        // 2^-20 of an integer, so the integer form is the same)
        const u32 lo3 = I.cls == 1 ? max(1u, (4u * hi3) / 5u) : least_c_3c6(T2);
        if (lo3 <= hi3) {
          len = hi3 - lo3 + 1u;
          R.wlo = (u64)T2; R.whi = (u64)(T2 >> 64);
          u32 m4 = 0;
#pragma unroll
          for (u32 i = 0; i < 4; ++i) {
            const u32 odd = (lo3 + i) & 1u;                // c^6 mod 8 = c odd ? 1 : 0
            const u32 t8 = ((u32)R.wlo - odd) & 7u;
            m4 |= ((P.s8 >> t8) & 1u) << i;
          }
          R.a = lo3;
          R.b = len | (m4 << 28);
          if constexpr (kSharp) {
            set_offsets_sharp(R, offx);
            for (u32 i = 0; i < 32; ++i) {
              const u32 t = ((u32)R.wlo - pow6_mod4096(lo3 + i)) & 63u;
              m32 |= (u32)((P.p64 >> t) & 1ull) << i;
            }
          } else {
            set_offsets(R);
          }
          ok = true;
        }
      }
    }
  }
  __syncwarp();
  const u32 bal = __ballot_sync(kFull, ok);
  const u32 nnew = __popc(bal);
  if (S.nbuf + nnew > kBuf) flush_rows<kSharp, kSet>(P, W, s_pat, S, I, lane);
  if (ok) {
    const u32 slot = S.nbuf + __popc(bal & lanemask_lt());
    W.rows[slot] = R;
    if constexpr (kSharp) {
      W.m32[slot] = m32;
      for (int k = 0; k < 4; ++k) W.offx[slot][k] = offx[k];
    }
    W.aux[slot] = c4 | ((h + src) << kC4Bits);
    S.pos += len;
  }
  S.nbuf += nnew;
  __syncwarp();
}

template <bool kSharp, bool kSet>
__global__ void __launch_bounds__(kThreads, kSharp ? 3 : 4) k_peel617(Peel617Params P) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr u32 kPW = kSharp ? (u32)kSharpWords : (u32)kPatWords;
  u32* s_pat = reinterpret_cast<u32*>(smem);
  u32* s_tri = s_pat + kPW;
  const u32 tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  Warp617T<kSharp>& W = reinterpret_cast<Warp617T<kSharp>*>(smem + smem_pat617<kSharp>() + kSmemTri)[warp];
  for (u32 i = tid; i < kPW; i += kThreads) s_pat[i] = P.pat3[i];
  for (u32 i = tid; i < (u32)kTriWords; i += kThreads) s_tri[i] = P.tri[i];
  __syncthreads();   // the only block barrier: the tables are shared
  const u16* p6_504 = reinterpret_cast<const u16*>(s_tri + kTriP504);
  const u16* p6_247 = p6_504 + 504;

  const u128 inv21 = ((u128)P.inv21_hi << 64) | P.inv21_lo;
  State617 S;
  S.pos = 0; S.probes = 0;
  u64 my_tri = 0, my_skip = 0;

  for (;;) {
    u32 it = 0;
    if (lane == 0) it = atomicAdd(P.work, 1u);
    it = __shfl_sync(kFull, it, 0);
    if (it >= P.n_items) break;
    const u64 packed = P.items[it];
    if (!S615_CHECK(item_unit(packed) < P.n_units, kChkItem)) continue;   // warp-uniform
    const DevUnit* U = P.units + item_unit(packed);
    Item617 I;
    I.unit_id = U->id;
    I.cls = U->cls;
    I.lim = U->lim;
    u32 nrows;
    u32 part = 0, nparts = 1;   // cls 7: this item's share of the rows' c4 blocks
    const bool single = I.cls == 1 || I.cls == S615_CLS_617_FIND4;
    if (single) {   // one row, T = base; this item's c4 are a chunk of [fmax2, fmax1]
      I.r0 = 0; I.mod = 0; I.j0 = 0;
      nrows = 1;
    } else {
      if (!S615_CHECK(item_res(packed) < U->nres1 && U->nres1 <= 24, kChkItem)) continue;
      I.r0 = U->res1[item_res(packed)];
      I.mod = U->mod1;
      u32 jmin, jend;
      class_rows(I.r0, I.mod, U->fmax1, &jmin, &jend);
      part = item_chunk(packed) % kParts617;
      nparts = kParts617;
      I.j0 = jmin + (item_chunk(packed) / kParts617) * kItemRows617;
      nrows = min(kItemRows617, jend - I.j0);
    }
    const bool tri = P.use_tri && I.cls != 1;   // cls 1 (k_find4) has no triple-sum gate
    const u128 base = ((u128)U->base_hi << 64) | U->base_lo;
    S.nbuf = 0; S.head = 0; S.qlen = 0;
    __syncwarp();

    for (u32 h = 0; h < nrows; h += 32) {
      // ---- the row of this lane: T(d), its c4 window and T mod 504 / 247 ----
      u64 tl = 0, th = 0;
      u32 lo4 = 0, len4 = 0, q504 = 0, q247 = 0;
      if (single) {
        if (lane == 0) {
          const u32 c0 = U->fmax2 + item_chunk(packed) * kC4Chunk;
          if (c0 <= U->fmax1) {
            tl = U->base_lo; th = U->base_hi;
            lo4 = c0;
            len4 = min(kC4Chunk, U->fmax1 - c0 + 1u);
            q504 = mod_small<504>(th, tl);   // the triple-sum gate of cls 8 rows
            q247 = mod_small<247>(th, tl);
          }
        }
      } else if (h + lane < nrows) {
        const u64 x = 21ull * ((u64)I.r0 + (u64)I.mod * (I.j0 + h + lane));
        const u128 x3 = (u128)(x * x) * x;
        const u128 Rm = base - x3 * x3;                          // R mod 2^128
        const u128 T = ((Rm >> 6) * inv21) & ((~(u128)0) >> 6);  // T mod 2^122
        if (T != 0 && (T >> 121) == 0) {
          const u32 hi4 = min(iroot6_u128(T), I.lim);
          if (hi4 >= 1) {
            const u32 l4 = least_c_3c6(T);
            if (l4 <= hi4) {
              lo4 = l4;
              len4 = hi4 - l4 + 1u;
              tl = (u64)T; th = (u64)(T >> 64);
              q504 = mod_small<504>(th, tl);
              q247 = mod_small<247>(th, tl);
            }
          }
        }
      }
      if (tri && part == 0) my_tri += len4;   // a row's c4 are counted once
      // ---- c4 step: triple-sum gate, survivors to the c4 queue ----
      u32 ch = 0, cl = 0;
      const u32 nd = min(32u, nrows - h);
      for (u32 j = 0; j < nd; ++j) {
        const u32 L = __shfl_sync(kFull, len4, j);
        if (L == 0) continue;
        const u32 lo = __shfl_sync(kFull, lo4, j);
        const u32 a504 = __shfl_sync(kFull, q504, j), a247 = __shfl_sync(kFull, q247, j);
        for (u32 c0 = 32u * part; c0 < L; c0 += 32u * nparts) {
          const u32 c4 = lo + c0 + lane;
          bool pass = c0 + lane < L;
          if (pass && tri) {
            u32 x = a504 + 504u - p6_504[c4 % 504u];
            if (x >= 504u) x -= 504u;
            u32 y = a247 + 247u - p6_247[c4 % 247u];
            if (y >= 247u) y -= 247u;
            pass = ((s_tri[kTriT504 + (x >> 5)] >> (x & 31u)) & 1u) &&
                   ((s_tri[kTriT247 + (y >> 5)] >> (y & 31u)) & 1u);
            if (!pass) ++my_skip;
          }
          const u32 bal = __ballot_sync(kFull, pass);
          if (pass) W.cq[(ch + cl + __popc(bal & lanemask_lt())) & (kCQ - 1)] = c4 | (j << kC4Bits);
          cl += __popc(bal);
          if (cl >= 32u) {
            __syncwarp();
            make_rows<kSharp, kSet>(P, W, s_pat, S, I, lane, ch, 32u, h, tl, th);
            ch = (ch + 32u) & (kCQ - 1);
            cl -= 32u;
          }
        }
      }
      if (cl) {   // the queue refers to this half's lane rows: empty it now
        __syncwarp();
        make_rows<kSharp, kSet>(P, W, s_pat, S, I, lane, ch, cl, h, tl, th);
      }
    }
    flush_rows<kSharp, kSet>(P, W, s_pat, S, I, lane);
  }

  // ---- counters: warp reduce, one atomic per warp ----
  u64 pos = S.pos, probes = S.probes;
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    pos += __shfl_xor_sync(kFull, pos, o);
    probes += __shfl_xor_sync(kFull, probes, o);
    my_tri += __shfl_xor_sync(kFull, my_tri, o);
    my_skip += __shfl_xor_sync(kFull, my_skip, o);
  }
  if (lane == 0 && P.count) {
    atomicAdd(&P.ctr->calls, (unsigned long long)pos);
    atomicAdd(&P.ctr->pos, (unsigned long long)pos);
    atomicAdd(&P.ctr->probes, (unsigned long long)probes);
    atomicAdd(&P.ctr->tri_total, (unsigned long long)my_tri);
    atomicAdd(&P.ctr->tri_skipped, (unsigned long long)my_skip);
  }
}

}  // namespace

namespace {

template <bool kSharp, bool kSet>
int launch617(s615_ctx* ctx, const TableView& tv, s615_batch* b, unsigned flags,
              cudaStream_t st, int grid_blocks) {
  // the shared-memory attribute belongs to each device's context: one bit per device
  static std::atomic<unsigned long long> attr_set{0};
  constexpr size_t kSmemTotal = smem_total617<kSharp>();
  const unsigned long long dev_bit = 1ull << (ctx->device & 63);
  if (!(attr_set.load() & dev_bit)) {
    S615_CU(cudaFuncSetAttribute(k_peel617<kSharp, kSet>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSmemTotal));
    attr_set.fetch_or(dev_bit);
  }
  const size_t n = b->n_items - b->n_main;
  if (n == 0) return S615_OK;
  Peel617Params P{};
  P.tv = tv;
  P.units = b->d_units;
  P.n_units = (u32)b->n_units;
  P.items = b->d_items + b->n_main;
  P.n_items = (u32)n;
  P.work = b->d_work + 1;
  P.hits = b->d_hits;
  P.hit_cap = b->hit_cap;
  P.ctr = b->d_ctr;
  const bool gated = !(flags & S615_F_NO_GATE);
  P.pat3 = kSharp ? ctx->d_sharp + kSharpWords : ctx->d_pat + 2 * kPatWords + (gated ? 0 : kPatWords);
  P.p64 = ctx->p64;
  P.count = (flags & kFlagNoCount) ? 0u : 1u;
  P.tri = ctx->d_tri;
  const u128 inv = inv_2adic_u128((u128)kM21);
  P.inv21_lo = (u64)inv;
  P.inv21_hi = (u64)(inv >> 64);
  P.s8 = gated ? 0x7u : 0xFFu;
  P.use_tri = (flags & S615_F_NO_TRI) ? 0u : 1u;
  int grid = grid_blocks;
  if (grid <= 0) {
    int per_sm = 0;
    S615_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_peel617<kSharp, kSet>, kThreads, kSmemTotal));
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
  S615_CU(cudaLaunchKernelEx(&cfg, k_peel617<kSharp, kSet>, P));
  ctx->launches++;
  S615_CU(cudaGetLastError());
  return S615_OK;
}

}  // namespace

int launch_peel617(s615_ctx* ctx, const TableView& tv, s615_batch* b, unsigned flags,
                   cudaStream_t st, int grid_blocks) {
  const bool sharp = (flags & S615_F_SHARP) && !(flags & S615_F_NO_GATE);
  if (tv.shards > 1)
    return sharp ? launch617<true, true>(ctx, tv, b, flags, st, grid_blocks)
                 : launch617<false, true>(ctx, tv, b, flags, st, grid_blocks);
  return sharp ? launch617<true, false>(ctx, tv, b, flags, st, grid_blocks)
               : launch617<false, false>(ctx, tv, b, flags, st, grid_blocks);
}

S615_CHECK_TAKE_DEFINE(check_take_peel617)

}  // namespace s615
