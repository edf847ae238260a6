// cls5_sieve.cu -- the class-5 2-D free peel, residue gate and xor probe.
//
// Replaces k_cls5_192 (fourcore_cls5_gpu_v4.cu:353-410) with the same
// results (raw hits and the calls/gated/probes counters) from a different
// schedule:
//
//  * Exact row arithmetic instead of per-point 192-bit powers.  For a unit
//    (base = B^6-u^6) and a row e, V(e) = (base - (14e)^6) / 21^6 is an exact
//    integer below 2^112, and for every d in the row
//        T(e,d) = (base - (14e)^6 - (21d)^6) / 42^6 = (V(e) - d^6) / 64,
//    so R > 0  <=>  d^6 < V(e)  <=>  d <= D(e) := iroot6(V(e) - 1).
//    The in-row limit and the probe key T mod 2^64 come from V, computed
//    once per row from base mod 2^128 and the 2-adic inverse of 21^6.
//  * The gate as a sieve.  The reference keeps T iff T mod 504 and T mod 247
//    are sums of two sixth powers.  Those sets are products over 8,9,7,13,19
//    ({0,1,2} mod 8, 9, 7; 5 of 13; 10 of 19), and along a row d = d0 + 64k
//    each factor is periodic in k.  A lane evaluates the gate for 32
//    consecutive k at once as the AND of one row constant (mod 8) and four
//    32-bit pattern words from shared memory (mod 9, 7, 13, 19).
//  * Compaction before probing.  Gate survivors go to a per-warp ring in
//    shared memory; each full batch of 32 is probed by all 32 lanes together
//    (three independent L2-only cell loads per lane in flight).
//  * Warps are independent workers: each pulls (unit, e residue, 64-row
//    chunk) items from one device-wide queue, sets its rows up in its own
//    slice of shared memory and sieves every d residue and k tile of them.
//    Nothing waits at a block barrier, so a slow item delays only its warp.
#include <cuda_runtime.h>

#include "s615_device.cuh"

namespace s615 {

namespace {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr u32 kRows = kItemRows;  // e-rows per item (64)
constexpr u32 kMaxD = 4;          // d residues per pass
constexpr u32 kQ = 64;            // warp ring capacity (power of two)
constexpr u32 kNoRow = 0xFFFFFFFFu;

struct __align__(16) RowRec {
  u64 vlo, vhi;   // V(e) mod 2^128
  u32 D;          // iroot6(V-1)
  u32 v512;       // V mod 512, or kNoRow when V <= 0 (no R>0 point)
  u16 off[4];     // pattern-table word offset per q for a = V mod q
};

struct WarpSmem {                 // one warp's private slice
  RowRec rows[kRows];             // 2048 B
  u16 K[kMaxD][kRows];            // in-row k limit per d residue (k < 2^16)
  u8 M4[kMaxD][kRows];            // mod-8 admissibility of k = 0..3 (mod 4)
  u32 ring[kQ];
  u32 d0s[kMaxD];                 // d residues of the current pass
};

struct SieveParams {
  TableView tv;
  const DevUnit5* units;
  const u32* items;
  u32 n_items;
  u32* work;
  s615_hit* hits;
  u32 hit_cap;
  Cls5Counters* ctr;
  const u32* pat;
  u64 inv21_lo, inv21_hi;  // (21^6)^-1 mod 2^128
  u32 s8;                  // admissible T mod 8, as a bitmask
};

constexpr size_t kSmemPat = kPatWords * sizeof(u32);                // 2640
constexpr size_t kSmemTotal = kSmemPat + kWarps * sizeof(WarpSmem);

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

// x^6 mod 512 for small x.
__device__ __forceinline__ u32 pow6_mod512(u32 x) {
  x &= 511;
  const u32 x2 = (x * x) & 511;
  const u32 x3 = (x2 * x) & 511;
  return (x3 * x3) & 511;
}

// Ring entry: k (16 bits) | row (6 bits) << 16 | d-residue slot (2 bits) << 22.
__device__ __forceinline__ u32 entry(u32 di, u32 r, u32 k) { return (di << 22) | (r << 16) | k; }

// Probe the ring entries [head, head+cnt) (one per lane).
__device__ __forceinline__ void probe_batch(const SieveParams& P, const WarpSmem& W, u32 head,
                                            u32 cnt, u32 e0, u32 j0, u32 unit_id, u32 lane) {
  if (lane >= cnt) return;
  const u32 ent = W.ring[(head + lane) & (kQ - 1)];
  const u32 k = ent & 0xFFFFu, r = (ent >> 16) & 63u, di = ent >> 22;
  const RowRec& R = W.rows[r];
  const u64 d = (u64)W.d0s[di] + 64ull * k;
  const u128 V = ((u128)R.vhi << 64) | R.vlo;
  const u128 diff = V - pow6_small(d);
  const u64 key = (u64)(diff >> 6);
  if (might_contain(P.tv, key)) {
    const unsigned long long idx = atomicAdd(&P.ctr->hits, 1ull);
    if (idx < P.hit_cap) {
      s615_hit h;
      h.unit = unit_id; h.a = 0; h.b = 0;
      h.d = (u32)d;
      h.e = e0 + 729u * (j0 + r);
      h.fp = key;
      P.hits[idx] = h;
    }
  }
}

__global__ void __launch_bounds__(kThreads, 6) k_cls5_sieve(SieveParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  u32* s_pat = reinterpret_cast<u32*>(smem);
  const u32 tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  WarpSmem& W = reinterpret_cast<WarpSmem*>(smem + kSmemPat)[warp];
  for (u32 i = tid; i < (u32)kPatWords; i += kThreads) s_pat[i] = P.pat[i];
  __syncthreads();   // the only block barrier: pattern tables are shared

  const u128 inv21 = ((u128)P.inv21_hi << 64) | P.inv21_lo;
  u64 my_calls = 0, my_pos = 0, my_probes = 0;

  for (;;) {
    u32 it = 0;
    if (lane == 0) it = atomicAdd(P.work, 1u);
    it = __shfl_sync(0xFFFFFFFFu, it, 0);
    if (it >= P.n_items) break;
    const u32 packed = P.items[it];
    const DevUnit5* U = P.units + item_unit(packed);
    const u32 e0 = U->res1[item_eres(packed)];
    const u32 fmax2 = U->fmax2, nres2 = U->nres2, unit_id = U->id;
    u32 jmin, jend;
    e_rows(e0, U->fmax1, &jmin, &jend);
    const u32 j0 = jmin + item_chunk(packed) * kRows;
    const u32 nrows = min(kRows, jend - j0);
    const u128 base = ((u128)U->base_hi << 64) | U->base_lo;

    // ---- row set-up: V, D and the residues of V (two rows per lane) ----
    for (u32 r = lane; r < nrows; r += 32) {
      const u64 x = 14ull * ((u64)e0 + 729ull * (j0 + r));
      const u128 x3 = (u128)(x * x) * x;           // (14e)^3 < 2^78
      const u128 V = (base - x3 * x3) * inv21;    // exact mod 2^128
      RowRec R;
      R.vlo = (u64)V; R.vhi = (u64)(V >> 64);
      if ((R.vhi >> 63) || V == 0) {
        R.D = 0; R.v512 = kNoRow;
        R.off[0] = R.off[1] = R.off[2] = R.off[3] = 0;
      } else {
        R.D = iroot6_u128(V - 1);
        R.v512 = (u32)(R.vlo & 511u);
        R.off[0] = (u16)(kPatB9 + 9 * mod_small<9>(R.vhi, R.vlo));
        R.off[1] = (u16)(kPatB7 + 7 * mod_small<7>(R.vhi, R.vlo));
        R.off[2] = (u16)(kPatB13 + 13 * mod_small<13>(R.vhi, R.vlo));
        R.off[3] = (u16)(kPatB19 + 19 * mod_small<19>(R.vhi, R.vlo));
      }
      W.rows[r] = R;
    }
    u32 head = 0, qlen = 0;

    for (u32 dg = 0; dg < nres2; dg += kMaxD) {
      const u32 nd = min(kMaxD, nres2 - dg);
      __syncwarp();
      if (lane < kMaxD) W.d0s[lane] = lane < nd ? U->res2[dg + lane] : 0u;
      __syncwarp();
      // ---- per (row, d residue): in-row limit and the mod-8 row mask ----
      u32 kmax = 0;
      for (u32 idx = lane; idx < nd * kRows; idx += 32) {
        const u32 di = idx / kRows, r = idx % kRows;
        if (r >= nrows) continue;
        const u32 d0 = W.d0s[di];
        const RowRec& R = W.rows[r];
        const u32 kcap = (d0 <= fmax2) ? (fmax2 - d0) / 64u + 1u : 0u;
        const u32 kpos = (R.v512 != kNoRow && R.D >= d0) ? (R.D - d0) / 64u + 1u : 0u;
        const u32 kend = min(kcap, kpos);
        const u32 kmin = (d0 == 0) ? 1u : 0u;
        if (kend > kmin) my_pos += kend - kmin;
        if (r == 0) my_calls += (u64)nrows * (kcap > kmin ? kcap - kmin : 0u);
        kmax = max(kmax, kend);
        u32 m4 = 0;
        if (R.v512 != kNoRow) {
#pragma unroll
          for (u32 i = 0; i < 4; ++i) {
            const u32 t8 = ((R.v512 - pow6_mod512(d0 + 64u * i)) & 511u) >> 6;
            m4 |= ((P.s8 >> t8) & 1u) << i;
          }
        }
        W.K[di][r] = (u16)kend;
        W.M4[di][r] = (u8)m4;
      }
#pragma unroll
      for (int o = 16; o; o >>= 1) kmax = max(kmax, __shfl_xor_sync(0xFFFFFFFFu, kmax, o));
      __syncwarp();

      // ---- sieve: lanes cover 32 words (1024 k) of a tile, rows in order ----
      const u32 ntiles = (kmax + 1023u) / 1024u;
      for (u32 di = 0; di < nd; ++di) {
        const u32 d0 = W.d0s[di];
        const u32 lowmask0 = (d0 == 0) ? ~1u : ~0u;
        for (u32 wt = 0; wt < ntiles; ++wt) {
          const u32 w = wt * 32u + lane;
          const u32 kbase = w * 32u;
          const u64 dstart = (u64)d0 + 64ull * kbase;
          const u32 s9 = (u32)(dstart % 9), s7 = (u32)(dstart % 7);
          const u32 s13 = (u32)(dstart % 13), s19 = (u32)(dstart % 19);
          const u32 lowmask = (kbase == 0) ? lowmask0 : ~0u;
          for (u32 r = 0; r < nrows; ++r) {
            const u32 kend = W.K[di][r];
            if (kend <= wt * 1024u) break;
            u32 m = 0;
            if (kbase < kend) {
              const uint2 offs = *reinterpret_cast<const uint2*>(&W.rows[r].off[0]);
              m = ((u32)W.M4[di][r] * 0x11111111u) & s_pat[(offs.x & 0xFFFFu) + s9] & s_pat[(offs.x >> 16) + s7] &
                  s_pat[(offs.y & 0xFFFFu) + s13] & s_pat[(offs.y >> 16) + s19];
              const u32 n = kend - kbase;
              if (n < 32u) m &= (1u << n) - 1u;
              m &= lowmask;
            }
            my_probes += __popc(m);
            while (__any_sync(0xFFFFFFFFu, m != 0)) {
              const bool has = m != 0;
              const u32 bit = has ? (u32)(__ffs(m) - 1) : 0u;
              m &= m - 1u;
              const u32 ballot = __ballot_sync(0xFFFFFFFFu, has);
              if (has)
                W.ring[(head + qlen + __popc(ballot & lanemask_lt())) & (kQ - 1)] =
                    entry(di, r, kbase + bit);
              qlen += __popc(ballot);
              if (qlen >= 32u) {
                __syncwarp();
                probe_batch(P, W, head, 32u, e0, j0, unit_id, lane);
                __syncwarp();
                head = (head + 32u) & (kQ - 1);
                qlen -= 32u;
              }
            }
          }
        }
      }
      __syncwarp();
      probe_batch(P, W, head, qlen, e0, j0, unit_id, lane);   // drain before d0s change
      head = 0;
      qlen = 0;
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
  if (lane == 0) {
    atomicAdd(&P.ctr->calls, (unsigned long long)my_calls);
    atomicAdd(&P.ctr->pos, (unsigned long long)my_pos);
    atomicAdd(&P.ctr->probes, (unsigned long long)my_probes);
  }
}

}  // namespace

int launch_cls5_sieve(s615_ctx* ctx, const TableView& tv, s615_batch* b, unsigned flags,
                      cudaStream_t st, int grid_blocks) {
  static bool attr_set = false;
  if (!attr_set) {
    S615_CU(cudaFuncSetAttribute(k_cls5_sieve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSmemTotal));
    attr_set = true;
  }
  SieveParams P{};
  P.tv = tv;
  P.units = b->d_units;
  P.items = b->d_items;
  P.n_items = (u32)b->n_items;
  P.work = b->d_work;
  P.hits = b->d_hits;
  P.hit_cap = b->hit_cap;
  P.ctr = b->d_ctr;
  const bool gated = !(flags & S615_F_NO_GATE);
  P.pat = gated ? ctx->d_pat_gate : ctx->d_pat_open;
  const u128 inv = inv_2adic_u128((u128)kM21);
  P.inv21_lo = (u64)inv;
  P.inv21_hi = (u64)(inv >> 64);
  P.s8 = gated ? 0x7u : 0xFFu;
  if (b->n_items == 0) return S615_OK;
  int grid = grid_blocks;
  if (grid <= 0) {
    int per_sm = 0;
    S615_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cls5_sieve, kThreads,
                                                          kSmemTotal));
    grid = ctx->num_sms * (per_sm > 0 ? per_sm : 1);
  }
  const size_t need = (b->n_items + kWarps - 1) / kWarps;
  if ((size_t)grid > need) grid = (int)need;
  k_cls5_sieve<<<grid, kThreads, kSmemTotal, st>>>(P);
  ctx->launches++;
  S615_CU(cudaGetLastError());
  return S615_OK;
}

}  // namespace s615
