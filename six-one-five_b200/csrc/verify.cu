// verify.cu -- exact re-derivation of the pairs behind filter hits.
//
// The reference expands a hit fingerprint into candidate pairs with
// PairRecover (fourcore_xor_store.hpp:23-51: all i<=j<=N with i^6+j^6 = fp
// mod 2^64) and keeps those whose exact sixth powers add up:
//   cls 5  : a,b <= lim and p6[a]+p6[b] == T          (cls5_gpu_v4.cu:513-523)
//   cls 2-4: b <= c3 and p6[a]+p6[b]+p6[c3] == T       (find_v4.cu:538-543)
//   cls 7  : a,b <= N and a^6+b^6+c3^6+c4^6 == T       (solve_617_v1.cu:1083-1088)
// The surviving set is exactly {(c1,c2): c1 <= c2 <= cmax, c1^6 + c2^6 = S}
// with S the hit's exact remainder and cmax = min(N, lim), min(N, c3) or N; this
// kernel enumerates it directly: one warp per hit, the c1 range
// [1, (S/2)^(1/6)] split into 32 segments, each walked with the two-pointer
// rule (c1 up, c2 down).  Identity, term and gcd checks run on the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstring>
#include <numeric>
#include <vector>

#include "s615_device.cuh"

namespace s615 {

namespace {

struct PairOut { u32 hit, c1, c2, pad; };

__global__ void k_verify(const DevUnit* __restrict__ units, const s615_hit* __restrict__ hits,
                         u32 n_hits, u32 N, u64 inv_lo, u64 inv_hi, PairOut* out, u32 cap,
                         u32* n_out) {
  const u32 lane = threadIdx.x & 31;
  const u32 warps = (gridDim.x * blockDim.x) >> 5;
  const u128 inv21 = ((u128)inv_hi << 64) | inv_lo;
  for (u32 hi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; hi < n_hits; hi += warps) {
    const s615_hit H = hits[hi];
    const DevUnit& U = units[H.unit];
    const u128 base = ((u128)U.base_hi << 64) | U.base_lo;
    u128 S;
    u32 cmax;
    if (U.cls == 1 || U.cls == S615_CLS_617_FIND4) {   // base holds T; S = T - c4^6 - c3^6
      const u128 T = base;
      const u128 c46 = pow6_small(H.c4) + pow6_small(H.e);
      if (T <= c46) continue;
      S = T - c46;
      // cls 1: a <= b <= c3 (run_batch mode 4, fourcore_find_v4.cu:548-554);
      // the (6,1,7) jobs take every pair up to N (expand_xor_hits)
      cmax = U.cls == 1 ? min(N, H.e) : N;
    } else if (U.cls == 5) {
      const u64 x = 14ull * H.e;
      const u128 x3 = (u128)(x * x) * x;
      const u128 V = (base - x3 * x3) * inv21;
      const u128 d6 = pow6_small(H.d);
      if ((V >> 127) || V <= d6) continue;
      const u128 diff = V - d6;
      if ((u64)diff & 63) continue;
      S = diff >> 6;
      cmax = min(N, U.lim);
    } else {
      const u64 x = (u64)U.f * H.d;
      const u128 x3 = (u128)(x * x) * x;
      const u128 T = (((base - x3 * x3) >> 6) * inv21) & ((~(u128)0) >> 6);
      const u128 c6 = pow6_small(H.e);
      if ((T >> 121) || T <= c6) continue;
      S = T - c6;
      cmax = min(N, H.e);
      if (U.cls == kClsJobRow && U.w) cmax = min(N, U.lim);   // find2: a, b <= lim (:537-541)
      if (U.cls == S615_CLS_617) {   // T - c3^6 - c4^6; pairs up to N
        const u128 c46 = pow6_small(H.c4);
        if (S <= c46) continue;
        S -= c46;
        cmax = N;
      }
    }
    const u32 c1max = iroot6_u128(S >> 1);
    if (c1max == 0) continue;
    const u32 seg = (c1max + 31) / 32;
    u32 c1 = 1 + lane * seg;
    const u32 end = min(c1max, c1 + seg - 1);
    if (c1 > c1max) continue;
    u32 c2 = min(iroot6_u128(S - pow6_small(c1)), cmax);
    while (c1 <= end && c2 >= c1) {
      const u128 s = pow6_small(c1) + pow6_small(c2);
      if (s == S) {
        const u32 k = atomicAdd(n_out, 1u);
        if (k < cap) out[k] = PairOut{hi, c1, c2, 0};
        ++c1;
        --c2;
      } else if (s < S) {
        ++c1;
      } else {
        --c2;
      }
    }
  }
}

}  // namespace

int verify_device(s615_ctx* ctx, const s615_unit* units, size_t n_units, const s615_hit* hits,
                  size_t n_hits, int N, s615_solution* out, size_t cap, size_t* n_out) {
  *n_out = 0;
  if (n_hits == 0) return S615_OK;
  for (size_t i = 0; i < n_hits; ++i)
    if (hits[i].unit >= n_units) return S615_E_ARG;
  // Device records for the units that have hits only (a batch can hold
  // millions of units and a handful of hits); the kernel's copy of the hits
  // indexes that short list, the host tail below keeps the caller's indices.
  std::vector<u32> ids(n_hits);
  for (size_t i = 0; i < n_hits; ++i) ids[i] = hits[i].unit;
  std::sort(ids.begin(), ids.end());
  ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
  std::vector<DevUnit> du(ids.size());
  for (size_t k = 0; k < ids.size(); ++k) {
    bool skip = false;
    const int s = make_dev_unit(units[ids[k]], ids[k], &du[k], &skip);
    if (s && !skip) std::memset(&du[k], 0, sizeof du[k]);
  }
  std::vector<s615_hit> kh(hits, hits + n_hits);
  for (s615_hit& h : kh)
    h.unit = (u32)(std::lower_bound(ids.begin(), ids.end(), h.unit) - ids.begin());
  const u32 pcap = (u32)std::min<size_t>(std::max<size_t>(4 * n_hits + 64, 1024), 1u << 26);
  // scratch from the context's grow-only arena: no cudaFree, so no
  // device-wide sync against kernels running on other streams
  void *d_u = nullptr, *d_h = nullptr, *d_p = nullptr, *d_n = nullptr;
  const size_t bu = du.size() * sizeof(DevUnit), bh = n_hits * sizeof(s615_hit);
  const size_t bp = pcap * sizeof(PairOut);
  int s = 0;
  if ((s = arena_get(ctx, 0, bu, &d_u)) || (s = arena_get(ctx, 1, bh, &d_h)) ||
      (s = arena_get(ctx, 2, bp, &d_p)) || (s = arena_get(ctx, 3, 16, &d_n)))
    return s;
  cudaStream_t st = ctx->stream;
  std::vector<PairOut> pairs;
  u32 np = 0;
  {
    const u128 inv = inv_2adic_u128((u128)kM21);
    cudaError_t e = cudaMemcpyAsync(d_u, du.data(), bu, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_h, kh.data(), bh, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_n, 0, 16, st);
    if (e == cudaSuccess) {
      const u32 blocks = (u32)std::min<size_t>((n_hits + 7) / 8, (size_t)ctx->num_sms * 32);
      k_verify<<<blocks, 256, 0, st>>>(static_cast<const DevUnit*>(d_u),
                                       static_cast<const s615_hit*>(d_h), (u32)n_hits, (u32)N,
                                       (u64)inv, (u64)(inv >> 64), static_cast<PairOut*>(d_p), pcap,
                                       static_cast<u32*>(d_n));
      ctx->launches++;
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&np, d_n, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && np > pcap) return S615_E_OVERFLOW;
    if (e == cudaSuccess) {
      pairs.resize(np);
      if (np) e = cudaMemcpyAsync(pairs.data(), d_p, np * sizeof(PairOut), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) return cuda_status(e);
  }
  std::sort(pairs.begin(), pairs.end(), [&](const PairOut& a, const PairOut& b) {
    const s615_hit &ha = hits[a.hit], &hb = hits[b.hit];
    if (ha.unit != hb.unit) return ha.unit < hb.unit;
    if (ha.e != hb.e) return ha.e < hb.e;
    if (ha.d != hb.d) return ha.d < hb.d;
    if (ha.c4 != hb.c4) return ha.c4 < hb.c4;
    if (a.hit != b.hit) return a.hit < b.hit;
    return a.c1 < b.c1;
  });
  size_t k = 0;
  std::vector<std::array<long long, 7>> reported;   // cls 7: distinct 7-tuples only
  for (const PairOut& p : pairs) {
    const s615_hit& H = hits[p.hit];
    const s615_unit& U = units[H.unit];
    s615_solution S{};
    S.unit = H.unit; S.kind = U.kind; S.cls = U.cls; S.B = U.B; S.u = U.u;
    S.c1 = p.c1; S.c2 = p.c2;
    W3 rhs;   // the peeled terms plus 42^6 times the core
    long long t[5];
    if (U.kind == S615_KIND_JOB) {
      // run_batch's exact filter (fourcore_find_v4.cu:536-560), then
      // report_solution's identity and term rules (:427-457).  An exact match
      // whose identity does not hold for (B, u, free terms) stays kind 2: the
      // reference counts it in `sols` but prints nothing.
      const u128 T = ((u128)U.base[1] << 64) | U.base[0];
      u128 core = pow6_u128(p.c1) + pow6_u128(p.c2);
      rhs = pow6_w3(U.u);
      S.d = U.res_d;
      S.e = U.res_e;
      if (U.cls == 1) {
        S.c3 = H.e; S.c4 = H.c4;
        core += pow6_u128(H.e) + pow6_u128(H.c4);
        t[2] = 42LL * H.e; t[3] = 42LL * H.c4;
      } else if (U.cls == 5) {
        add_w3(rhs, pow6_w3(21ULL * U.res_d));
        add_w3(rhs, pow6_w3(14ULL * U.res_e));
        t[2] = 21LL * U.res_d; t[3] = 14LL * U.res_e;
      } else {
        const u64 f = (u64)free_factor((int)U.cls);
        S.c3 = H.e;
        core += pow6_u128(H.e);
        add_w3(rhs, pow6_w3(f * U.res_d));
        t[2] = 42LL * H.e; t[3] = (long long)(f * U.res_d);
      }
      if (core != T) continue;
      add_w3(rhs, mul_w3_u64(W3{{(u64)core, (u64)(core >> 64), 0}}, kM42));
      t[0] = 42LL * p.c1; t[1] = 42LL * p.c2; t[4] = (long long)U.u;
      std::sort(t, t + 5);
      bool ok = eq_w3(rhs, pow6_w3(U.B)) && t[0] >= 1 && t[4] < (long long)U.B;
      for (int i = 0; i < 4; ++i) if (t[i] == t[i + 1]) ok = false;
      if (ok) {
        long long g = t[0];
        for (int i = 1; i < 5; ++i) g = std::gcd(g, t[i]);
        g = std::gcd(g, (long long)U.B);
        for (int i = 0; i < 5; ++i) S.a[i] = t[i];
        S.gcd = g;
        S.kind = 0;
      }
      if (k < cap) out[k] = S;
      ++k;
      continue;
    }
    if (U.cls == S615_CLS_617_FIND4) {   // B^6 = u^6 + w^6 + 42^6 (c1^6 + .. + c5^6)
      S.c3 = H.e; S.c4 = H.c4; S.w = U.w;
      S.d = U.res_d;    // the (6,1,7) class
      S.e = U.res_e;    // c5
      const u128 core = pow6_u128(p.c1) + pow6_u128(p.c2) + pow6_u128(H.e) + pow6_u128(H.c4);
      const u128 Q4 = ((u128)U.base[1] << 64) | U.base[0];
      if (core != Q4) continue;   // the find4 identity (verify_hit, solve_617_v1.cu:1079-1082)
      W3 r = mul_w3_u64(W3{{(u64)(core + pow6_u128(U.res_e)), (u64)((core + pow6_u128(U.res_e)) >> 64), 0}}, kM42);
      add_w3(r, pow6_w3(U.u));
      add_w3(r, pow6_w3(U.w));
      if (!eq_w3(r, pow6_w3(U.B))) continue;
      std::array<long long, 7> t7 = {42LL * p.c1, 42LL * p.c2, 42LL * H.e, 42LL * H.c4,
                                     42LL * U.res_e, (long long)U.w, (long long)U.u};
      std::sort(t7.begin(), t7.end());
      bool bad = false;
      for (int i = 0; i < 6; ++i) if (t7[i] == t7[i + 1]) bad = true;
      if (bad || t7[6] >= (long long)U.B || t7[0] < 1) continue;
      if (std::find(reported.begin(), reported.end(), t7) != reported.end()) continue;
      reported.push_back(t7);
      long long g = t7[0];
      for (int i = 1; i < 7; ++i) g = std::gcd(g, t7[i]);
      g = std::gcd(g, (long long)U.B);
      for (int i = 0; i < 7; ++i) S.a[i] = t7[i];
      S.gcd = g;
      if (k < cap) out[k] = S;
      ++k;
      continue;
    }
    if (U.cls == 1) {   // B^6 = u^6 + 42^6 (c1^6 + c2^6 + c3^6 + c4^6)
      S.c3 = H.e; S.c4 = H.c4;
      const u128 core = pow6_u128(p.c1) + pow6_u128(p.c2) + pow6_u128(H.e) + pow6_u128(H.c4);
      rhs = mul_w3_u64(W3{{(u64)core, (u64)(core >> 64), 0}}, kM42);
      if (U.kind == 1) {
        if (!eq_w3(rhs, W3{{U.base[0], U.base[1], U.base[2]}})) continue;
      } else {
        add_w3(rhs, pow6_w3(U.u));
        if (!eq_w3(rhs, pow6_w3(U.B))) continue;
        t[0] = 42LL * p.c1; t[1] = 42LL * p.c2; t[2] = 42LL * H.e; t[3] = 42LL * H.c4;
        t[4] = (long long)U.u;
        std::sort(t, t + 5);
        bool bad = false;
        for (int i = 0; i < 4; ++i) if (t[i] == t[i + 1]) bad = true;
        if (bad || t[4] >= (long long)U.B || t[0] < 1) continue;
        long long g = t[0];
        for (int i = 1; i < 5; ++i) g = std::gcd(g, t[i]);
        g = std::gcd(g, (long long)U.B);
        for (int i = 0; i < 5; ++i) S.a[i] = t[i];
        S.gcd = g;
      }
      if (k < cap) out[k] = S;
      ++k;
      continue;
    }
    if (U.cls == S615_CLS_617) {
      S.d = H.d; S.c3 = H.e; S.c4 = H.c4; S.w = U.w;
      rhs = pow6_w3(21ULL * H.d);
      const u128 core = pow6_u128(p.c1) + pow6_u128(p.c2) + pow6_u128(H.e) + pow6_u128(H.c4);
      add_w3(rhs, mul_w3_u64(W3{{(u64)core, (u64)(core >> 64), 0}}, kM42));
      if (U.kind == 1) {
        if (!eq_w3(rhs, W3{{U.base[0], U.base[1], U.base[2]}})) continue;
      } else {
        add_w3(rhs, pow6_w3(U.u));
        add_w3(rhs, pow6_w3(U.w));
        if (!eq_w3(rhs, pow6_w3(U.B))) continue;
        std::array<long long, 7> t7 = {42LL * p.c1, 42LL * p.c2, 42LL * H.e, 42LL * H.c4,
                                       21LL * H.d, (long long)U.u, (long long)U.w};
        std::sort(t7.begin(), t7.end());
        bool bad = false;
        for (int i = 0; i < 6; ++i) if (t7[i] == t7[i + 1]) bad = true;
        if (bad || t7[6] >= (long long)U.B || t7[0] < 1) continue;
        if (std::find(reported.begin(), reported.end(), t7) != reported.end()) continue;
        reported.push_back(t7);
        long long g = t7[0];
        for (int i = 1; i < 7; ++i) g = std::gcd(g, t7[i]);
        g = std::gcd(g, (long long)U.B);
        for (int i = 0; i < 7; ++i) S.a[i] = t7[i];
        S.gcd = g;
      }
      if (k < cap) out[k] = S;
      ++k;
      continue;
    }
    if (U.cls == 5) {
      S.d = H.d; S.e = H.e;
      rhs = pow6_w3(21ULL * H.d);
      add_w3(rhs, pow6_w3(14ULL * H.e));
      const u128 core = pow6_u128(p.c1) + pow6_u128(p.c2);
      add_w3(rhs, mul_w3_u64(W3{{(u64)core, (u64)(core >> 64), 0}}, kM42));
      t[0] = 42LL * p.c1; t[1] = 42LL * p.c2; t[2] = 21LL * H.d; t[3] = 14LL * H.e;
    } else {
      const u64 f = (u64)free_factor((int)U.cls);
      S.d = H.d; S.c3 = H.e;
      rhs = pow6_w3(f * H.d);
      const u128 core = pow6_u128(p.c1) + pow6_u128(p.c2) + pow6_u128(H.e);
      add_w3(rhs, mul_w3_u64(W3{{(u64)core, (u64)(core >> 64), 0}}, kM42));
      t[0] = 42LL * p.c1; t[1] = 42LL * p.c2; t[2] = 42LL * H.e; t[3] = (long long)(f * H.d);
    }
    if (U.kind == 1) {
      if (!eq_w3(rhs, W3{{U.base[0], U.base[1], U.base[2]}})) continue;
    } else {
      add_w3(rhs, pow6_w3(U.u));
      if (!eq_w3(rhs, pow6_w3(U.B))) continue;
      t[4] = (long long)U.u;
      std::sort(t, t + 5);
      bool bad = false;
      for (int i = 0; i < 4; ++i) if (t[i] == t[i + 1]) bad = true;
      if (bad || t[4] >= (long long)U.B || t[0] < 1) continue;
      long long g = t[0];
      for (int i = 1; i < 5; ++i) g = std::gcd(g, t[i]);
      g = std::gcd(g, (long long)U.B);
      for (int i = 0; i < 5; ++i) S.a[i] = t[i];
      S.gcd = g;
    }
    if (k < cap) out[k] = S;
    ++k;
  }
  *n_out = k;
  return k > cap ? S615_E_OVERFLOW : S615_OK;
}

}  // namespace s615
