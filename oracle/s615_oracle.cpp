// s615_oracle.cpp -- CPU oracle for the cls5 peel / gate / xor-probe path.
//
// TEST INFRASTRUCTURE ONLY: a plain CPU restatement of the reference
// (cavedave/six-one-five) used as the checker by tests/, by
// __graft_entry__.smoke() and by bench.py's cpu_baseline / reference leg.
// It deliberately follows the reference algorithm step for step (per-point
// 192-bit peel, mod-192 gate, funnel fingerprint, FIFO xor peel), not the
// product's algorithm, so that agreement between the two is evidence.
//
// Exact arithmetic uses unsigned __int128 and 3-limb words (the reference uses
// GMP for the same values; GMP only computes exact powers and differences).

#include "s615_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#include <random>
#endif

typedef unsigned __int128 u128;
typedef uint64_t u64;
typedef uint32_t u32;

namespace {

// ----------------------------------------------------------------- constants
// fourcore_classes_v3.hpp:30-35
constexpr long long kM2 = 64, kM3 = 729, kM7 = 117649;
constexpr u64 kM42 = 5489031744ULL;   // 42^6
constexpr u64 kM21 = 85766121ULL;     // 21^6
constexpr u64 kPhi = 0x9E3779B97F4A7C15ULL;
constexpr u64 kSeedBase = 0x615615615615615ULL;  // xor_filter.hpp:448
constexpr u32 kMagic = 0x53353136u;              // store_header.hpp:151

// ------------------------------------------------------ 192-bit exact words
struct W3 { u64 l[3]; };  // little-endian limbs l[0] lowest

W3 w3_u128(u128 v) { return W3{{(u64)v, (u64)(v >> 64), 0}}; }

// x^6 exact for x < 2^32 (cls5_gpu_v4.cu:78-93 computes the same value).
W3 w3_pow6(u64 x) {
  const u64 x2 = x * x;                    // < 2^64
  const u128 x4 = (u128)x2 * x2;           // < 2^128
  const u128 lo = (u128)(u64)x4 * x2;
  const u128 hi = (u128)(u64)(x4 >> 64) * x2;
  W3 r;
  r.l[0] = (u64)lo;
  const u128 mid = (lo >> 64) + (u128)(u64)hi;
  r.l[1] = (u64)mid;
  r.l[2] = (u64)(hi >> 64) + (u64)(mid >> 64);
  return r;
}

// a -= b; returns true on borrow (cls5_gpu_v4.cu:95-108 semantics).
bool w3_sub(W3& a, const W3& b) {
  u64 br = 0;
  for (int i = 0; i < 3; ++i) {
    const u128 d = (u128)a.l[i] - b.l[i] - br;
    a.l[i] = (u64)d;
    br = (u64)(d >> 64) ? 1 : 0;
  }
  return br != 0;
}
void w3_add(W3& a, const W3& b) {
  u128 c = 0;
  for (int i = 0; i < 3; ++i) {
    c += (u128)a.l[i] + b.l[i];
    a.l[i] = (u64)c;
    c >>= 64;
  }
}
W3 w3_mul_u64(const W3& a, u64 m) {
  W3 r;
  u128 c = 0;
  for (int i = 0; i < 3; ++i) {
    c += (u128)a.l[i] * m;
    r.l[i] = (u64)c;
    c >>= 64;
  }
  return r;
}
bool w3_zero(const W3& a) { return (a.l[0] | a.l[1] | a.l[2]) == 0; }
bool w3_eq(const W3& a, const W3& b) {
  return a.l[0] == b.l[0] && a.l[1] == b.l[1] && a.l[2] == b.l[2];
}
// Exact a mod m (the value mod192 of cls5_gpu_v4.cu:300-308 returns).
u64 w3_mod(const W3& a, u64 m) {
  u128 r = 0;
  for (int i = 2; i >= 0; --i) r = ((r << 64) | a.l[i]) % m;
  return (u64)r;
}
// Exact division by a 64-bit divisor; returns remainder.
u64 w3_divmod(W3& a, u64 m) {
  u128 r = 0;
  for (int i = 2; i >= 0; --i) {
    const u128 cur = (r << 64) | a.l[i];
    a.l[i] = (u64)(cur / m);
    r = cur % m;
  }
  return (u64)r;
}
bool w3_fits128(const W3& a) { return a.l[2] == 0; }
u128 w3_to128(const W3& a) { return ((u128)a.l[1] << 64) | a.l[0]; }

u128 pow6_u128(u64 x) { const u128 a = (u128)x * x; return a * a * a; }

// ------------------------------------------------ modular helpers (classes)
// fourcore_classes_v3.hpp:37-66
long long mod_pow6(long long b, long long m) {
  long long r = 1;
  b %= m; if (b < 0) b += m;
  for (int i = 0; i < 6; ++i) r = (long long)((__int128)r * b % m);
  return r;
}
long long egcd(long long a, long long b, long long& x, long long& y) {
  if (b == 0) { x = 1; y = 0; return a; }
  long long x1, y1;
  const long long g = egcd(b, a % b, x1, y1);
  x = y1; y = x1 - y1 * (a / b);
  return g;
}
long long mod_inv(long long a, long long m) {
  long long x, y;
  egcd(a, m, x, y);
  x %= m; if (x < 0) x += m;
  return x;
}
long long crt2(long long r1, long long m1, long long r2, long long m2) {
  long long x, y;
  const long long g = egcd(m1, m2, x, y);
  const long long t = ((r2 - r1) / g) * x;
  const long long mod = m1 / g * m2;
  long long a = r1 + m1 * (t % (m2 / g));
  a %= mod; if (a < 0) a += mod;
  return a;
}

// Sixth-power root tables over units (fourcore_classes_v3.hpp:68-78).
struct Roots {
  std::vector<std::vector<long long>> r2, r3, r7;
  Roots() : r2(kM2), r3(kM3), r7(kM7) {
    for (long long a = 1; a < kM2; ++a) if (std::gcd(a, kM2) == 1) r2[mod_pow6(a, kM2)].push_back(a);
    for (long long a = 1; a < kM3; ++a) if (std::gcd(a, kM3) == 1) r3[mod_pow6(a, kM3)].push_back(a);
    for (long long a = 1; a < kM7; ++a) if (std::gcd(a, kM7) == 1) r7[mod_pow6(a, kM7)].push_back(a);
  }
};
const Roots& roots() { static Roots R; return R; }

long long class_modulus(int cls) {  // classes_v3.hpp:84-91
  switch (cls) { case 1: return kM2 * kM3 * kM7; case 2: return kM2 * kM7;
                 case 3: return kM3 * kM7; default: return kM7; }
}
bool unit_ok(long long u, int cls) {  // classes_v3.hpp:102-111
  switch (cls) {
    case 1: return (u & 1) && std::gcd(u, 42LL) == 1;
    case 2: return (u & 1) && (u % 3 == 0) && (u % 9 != 0);
    case 3: return !(u & 1) && std::gcd(u, 21LL) == 1;
    case 4: case 5: return (u % 6 == 0) && (u % 7 != 0);
  }
  return false;
}
// classes_v3.hpp:114-135
std::vector<long long> seeds_for_B(long long B, int cls) {
  const Roots& rt = roots();
  const long long b2 = mod_pow6(B, kM2), b3 = mod_pow6(B, kM3), b7 = mod_pow6(B, kM7);
  std::vector<long long> out;
  if (cls == 1) {
    for (long long s2 : rt.r2[b2]) for (long long s3 : rt.r3[b3]) {
      const long long s23 = crt2(s2, kM2, s3, kM3);
      for (long long s7 : rt.r7[b7]) out.push_back(crt2(s23, kM2 * kM3, s7, kM7));
    }
  } else if (cls == 2) {
    for (long long s2 : rt.r2[b2]) for (long long s7 : rt.r7[b7]) out.push_back(crt2(s2, kM2, s7, kM7));
  } else if (cls == 3) {
    for (long long s3 : rt.r3[b3]) for (long long s7 : rt.r7[b7]) out.push_back(crt2(s3, kM3, s7, kM7));
  } else {
    out = rt.r7[b7];
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}
// classes_v3.hpp:137-154 with the full band lo_frac=0, hi_frac=1.
std::vector<long long> unit_candidates(long long B, int cls) {
  const long long M = class_modulus(cls);
  const long long lo = std::max(1LL, (long long)(0.0 * (double)B));
  const long long hi = std::min(B - 1, (long long)(1.0 * (double)B));
  std::vector<long long> out;
  if (lo > hi) return out;
  for (long long s : seeds_for_B(B, cls)) {
    long long u = s % M; if (u < 0) u += M;
    if (u < lo) u += (lo - u + M - 1) / M * M;
    for (; u <= hi; u += M) if (unit_ok(u, cls)) out.push_back(u);
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}
// classes_v3.hpp:156-180
std::vector<long long> classes_d_cls2(long long B) {
  const long long t = mod_pow6(B, kM3) * mod_inv(mod_pow6(14, kM3), kM3) % kM3;
  return roots().r3[t];
}
std::vector<long long> classes_d_cls3(long long B, long long u) {
  long long rhs = (mod_pow6(B, kM2) - mod_pow6(u, kM2)) % kM2; if (rhs < 0) rhs += kM2;
  const long long t = rhs * mod_inv(mod_pow6(21, kM2), kM2) % kM2;
  return roots().r2[t];
}
std::vector<long long> classes_d_cls4(long long B) {
  const long long t2 = mod_pow6(B, kM2) * mod_inv(mod_pow6(7, kM2), kM2) % kM2;
  const long long t3 = mod_pow6(B, kM3) * mod_inv(mod_pow6(7, kM3), kM3) % kM3;
  std::vector<long long> out;
  for (long long a : roots().r2[t2]) for (long long b : roots().r3[t3]) out.push_back(crt2(a, kM2, b, kM3));
  std::sort(out.begin(), out.end());
  return out;
}

// ----------------------------------------------------------------- mixers
// spike/ribbon/mix64.hpp:13-25
u64 mix64(u64 x) {
  x ^= x >> 33; x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33;
  return x;
}

// ---------------------------------------------------- packed cells (xor_pack)
u64 fp_mask(u32 r) { return r >= 64 ? ~0ULL : ((1ULL << r) - 1ULL); }  // xor_pack.hpp:14-16
size_t packed_bytes(u64 m, u32 r) {                                     // xor_pack.hpp:19-23
  if (m == 0 || r == 0) return 0;
  return (size_t)((m * (u64)r + 7) / 8 + 8);
}
u64 rd8(const uint8_t* p) { u64 w; std::memcpy(&w, p, 8); return w; }
void wr8(uint8_t* p, u64 w) { std::memcpy(p, &w, 8); }
// xor_pack.hpp:29-60
u64 load_cell(const uint8_t* p, u64 i, u32 r) {
  const u64 bit = i * (u64)r, byte = bit >> 3;
  const unsigned off = (unsigned)(bit & 7);
  const u64 w = rd8(p + byte);
  if (off + r <= 64) return (w >> off) & fp_mask(r);
  const u64 w2 = rd8(p + byte + 8);
  return ((w >> off) | (w2 << (64 - off))) & fp_mask(r);
}
// xor_pack.hpp:67-113
void store_cell(uint8_t* p, u64 i, u32 r, u64 v) {
  v &= fp_mask(r);
  const u64 bit = i * (u64)r, byte = bit >> 3;
  const unsigned off = (unsigned)(bit & 7);
  if (off + r <= 64) {
    const u64 wm = fp_mask(r) << off;
    wr8(p + byte, (rd8(p + byte) & ~wm) | (v << off));
    return;
  }
  const unsigned lowb = 64 - off;
  const u64 lowm = lowb >= 64 ? ~0ULL : ((1ULL << lowb) - 1);
  wr8(p + byte, (rd8(p + byte) & ~(lowm << off)) | ((v & lowm) << off));
  const unsigned highb = r - lowb;
  const u64 highm = highb >= 64 ? ~0ULL : ((1ULL << highb) - 1);
  wr8(p + byte + 8, (rd8(p + byte + 8) & ~highm) | ((v >> lowb) & highm));
}

// xor_filter.hpp:185-192
size_t capacity_for(size_t n) {
  const double need = 32.0 + 1.23 * (double)n;
  size_t cap = (size_t)(need + 0.999);
  if (cap < 3) cap = 3;
  return (cap + 2) / 3 * 3;
}
// xor_filter.hpp:53-60
void hashes3(u64 h, u64 block, u64 out[3]) {
  out[0] = h % block;
  out[1] = mix64(h ^ 0x9E3779B97F4A7C15ULL) % block + block;
  out[2] = mix64(h ^ 0xBF58476D1CE4E5B9ULL) % block + 2 * block;
}

}  // namespace

struct orc_table {
  orc_header hdr;
  std::vector<uint8_t> packed;
  // a shard set: the probe of key k goes to parts[mix64(k + shard_seed) % S]
  std::vector<const orc_table*> parts;
  u64 shard_seed = 0;
};

namespace {

orc_header make_header(u32 r, u64 n, u64 m, u64 seed) {
  orc_header h{};
  h.magic = kMagic; h.version = 2; h.kind = 1; h.r = r; h.w = 0; h.N = 0;
  h.n_keys = n; h.m_cells = m; h.mix_seed = seed;
  h.shard_count = 1; h.shard_index = 0; h.shard_mode = 0; h.reserved = 0;
  return h;
}

// construct_with_seed (xor_filter.hpp:256-431), in memory: incidence, FIFO
// peel queue seeded with every count-1 cell in index order, reverse fill.
bool construct(const std::vector<u64>& keys, u32 r, u64 seed, orc_table& out) {
  const size_t n = keys.size();
  if (n == 0) {
    out.hdr = make_header(r, 0, 0, seed);
    out.packed.clear();
    return true;
  }
  const size_t m = capacity_for(n);
  const u64 block = m / 3;
  std::vector<u64> setxor(m, 0);
  std::vector<uint16_t> counts(m, 0);
  for (size_t k = 0; k < n; ++k) {
    const u64 h = mix64(keys[k] + seed);
    u64 hs[3]; hashes3(h, block, hs);
    for (int t = 0; t < 3; ++t) {
      setxor[hs[t]] ^= h;
      if (counts[hs[t]] == 0xffff) throw std::runtime_error("cell incidence overflow");
      counts[hs[t]]++;
    }
  }
  std::vector<u64> queue;
  for (size_t i = 0; i < m; ++i) if (counts[i] == 1) queue.push_back(i);
  std::vector<std::pair<u64, u64>> stack;  // (hash, alone cell)
  stack.reserve(n);
  for (size_t q = 0; q < queue.size(); ++q) {
    const u64 i = queue[q];
    if (counts[i] != 1) continue;
    const u64 h = setxor[i];
    u64 hs[3]; hashes3(h, block, hs);
    stack.emplace_back(h, i);
    for (int t = 0; t < 3; ++t) {
      const u64 j = hs[t];
      setxor[j] ^= h;
      if (counts[j] > 0) { counts[j]--; if (counts[j] == 1) queue.push_back(j); }
    }
  }
  if (stack.size() != n) return false;
  out.packed.assign(packed_bytes(m, r), 0);
  for (size_t k = stack.size(); k-- > 0;) {
    const u64 h = stack[k].first, idx = stack[k].second;
    u64 hs[3]; hashes3(h, block, hs);
    u64 v = h & fp_mask(r);
    for (int t = 0; t < 3; ++t) if (hs[t] != idx) v ^= load_cell(out.packed.data(), hs[t], r);
    store_cell(out.packed.data(), idx, r, v & fp_mask(r));
  }
  out.hdr = make_header(r, n, m, seed);
  return true;
}

// shard_of_key (spike/ribbon/shard.hpp:19-24): mix64_seeded(key, seed) % S.
u32 shard_of(u64 key, u64 seed, u32 S) { return S <= 1 ? 0u : (u32)(mix64(key + seed) % S); }

bool might_contain(const orc_table& t, u64 key) {  // xor_filter.hpp:472-483
  if (!t.parts.empty()) {   // residue-steered probe: one query, in the key's own shard
    const orc_table* p = t.parts[shard_of(key, t.shard_seed, (u32)t.parts.size())];
    return p && might_contain(*p, key);   // a shard not held here answers nothing
  }
  if (t.hdr.n_keys == 0) return false;
  if (t.packed.empty() || t.hdr.m_cells < 3) return false;
  const u64 block = t.hdr.m_cells / 3;
  const u64 h = mix64(key + t.hdr.mix_seed);
  u64 hs[3]; hashes3(h, block, hs);
  const u64 got = load_cell(t.packed.data(), hs[0], t.hdr.r) ^
                  load_cell(t.packed.data(), hs[1], t.hdr.r) ^
                  load_cell(t.packed.data(), hs[2], t.hdr.r);
  return got == (h & fp_mask(t.hdr.r));
}

// ------------------------------------------------------------------- gate
// cls5_gpu_v4.cu:111-137: achievable pair sums i^6+j^6 mod 504 and mod 247.
struct Gate {
  uint8_t g504[504], g247[247];
  u32 p6504[504], p6247[247];
  Gate() {
    std::memset(g504, 0, sizeof g504); std::memset(g247, 0, sizeof g247);
    for (int i = 0; i < 504; ++i) p6504[i] = (u32)mod_pow6(i, 504);
    for (int i = 0; i < 247; ++i) p6247[i] = (u32)mod_pow6(i, 247);
    for (int i = 0; i < 504; ++i) for (int j = i; j < 504; ++j) g504[(p6504[i] + p6504[j]) % 504] = 1;
    for (int i = 0; i < 247; ++i) for (int j = i; j < 247; ++j) g247[(p6247[i] + p6247[j]) % 247] = 1;
  }
};
const Gate& gate() { static Gate G; return G; }

u64 inv_mod_2_64(u64 a) {  // Newton iteration for an odd a
  u64 x = a;
  for (int i = 0; i < 6; ++i) x *= 2 - a * x;
  return x;
}

// ---------------------------------------------------------------- packing
bool pack_unit5(u64 B, u64 u, orc_unit5& U) {  // cls5_gpu_v4.cu:169-184
  std::memset(&U, 0, sizeof U);
  U.B = B; U.u = u; U.lim = (u32)((B - 1) / 42);
  W3 base = w3_pow6(B);
  if (u >= B) return false;
  if (w3_sub(base, w3_pow6(u)) || w3_zero(base)) return false;
  std::memcpy(U.base, base.l, sizeof U.base);
  const auto er = classes_d_cls2((long long)B);          // e: (14e)^6 = B^6 (3^6)
  const auto dr = classes_d_cls3((long long)B, (long long)u);  // d: (21d)^6 = B^6-u^6 (2^6)
  U.mod1 = (u32)kM3; U.fmax1 = (u32)((B - 1) / 14);
  U.mod2 = (u32)kM2; U.fmax2 = (u32)((B - 1) / 21);
  U.nres1 = (u32)std::min<size_t>(er.size(), 12);
  U.nres2 = (u32)std::min<size_t>(dr.size(), 12);
  for (u32 i = 0; i < U.nres1; ++i) U.res[i] = (u32)er[i];
  for (u32 i = 0; i < U.nres2; ++i) U.res[U.nres1 + i] = (u32)dr[i];
  return U.nres1 > 0 && U.nres2 > 0;
}

// ------------------------------------------------- per-unit peel (k_cls5_192)
struct PeelCtx {
  u64 inv216, m504, c504, inv42_247;
  PeelCtx() {
    inv216 = inv_mod_2_64(kM21);
    m504 = 504ULL * kM42;
    inv42_247 = (u64)mod_inv(mod_pow6(42, 247), 247);
  }
};

template <typename OnHit>
void peel_unit(const orc_table& t, const orc_unit5& U, u32 ui, bool use_gate,
               u64 ctr[3], OnHit&& on_hit) {
  static const PeelCtx C;
  const Gate& G = gate();
  const W3 base{{U.base[0], U.base[1], U.base[2]}};
  const u32 kmax1 = U.fmax1 / U.mod1 + 1;
  const u32 total2 = U.nres2 * (U.fmax2 / U.mod2 + 1);
  for (u32 t1 = 0; t1 < U.nres1 * kmax1; ++t1) {                // blockIdx.y
    const u32 e = U.res[t1 % U.nres1] + (t1 / U.nres1) * U.mod1;
    if (e == 0 || e > U.fmax1) continue;
    const W3 E = w3_pow6(14u * e);
    for (u32 t2 = 0; t2 < total2; ++t2) {                      // threads stride d
      const u32 d = U.res[U.nres1 + t2 % U.nres2] + (t2 / U.nres2) * U.mod2;
      if (d == 0 || d > U.fmax2) continue;
      ++ctr[0];
      W3 R = base;
      if (w3_sub(R, E)) continue;
      if (w3_sub(R, w3_pow6(21u * d))) continue;
      if (w3_zero(R)) continue;
      if (use_gate) {
        const u64 rmod = w3_mod(R, C.m504);
        const u32 t504 = (u32)((rmod / kM42) % 504);
        const u64 r247 = w3_mod(R, 247);
        const u32 t247 = (u32)(r247 * C.inv42_247 % 247);
        if (!(G.g504[t504] && G.g247[t247])) { ++ctr[1]; continue; }
      }
      ++ctr[2];
      const u64 fp = ((R.l[0] >> 6) | (R.l[1] << 58)) * C.inv216;   // funnel
      if (might_contain(t, fp)) on_hit(orc_hit{ui, 0, 0, d, e, fp});
    }
  }
}

// ------------------------------------------------------- PairRecover + verify
// fourcore_xor_store.hpp:23-51
struct PairRecover {
  int N = 0;
  std::vector<u64> pw6;
  std::unordered_map<u64, std::vector<u32>> by6;
  explicit PairRecover(int n) : N(n), pw6((size_t)n + 1, 0) {
    for (int x = 1; x <= n; ++x) { const u64 x2 = (u64)x * (u64)x; pw6[x] = x2 * x2 * x2; }
    by6.reserve((size_t)n * 2);
    for (int x = 1; x <= n; ++x) by6[pw6[x]].push_back((u32)x);
  }
  void recover(u64 fp, std::vector<std::pair<u32, u32>>& out) const {
    out.clear();
    for (int i = 1; i <= N; ++i) {
      auto it = by6.find(fp - pw6[i]);
      if (it == by6.end()) continue;
      for (u32 j : it->second) if ((u32)i <= j) out.emplace_back((u32)i, j);
    }
  }
};

// Exact T = (base' - (21d)^6 - (14e)^6)/42^6 where base' = B^6-u^6 for real
// units (fourcore_gmp.hpp:55-62) or the planted base.
bool exact_T(const orc_unit5& U, u64 d, u64 e, u128& T) {
  W3 R;
  if (U.planted) {
    R = W3{{U.base[0], U.base[1], U.base[2]}};
  } else {
    if (U.u >= U.B || d < 1 || e < 1) return false;
    R = w3_pow6(U.B);
    if (w3_sub(R, w3_pow6(U.u))) return false;
  }
  if (w3_sub(R, w3_pow6(21 * d))) return false;
  if (w3_sub(R, w3_pow6(14 * e))) return false;
  if (w3_zero(R)) return false;
  if (w3_divmod(R, kM42) != 0) return false;
  if (!w3_fits128(R)) return false;
  T = w3_to128(R);
  return true;
}

}  // namespace

// ============================================================== C API
extern "C" {

size_t orc_unit_candidates(uint64_t B, int cls, uint64_t* out, size_t cap) {
  const auto v = unit_candidates((long long)B, cls);
  for (size_t i = 0; i < v.size() && i < cap; ++i) out[i] = (u64)v[i];
  return v.size();
}
size_t orc_seed_count(uint64_t B, int cls) { return seeds_for_B((long long)B, cls).size(); }
int orc_pack_unit5(uint64_t B, uint64_t u, orc_unit5* out) { return pack_unit5(B, u, *out) ? 1 : 0; }

int orc_free_d_cls234(uint64_t B, uint64_t u, int cls, uint32_t* res, uint32_t* nres,
                      uint64_t* mod, uint64_t* fmax) {
  std::vector<long long> r;
  switch (cls) {  // classes_v3.hpp:188-209
    case 2: r = classes_d_cls2((long long)B); *mod = kM3; *fmax = (B - 1) / 14; break;
    case 3: r = classes_d_cls3((long long)B, (long long)u); *mod = kM2; *fmax = (B - 1) / 21; break;
    case 4: r = classes_d_cls4((long long)B); *mod = kM2 * kM3; *fmax = (B - 1) / 7; break;
    default: return 0;
  }
  *nres = (u32)r.size();
  for (size_t i = 0; i < r.size() && i < 32; ++i) res[i] = (u32)r[i];
  return 1;
}

void orc_pow6_192(uint32_t x, uint64_t out[3]) {
  const W3 w = w3_pow6(x);
  out[0] = w.l[0]; out[1] = w.l[1]; out[2] = w.l[2];
}
int orc_T_peel2(uint64_t B, uint64_t u, uint64_t d, uint64_t e, uint64_t T[2]) {
  orc_unit5 U{}; U.B = B; U.u = u; U.planted = 0;
  u128 t = 0;
  if (!exact_T(U, d, e, t)) return 0;
  T[0] = (u64)t; T[1] = (u64)(t >> 64);
  return 1;
}
uint64_t orc_funnel_fp(const orc_unit5* U, uint32_t d, uint32_t e, int* ok) {
  static const PeelCtx C;
  W3 R{{U->base[0], U->base[1], U->base[2]}};
  *ok = !(w3_sub(R, w3_pow6(14u * e)) || w3_sub(R, w3_pow6(21u * d)));
  return ((R.l[0] >> 6) | (R.l[1] << 58)) * C.inv216;
}
void orc_gate_tables(uint8_t g504[504], uint8_t g247[247]) {
  std::memcpy(g504, gate().g504, 504);
  std::memcpy(g247, gate().g247, 247);
}

uint64_t orc_mix64(uint64_t x) { return mix64(x); }
size_t orc_capacity_for(size_t n) { return capacity_for(n); }
size_t orc_packed_bytes(uint64_t m, uint32_t r) { return packed_bytes(m, r); }

// build_xor (xor_filter.hpp:447-470): sort+unique, then one construction per
// seed try.  The reference frees the key vector after the first incidence
// pass, so a stalled first try ends the call; the same outcome is kept here.
orc_table* orc_build_xor(const uint64_t* keys, size_t n, int r, uint64_t base_seed,
                         int max_seed_tries) {
  if (r <= 0 || r > 64) return nullptr;
  std::vector<u64> k(keys, keys + n);
  std::sort(k.begin(), k.end());
  k.erase(std::unique(k.begin(), k.end()), k.end());
  auto* t = new orc_table();
  for (int i = 0; i < max_seed_tries && i < 1; ++i) {
    if (construct(k, (u32)r, base_seed + (u64)i * kPhi, *t)) return t;
  }
  delete t;
  return nullptr;
}

// xor_build_pairs (fourcore_xor_store.hpp:67-119): keys (i^6+j^6) mod 2^64,
// 1<=i<=j<=N; four outer seed bases base+o*phi.
orc_table* orc_build_pairs(int N, int r) {
  std::vector<u64> pw6((size_t)N + 1, 0);
  for (int x = 1; x <= N; ++x) { const u64 x2 = (u64)x * (u64)x; pw6[x] = x2 * x2 * x2; }
  std::vector<u64> keys;
  keys.reserve((size_t)N * (N + 1) / 2);
  for (int i = 1; i <= N; ++i) for (int j = i; j <= N; ++j) keys.push_back(pw6[i] + pw6[j]);
  for (int o = 0; o < 4; ++o) {
    orc_table* t = orc_build_xor(keys.data(), keys.size(), r, kSeedBase + (u64)o * kPhi, 64);
    if (t) { t->hdr.N = (u32)N; return t; }
  }
  return nullptr;
}

// Shard s of S of the pair-key store: xor_build_pairs over the keys with
// shard_of_key(key, seed, S) == s; the header records shard_count, shard_index
// and shard_mode 0 (key % S after the mix, store_header.hpp:19-21, 33-35).
orc_table* orc_build_pairs_shard(int N, int r, int S, int s, uint64_t seed) {
  std::vector<u64> pw6((size_t)N + 1, 0);
  for (int x = 1; x <= N; ++x) { const u64 x2 = (u64)x * (u64)x; pw6[x] = x2 * x2 * x2; }
  std::vector<u64> keys;
  for (int i = 1; i <= N; ++i)
    for (int j = i; j <= N; ++j) {
      const u64 k = pw6[i] + pw6[j];
      if (shard_of(k, seed, (u32)S) == (u32)s) keys.push_back(k);
    }
  for (int o = 0; o < 4; ++o) {
    orc_table* t = orc_build_xor(keys.data(), keys.size(), r, kSeedBase + (u64)o * kPhi, 64);
    if (t) {
      t->hdr.N = (u32)N;
      t->hdr.shard_count = (u32)S;
      t->hdr.shard_index = (u32)s;
      t->hdr.shard_mode = 0;
      return t;
    }
  }
  return nullptr;
}

// A shard set over parts[0..S) (not owned; each part's header says which
// shard it is; a null part is a shard held elsewhere, whose keys find
// nothing here).  Null unless the parts are shards 0..S-1 of one S.
orc_table* orc_shard_set(const orc_table* const* parts, int S, uint64_t seed) {
  if (S < 1) return nullptr;
  auto* t = new orc_table();
  const orc_table* any = nullptr;
  for (int s = 0; s < S; ++s) {
    t->parts.push_back(parts[s]);
    if (!parts[s]) continue;   // a shard held elsewhere
    any = parts[s];
    const orc_header& h = parts[s]->hdr;
    if ((int)h.shard_count != S || (int)h.shard_index != s || h.shard_mode != 0) {
      delete t;
      return nullptr;
    }
    t->hdr.n_keys += h.n_keys;
    t->hdr.m_cells += h.m_cells;
  }
  if (!any) { delete t; return nullptr; }
  t->hdr.magic = kMagic; t->hdr.version = 2; t->hdr.kind = 1;
  t->hdr.r = any->hdr.r; t->hdr.N = any->hdr.N;
  t->hdr.shard_count = (u32)S;
  t->shard_seed = seed;
  return t;
}

uint32_t orc_shard_of(uint64_t key, uint64_t seed, uint32_t S) { return shard_of(key, seed, S); }

orc_table* orc_load(const char* path, int expected_N) {  // fourcore_xor_store.hpp:147-181
  FILE* f = std::fopen(path, "rb");
  if (!f) return nullptr;
  auto* t = new orc_table();
  bool ok = std::fread(&t->hdr, sizeof t->hdr, 1, f) == 1;
  const orc_header& h = t->hdr;
  ok = ok && h.magic == kMagic && h.version == 2 && h.shard_count >= 1 &&
       h.shard_index < h.shard_count && h.r > 0 && h.r <= 64 && h.kind == 1;
  ok = ok && !(expected_N > 0 && (int)h.N != expected_N);
  if (ok) {
    const size_t want = packed_bytes(h.m_cells, h.r);
    t->packed.assign(want, 0);
    ok = !want || std::fread(t->packed.data(), 1, want, f) == want;
  }
  std::fclose(f);
  if (!ok) { delete t; return nullptr; }
  return t;
}
// A table from a header and its packed bytes already in memory (the
// reference's XorFilter after xor_load_file, without the file).
orc_table* orc_from_memory(const orc_header* h, const uint8_t* bytes, size_t len) {
  if (!h || h->magic != kMagic || h->version != 2 || h->kind != 1 || h->r == 0 || h->r > 64)
    return nullptr;
  if (len != packed_bytes(h->m_cells, h->r)) return nullptr;
  auto* t = new orc_table();
  t->hdr = *h;
  t->packed.assign(bytes, bytes + len);
  return t;
}

int orc_save(const orc_table* t, const char* path) {  // fourcore_xor_store.hpp:126-143
  FILE* f = std::fopen(path, "wb");
  if (!f) return 0;
  bool ok = std::fwrite(&t->hdr, sizeof t->hdr, 1, f) == 1;
  if (ok && !t->packed.empty()) ok = std::fwrite(t->packed.data(), 1, t->packed.size(), f) == t->packed.size();
  std::fclose(f);
  return ok ? 1 : 0;
}
void orc_free(orc_table* t) { delete t; }
void orc_table_header(const orc_table* t, orc_header* h) { *h = t->hdr; }
const uint8_t* orc_table_bytes(const orc_table* t, size_t* n) { *n = t->packed.size(); return t->packed.data(); }

void orc_query(const orc_table* t, const uint64_t* keys, size_t n, uint8_t* out) {
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)n; ++i) out[i] = might_contain(*t, keys[i]) ? 1 : 0;
}
// The filter's residue for each key of a single table: cell(i0) ^ cell(i1) ^
// cell(i2) ^ (h & mask), zero exactly when xor_might_contain answers "maybe"
// (xor_filter.hpp:472-483).  For a non-key every r-bit residue is equally
// likely, so the rate of residues whose low b bits are zero is 2^-b; this
// measures the fingerprint statistics of a wide (r = 48) table, whose
// false-positive rate 2^-48 no sample can reach.
void orc_residue(const orc_table* t, const uint64_t* keys, size_t n, uint64_t* out) {
  const u64 block = t->hdr.m_cells / 3;
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)n; ++i) {
    const u64 h = mix64(keys[i] + t->hdr.mix_seed);
    u64 hs[3]; hashes3(h, block, hs);
    out[i] = load_cell(t->packed.data(), hs[0], t->hdr.r) ^ load_cell(t->packed.data(), hs[1], t->hdr.r) ^
             load_cell(t->packed.data(), hs[2], t->hdr.r) ^ (h & fp_mask(t->hdr.r));
  }
}
// n draws of std::mt19937_64(seed): the non-key stream of the reference's FPR
// test (spike/ribbon/xor_filter_test.cpp:67-75 seeds it with 0xF15EED + n).
void orc_mt64(uint64_t seed, size_t n, uint64_t* out) {
  std::mt19937_64 rng(seed);
  for (size_t i = 0; i < n; ++i) out[i] = rng();
}
int orc_fpr_smoke(const orc_table* t) {  // fourcore_xor_store.hpp:54-65
  if (t->parts.empty() && (t->packed.empty() || t->hdr.m_cells < 3 || t->hdr.r == 0)) return -1;
  int hits = 0;
  u64 x = 0x123456789abcdef0ULL;
  for (int i = 0; i < 200000; ++i) { x = x * kPhi + 1; if (might_contain(*t, x)) ++hits; }
  return hits;
}

size_t orc_cls5_run(const orc_table* t, const orc_unit5* units, size_t n, int use_gate,
                    int threads, orc_hit* hits, size_t cap, uint64_t counters[3]) {
  u64 c0 = 0, c1 = 0, c2 = 0;
  size_t nh = 0;
#ifdef _OPENMP
  const int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt) reduction(+ : c0, c1, c2)
#endif
  for (long long i = 0; i < (long long)n; ++i) {
    u64 ctr[3] = {0, 0, 0};
    std::vector<orc_hit> local;
    peel_unit(*t, units[i], (u32)i, use_gate != 0, ctr, [&](const orc_hit& h) { local.push_back(h); });
    c0 += ctr[0]; c1 += ctr[1]; c2 += ctr[2];
    if (!local.empty()) {
#pragma omp critical(orc_hits)
      {
        for (const auto& h : local) { if (nh < cap) hits[nh] = h; ++nh; }
      }
    }
  }
  counters[0] = c0; counters[1] = c1; counters[2] = c2;
  return nh;
}

// Host verify of raw hits (cls5_gpu_v4.cu:513-542): PairRecover over the
// table's N, a,b <= lim, exact T, p6[a]+p6[b]==T, exact identity, sorted
// distinct terms below B, gcd -> SOLUTION line.  Planted units print a PLANT
// line when base == (21d)^6+(14e)^6+42^6(a^6+b^6) holds exactly.
size_t orc_cls5_verify(const orc_unit5* units, const orc_hit* hits, size_t nh, int N,
                       int stop_first, char* buf, size_t buflen) {
  PairRecover pr(N);
  std::vector<std::pair<u32, u32>> pairs;
  std::string text;
  size_t lines = 0;
  for (size_t k = 0; k < nh; ++k) {
    const orc_hit& H = hits[k];
    const orc_unit5& U = units[H.unit];
    pr.recover(H.fp, pairs);
    for (auto [a, b] : pairs) {
      if (a > U.lim || b > U.lim) continue;
      u128 T = 0;
      if (!exact_T(U, H.d, H.e, T)) continue;
      if (pow6_u128(a) + pow6_u128(b) != T) continue;
      char line[256];
      if (U.planted) {
        W3 rhs = w3_pow6(21ULL * H.d);
        w3_add(rhs, w3_pow6(14ULL * H.e));
        W3 core = w3_u128(pow6_u128(a) + pow6_u128(b));
        w3_add(rhs, w3_mul_u64(core, kM42));
        if (!w3_eq(rhs, W3{{U.base[0], U.base[1], U.base[2]}})) continue;
        std::snprintf(line, sizeof line, "PLANT unit=%u d=%u e=%u c1=%u c2=%u\n", H.unit, H.d, H.e, a, b);
      } else {
        // verify_cls5_gmp (fourcore_gmp.hpp:113-117)
        W3 rhs = w3_pow6(U.u);
        w3_add(rhs, w3_pow6(21ULL * H.d));
        w3_add(rhs, w3_pow6(14ULL * H.e));
        W3 core = w3_u128(pow6_u128(a) + pow6_u128(b));
        w3_add(rhs, w3_mul_u64(core, kM42));
        if (!w3_eq(rhs, w3_pow6(U.B))) continue;
        long long terms[5] = {42LL * a, 42LL * b, 21LL * H.d, 14LL * H.e, (long long)U.u};
        std::sort(terms, terms + 5);
        bool bad = false;
        for (int i = 0; i < 4; ++i) if (terms[i] == terms[i + 1]) bad = true;
        if (bad || terms[4] >= (long long)U.B) continue;
        long long g = terms[0];
        for (int i = 1; i < 5; ++i) g = std::gcd(g, terms[i]);
        g = std::gcd(g, (long long)U.B);
        std::snprintf(line, sizeof line,
                      "SOLUTION cls=5 B=%llu u=%llu a1=%lld a2=%lld a3=%lld a4=%lld a5=%lld gcd=%lld %s\n",
                      (unsigned long long)U.B, (unsigned long long)U.u, terms[0], terms[1], terms[2],
                      terms[3], terms[4], g, g == 1 ? "primitive" : "NON-PRIMITIVE");
      }
      text += line;
      ++lines;
      if (stop_first) break;
    }
    if (stop_first && lines) break;
  }
  if (buf && buflen) {
    const size_t c = std::min(buflen - 1, text.size());
    std::memcpy(buf, text.data(), c);
    buf[c] = 0;
  }
  return lines;
}

// ------------------------------------------------ cls2-4 find3 (config 3)
// expand_unit (fourcore_find_v4.cu:165-205) + make_cand mode 3 (:401-425).
size_t orc_expand_cls234(uint64_t B, uint64_t u, int cls, orc_job3* out, size_t cap) {
  u32 res[32]; u32 nres = 0; u64 mod = 0, fmax = 0;
  if (!orc_free_d_cls234(B, u, cls, res, &nres, &mod, &fmax)) return 0;
  const u64 f = cls == 2 ? 14 : cls == 3 ? 21 : 7;
  const u32 lim = (u32)((B - 1) / 42);
  size_t k = 0;
  if (mod <= 0 || fmax < 1) return 0;
  for (u32 ri = 0; ri < nres; ++ri) {         // for_each_free, classes_v3.hpp:224-232
    for (u64 d = res[ri]; d <= fmax; d += mod) {
      if (d == 0) continue;
      if (u >= B) continue;
      W3 R = w3_pow6(B);
      if (w3_sub(R, w3_pow6(u))) continue;
      if (w3_sub(R, w3_pow6(f * d))) continue;           // compute_T_peel1_gmp
      if (w3_zero(R)) continue;
      if (w3_divmod(R, kM42) != 0 || !w3_fits128(R)) continue;
      const u128 T = w3_to128(R);
      if (T == 0) continue;
      // iroot6_host: double estimate then exact fix-up (find_v4.cu:115-123)
      const double x = std::ldexp((double)(u64)(T >> 64), 64) + (double)(u64)T;
      u64 a = x < 1.0 ? 0 : (u64)std::pow(x, 1.0 / 6.0);
      while (pow6_u128(a + 1) <= T && a < 0xffffffffULL - 2) ++a;
      while (a && pow6_u128(a) > T) --a;
      u32 hi = std::min((u32)a, lim), lo = 1;
      while (lo <= hi && pow6_u128(lo) * 3 < T) ++lo;
      orc_job3 J{};
      J.cls = (u32)cls; J.lim = lim; J.B = B; J.u = u; J.d = d;
      J.T[0] = (u64)T; J.T[1] = (u64)(T >> 64);
      if (lo > hi) { J.lo = 1; J.hi = 0; } else { J.lo = lo; J.hi = hi; }
      if (k < cap) out[k] = J;
      ++k;
    }
  }
  return k;
}

// iroot6_host (fourcore_find_v4.cu:115-123): double estimate then exact fix-up.
static u32 iroot6_find(u128 T) {
  const double x = std::ldexp((double)(u64)(T >> 64), 64) + (double)(u64)T;
  u64 a = x < 1.0 ? 0 : (u64)std::pow(x, 1.0 / 6.0);
  while (pow6_u128(a + 1) <= T && a < 0xffffffffULL - 2) ++a;
  while (a && pow6_u128(a) > T) --a;
  return (u32)a;
}

size_t orc_expand_cls1(uint64_t B, uint64_t u, orc_job3* out, size_t cap) {
  if (u >= B) return 0;                                  // compute_T_gmp (fourcore_gmp.hpp:34-42)
  W3 R = w3_pow6(B);
  if (w3_sub(R, w3_pow6(u)) || w3_zero(R)) return 0;
  if (w3_divmod(R, kM42) != 0 || !w3_fits128(R)) return 0;
  const u128 T = w3_to128(R);
  const u32 lim = (u32)((B - 1) / 42);
  const u32 hi = std::min(iroot6_find(T), lim);          // make_cand mode 4 (:415-419)
  u64 lo = 1;
  while (lo <= hi && pow6_u128(lo) * 4 < T) ++lo;
  if (lo > hi) return 0;                                 // run_batch drops empty windows (:486)
  orc_job3 J{};
  J.cls = 1; J.lim = lim; J.B = B; J.u = u; J.d = 0;
  J.T[0] = (u64)T; J.T[1] = (u64)(T >> 64);
  J.lo = (u32)lo; J.hi = hi;
  if (cap) out[0] = J;
  return 1;
}

size_t orc_find4_run(const orc_table* t, const orc_job3* jobs, size_t n, int use_gate,
                     int ref_tiles, int threads, orc_hit4* hits, size_t cap, uint64_t counters[3]) {
  const Gate& G = gate();
  u64 c0 = 0, c1 = 0, c2 = 0;
  size_t nh = 0;
#ifdef _OPENMP
  const int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt) reduction(+ : c0, c1, c2)
#endif
  for (long long i = 0; i < (long long)n; ++i) {
    const orc_job3& J = jobs[i];
    const u128 T = ((u128)J.T[1] << 64) | J.T[0];
    const u32 t504 = (u32)(T % 504), t247 = (u32)(T % 247);
    std::vector<orc_hit4> local;
    for (u64 c4 = J.lo; c4 <= J.hi; ++c4) {              // k_find4 (:287-338)
      if (c4 < 1 || c4 > J.lim) continue;
      const u64 mult = ref_tiles ? (c4 - J.lo) / 2048 + 1 : 1;
      const u128 c46 = pow6_u128(c4);
      if (c46 >= T) continue;                            // R' <= 0
      const u128 R2 = T - c46;
      u32 hi3 = iroot6_find(R2);
      const u32 capm = J.lim < c4 ? J.lim : (u32)c4;
      if (hi3 > capm) hi3 = capm;
      if (hi3 < 1) continue;
      u32 lo3 = (u32)(hi3 * 0.8);
      if (lo3 < 1) lo3 = 1;
      if (lo3 > hi3) continue;
      const u64 tfp = J.T[0] - (u64)pow6_u128(c4);
      const u32 r4_504 = G.p6504[c4 % 504], r4_247 = G.p6247[c4 % 247];
      for (u64 c3 = lo3; c3 <= hi3; ++c3) {
        c0 += mult;
        if (use_gate) {
          u32 r504 = t504 + 1008 - r4_504 - G.p6504[c3 % 504];
          while (r504 >= 504) r504 -= 504;
          u32 r247 = t247 + 494 - r4_247 - G.p6247[c3 % 247];
          while (r247 >= 247) r247 -= 247;
          if (!(G.g504[r504] && G.g247[r247])) { c1 += mult; continue; }
        }
        c2 += mult;
        const u64 c32 = c3 * c3;
        const u64 fp = tfp - c32 * c32 * c32;
        if (might_contain(*t, fp))
          for (u64 k = 0; k < mult; ++k) local.push_back(orc_hit4{(u32)i, (u32)c3, (u32)c4, 0, fp});
      }
    }
    if (!local.empty()) {
#pragma omp critical(orc_hits4)
      {
        for (const auto& h : local) { if (nh < cap) hits[nh] = h; ++nh; }
      }
    }
  }
  counters[0] = c0; counters[1] = c1; counters[2] = c2;
  return nh;
}

// k_find3 (fourcore_find_v4.cu:255-284) with u64 cell indices (xor_filter.hpp:53-60).
size_t orc_find3_run(const orc_table* t, const orc_job3* jobs, size_t n, int use_gate,
                     int threads, orc_hit3* hits, size_t cap, uint64_t counters[3]) {
  const Gate& G = gate();
  u64 c0 = 0, c1 = 0, c2 = 0;
  size_t nh = 0;
#ifdef _OPENMP
  const int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt) reduction(+ : c0, c1, c2)
#endif
  for (long long i = 0; i < (long long)n; ++i) {
    const orc_job3& J = jobs[i];
    const u128 T = ((u128)J.T[1] << 64) | J.T[0];
    const u32 t504 = (u32)(T % 504), t247 = (u32)(T % 247);
    std::vector<orc_hit3> local;
    for (u64 c3 = J.lo; c3 <= J.hi; ++c3) {
      ++c0;
      if (use_gate) {
        u32 r504 = t504 + 504 - G.p6504[c3 % 504]; if (r504 >= 504) r504 -= 504;
        u32 r247 = t247 + 247 - G.p6247[c3 % 247]; if (r247 >= 247) r247 -= 247;
        if (!(G.g504[r504] && G.g247[r247])) { ++c1; continue; }
      }
      ++c2;
      const u64 c2x = c3 * c3, p6 = c2x * c2x * c2x;
      const u64 fp = J.T[0] - p6;
      if (might_contain(*t, fp)) local.push_back(orc_hit3{(u32)i, (u32)c3, fp});
    }
    if (!local.empty()) {
#pragma omp critical(orc_hits3)
      {
        for (const auto& h : local) { if (nh < cap) hits[nh] = h; ++nh; }
      }
    }
  }
  counters[0] = c0; counters[1] = c1; counters[2] = c2;
  return nh;
}

// ------------------------------------------- reduced-T jobs (find2/3/4)
// T = (B^6 - u^6 - sum of the peeled terms^6) / D^6 as compute_T_gmp /
// compute_T_peel1_gmp / compute_T_peel2_gmp (fourcore_gmp.hpp:34-62):
// false when the difference is not positive, not divisible, or T >= 2^128.
static bool o_job_T(u64 B, u64 u, const u64* terms, int nt, u64 D6, u128* T) {
  if (u >= B) return false;
  W3 R = w3_pow6(B);
  if (w3_sub(R, w3_pow6(u))) return false;
  for (int i = 0; i < nt; ++i)
    if (w3_sub(R, w3_pow6(terms[i]))) return false;
  if (w3_zero(R) || w3_divmod(R, D6) != 0 || !w3_fits128(R)) return false;
  *T = w3_to128(R);
  return true;
}

size_t orc_expand_unit(uint64_t B, uint64_t u, int cls, orc_job* out, size_t cap,
                       uint64_t* fail_t) {
  size_t k = 0;
  u64 fails = 0;
  const u32 lim = (u32)((B - 1) / 42);
  auto push = [&](u64 f1, u64 f2, u128 T) {
    if (T == 0) return;
    orc_job J{};
    J.cls = (u32)cls; J.lim = lim; J.B = B; J.u = u; J.free1 = f1; J.free2 = f2;
    J.T[0] = (u64)T; J.T[1] = (u64)(T >> 64);
    if (k < cap) out[k] = J;
    ++k;
  };
  // for_each_free (classes_v3.hpp:224-232)
  auto each = [](const std::vector<long long>& res, u64 mod, u64 fmax, auto&& fn) {
    if (mod == 0 || fmax < 1) return;
    for (long long r : res)
      for (u64 x = (u64)r; x <= fmax; x += mod)
        if (x) fn(x);
  };
  u128 T = 0;
  if (cls == 1) {
    if (o_job_T(B, u, nullptr, 0, kM42, &T)) push(0, 0, T);   // D = 42 (:172-176)
    else ++fails;
  } else if (cls >= 2 && cls <= 4) {
    u32 res[32]; u32 nres = 0; u64 mod = 0, fmax = 0;
    orc_free_d_cls234(B, u, cls, res, &nres, &mod, &fmax);
    const u64 f = cls == 2 ? 14 : cls == 3 ? 21 : 7;
    std::vector<long long> rv(res, res + nres);
    each(rv, mod, fmax, [&](u64 d) {
      const u64 t1 = f * d;
      if (o_job_T(B, u, &t1, 1, kM42, &T)) push(d, 0, T);
      else ++fails;
    });
  } else if (cls == 5) {                                        // free_de_cls5, e outer (:191-203)
    const auto er = classes_d_cls2((long long)B);
    const auto dr = classes_d_cls3((long long)B, (long long)u);
    each(er, kM3, (B - 1) / 14, [&](u64 e) {
      each(dr, kM2, (B - 1) / 21, [&](u64 d) {
        const u64 t2[2] = {21 * d, 14 * e};
        if (o_job_T(B, u, t2, 2, kM42, &T)) push(d, e, T);
        else ++fails;
      });
    });
  }
  if (fail_t) *fail_t = fails;
  return k;
}

size_t orc_jobs_run(const orc_table* t, const orc_job* jobs, size_t n, int use_gate, int ref_tiles,
                    int threads, orc_hit4* hits, size_t cap, uint64_t counters[3]) {
  const Gate& G = gate();
  std::vector<orc_job3> j3, j4;
  std::vector<u32> i3, i4;
  u64 c[3] = {0, 0, 0};
  size_t nh = 0;
  auto add = [&](u32 job, u32 c3, u32 c4, u64 fp) {
    if (nh < cap) hits[nh] = orc_hit4{job, c3, c4, 0, fp};
    ++nh;
  };
  for (size_t i = 0; i < n; ++i) {
    const orc_job& J = jobs[i];
    const u128 T = ((u128)J.T[1] << 64) | J.T[0];
    if (J.cls == 5) {                                           // k_find2 (:233-252)
      ++c[0];
      if (use_gate && !(G.g504[(u32)(T % 504)] && G.g247[(u32)(T % 247)])) { ++c[1]; continue; }
      ++c[2];
      if (might_contain(*t, J.T[0])) add((u32)i, 0, 0, J.T[0]);
      continue;
    }
    if (J.cls < 1 || J.cls > 4) continue;
    const u32 k = J.cls == 1 ? 4 : 3;                          // make_cand (:401-425)
    const u32 hi = std::min(iroot6_find(T), J.lim);
    u64 lo = 1;
    while (lo <= hi && pow6_u128(lo) * k < T) ++lo;
    if (lo > hi) continue;
    orc_job3 X{};
    X.cls = J.cls; X.lim = J.lim; X.B = J.B; X.u = J.u; X.d = J.free1;
    X.T[0] = J.T[0]; X.T[1] = J.T[1]; X.lo = (u32)lo; X.hi = hi;
    (k == 4 ? j4 : j3).push_back(X);
    (k == 4 ? i4 : i3).push_back((u32)i);
  }
  if (!j3.empty()) {
    std::vector<orc_hit3> h(1 << 20);
    u64 cc[3];
    const size_t m = orc_find3_run(t, j3.data(), j3.size(), use_gate, threads, h.data(), h.size(), cc);
    for (size_t q = 0; q < std::min(m, h.size()); ++q) add(i3[h[q].job], h[q].c3, 0, h[q].fp);
    for (int q = 0; q < 3; ++q) c[q] += cc[q];
  }
  if (!j4.empty()) {
    std::vector<orc_hit4> h(1 << 20);
    u64 cc[3];
    const size_t m = orc_find4_run(t, j4.data(), j4.size(), use_gate, ref_tiles, threads, h.data(),
                                   h.size(), cc);
    for (size_t q = 0; q < std::min(m, h.size()); ++q) add(i4[h[q].job], h[q].c3, h[q].c4, h[q].fp);
    for (int q = 0; q < 3; ++q) c[q] += cc[q];
  }
  for (int q = 0; q < 3; ++q) counters[q] = c[q];
  return nh;
}

size_t orc_jobs_verify(const orc_job* jobs, const orc_hit4* hits, size_t nh, int N, char* buf,
                       size_t buflen, size_t* n_lines) {
  PairRecover pr(N);
  std::vector<std::pair<u32, u32>> pairs;
  std::string text;
  size_t exact = 0, lines = 0;
  for (size_t q = 0; q < nh; ++q) {
    const orc_hit4& H = hits[q];
    const orc_job& J = jobs[H.job];
    const u128 T = ((u128)J.T[1] << 64) | J.T[0];
    pr.recover(H.fp, pairs);
    for (auto [a, b] : pairs) {
      u128 core = pow6_u128(a) + pow6_u128(b);
      W3 rhs = w3_pow6(J.u);
      long long t[5];
      if (J.cls == 5) {                                         // mode 2 (:537-541)
        if (a > J.lim || b > J.lim || core != T) continue;
        w3_add(rhs, w3_pow6(21 * J.free1));                     // verify_cls5_gmp
        w3_add(rhs, w3_pow6(14 * J.free2));
        t[2] = 21LL * (long long)J.free1; t[3] = 14LL * (long long)J.free2;
      } else if (J.cls >= 2 && J.cls <= 4) {                    // mode 3 (:542-547)
        if (H.c3 < 1 || b > H.c3) continue;
        core += pow6_u128(H.c3);
        if (core != T) continue;
        const u64 f = J.cls == 2 ? 14 : J.cls == 3 ? 21 : 7;
        w3_add(rhs, w3_pow6(f * J.free1));                      // verify_cls234_gmp
        t[2] = 42LL * H.c3; t[3] = (long long)(f * J.free1);
      } else {                                                  // mode 4 (:548-554)
        if (H.c3 < 1 || H.c4 < 1 || b > H.c3 || H.c3 > H.c4) continue;
        core += pow6_u128(H.c3) + pow6_u128(H.c4);
        if (core != T) continue;
        t[2] = 42LL * H.c3; t[3] = 42LL * H.c4;                 // verify_fourcore_gmp, D = 42
      }
      ++exact;
      w3_add(rhs, w3_mul_u64(w3_u128(core), kM42));
      if (!w3_eq(rhs, w3_pow6(J.B))) continue;
      t[0] = 42LL * a; t[1] = 42LL * b; t[4] = (long long)J.u;
      std::sort(t, t + 5);                                      // report_solution (:427-457)
      bool bad = false;
      for (int i = 0; i < 4; ++i) if (t[i] == t[i + 1]) bad = true;
      if (bad || t[4] >= (long long)J.B || t[0] < 1) continue;
      long long g = t[0];
      for (int i = 1; i < 5; ++i) g = std::gcd(g, t[i]);
      g = std::gcd(g, (long long)J.B);
      char line[256];
      std::snprintf(line, sizeof line,
                    "SOLUTION cls=%u B=%llu u=%llu a1=%lld a2=%lld a3=%lld a4=%lld a5=%lld gcd=%lld %s\n",
                    J.cls, (unsigned long long)J.B, (unsigned long long)J.u, t[0], t[1], t[2], t[3],
                    t[4], g, g == 1 ? "primitive" : "NON-PRIMITIVE");
      text += line;
      ++lines;
    }
  }
  if (buf && buflen) {
    const size_t m = std::min(text.size(), buflen - 1);
    std::memcpy(buf, text.data(), m);
    buf[m] = 0;
  }
  if (n_lines) *n_lines = lines;
  return exact;
}

}  // extern "C"

// ===================================================== (6,1,7) Branch-A cls5
// Restates solve_617_v1.cu: gen_class_cands(cls=5) (:885-906),
// k_find4_cls5 (:563-657) and verify_hit (:1040-1110).
namespace {

typedef __int128 i128;

// scaled comparisons of solve_617_v1.cu:405-452 in exact u128 arithmetic: a
// product that overflows 128 bits counts as larger than any R.
bool o617_scaled_gt(u128 R, u64 c, u64 scale) {       // scale*c^6 > R
  const u128 c6 = pow6_u128(c);
  if (c6 > (~(u128)0) / scale) return true;
  return c6 * scale > R;
}
bool o617_scaled_lt(u128 R, u64 c, u64 scale) {       // R > scale*c^6
  const u128 c6 = pow6_u128(c);
  if (c6 > (~(u128)0) / scale) return false;
  return R > c6 * scale;
}
// iroot6_fix: largest r with scale*r^6 <= R (double estimate + exact fix-up).
u32 o617_iroot6_fix(u128 R, u64 scale) {
  const double d = (double)(u64)(R >> 64) * 18446744073709551616.0 + (double)(u64)R;
  u64 r = (u64)std::pow(d / (double)scale, 1.0 / 6.0) + 2;
  while (r > 0 && o617_scaled_gt(R, r, scale)) --r;
  while (!o617_scaled_gt(R, r + 1, scale)) ++r;
  return (u32)r;
}
// min_c_fix: least c >= 1 with !(R > 3*scale*c^6).
u32 o617_min_c_fix(u128 R, u32 r_hi, u64 scale) {
  u64 c = (u64)(r_hi * 0.8326831149);
  if (c < 1) c = 1;
  while (o617_scaled_lt(R, c, 3 * scale)) ++c;
  while (c > 1 && !o617_scaled_lt(R, c - 1, 3 * scale)) --c;
  return (u32)c;
}

// {(a^6 + b^6 + c^6) mod m} (build_tri_set, solve_617_v1.cu:334-342).
std::vector<uint8_t> tri_set(int m) {
  std::vector<uint8_t> sp(m, 0), p2(m, 0), p3(m, 0);
  for (int i = 0; i < m; ++i) sp[mod_pow6(i, m)] = 1;
  for (int a = 0; a < m; ++a) if (sp[a]) for (int c = 0; c < m; ++c) if (sp[c]) p2[(a + c) % m] = 1;
  for (int a = 0; a < m; ++a) if (p2[a]) for (int c = 0; c < m; ++c) if (sp[c]) p3[(a + c) % m] = 1;
  return p3;
}

// lift residue classes (mod m) to the values <= maxv (gen_class_cands :815-824).
std::vector<long long> lift617(const std::vector<long long>& res, long long m, long long maxv) {
  std::vector<long long> v;
  for (long long r : res) {
    long long x = r % m;
    if (x == 0) x = m;
    for (; x <= maxv; x += m) v.push_back(x);
  }
  std::sort(v.begin(), v.end());
  return v;
}

// roots of (scale*x)^6 = b6 (mod mod) (scaled_roots, solve_617_v1.cu:217-221).
std::vector<long long> scaled_roots617(const std::vector<std::vector<long long>>& tab, long long b6,
                                       long long scale, long long mod) {
  return tab[b6 * mod_inv(mod_pow6(scale, mod), mod) % mod];
}

}  // namespace

extern "C" {

size_t orc_617_cands(uint64_t B, orc_cand617* out, size_t cap) {
  const Roots& rt = roots();
  const long long lo = 1, hi = (long long)B - 1;
  const u128 B6 = pow6_u128(B);
  const u32 lim = (u32)((B - 1) / 42);
  const auto wres = scaled_roots617(rt.r2, mod_pow6((long long)B, kM2), 21, kM2);
  const auto ures = classes_d_cls2((long long)B);                       // (14u')^6 = B^6 (3^6)
  const auto vres = scaled_roots617(rt.r7, mod_pow6((long long)B, kM7), 6, kM7);  // (6v')^6 = B^6 (7^6)
  size_t k = 0;
  for (long long up : lift617(ures, kM3, ((long long)B - 1) / 14)) {
    const long long u = 14 * up;
    if (u < lo || u > hi) continue;
    const u128 u6 = pow6_u128((u64)u);
    for (long long vp : lift617(vres, kM7, ((long long)B - 1) / 6)) {
      const i128 base = (i128)B6 - (i128)u6 - (i128)pow6_u128((u64)(6 * vp));
      if (base <= 0) continue;
      orc_cand617 C{};
      C.base[0] = (u64)(u128)base; C.base[1] = (u64)((u128)base >> 64);
      C.B = (u32)B; C.u = (u32)u; C.w = (u32)(6 * vp); C.lim = lim;
      C.mod1 = (u32)kM2; C.fmax1 = (u32)((B - 1) / 21);
      C.nres1 = (u32)std::min<size_t>(wres.size(), 24);
      for (u32 i = 0; i < C.nres1; ++i) C.res[i] = (u32)wres[i];
      if (k < cap) out[k] = C;
      ++k;
    }
  }
  return k;
}

size_t orc_617_run(const orc_table* t, const orc_cand617* cands, size_t n, int use_gate,
                   int use_tri, int zmax, int threads, orc_hit617* hits, size_t cap,
                   uint64_t counters[5]) {
  static const PeelCtx PC;
  const Gate& G = gate();
  static const std::vector<uint8_t> t504 = tri_set(504), t247 = tri_set(247);
  u64 c_calls = 0, c_gated = 0, c_tri_tot = 0, c_tri_skip = 0;
  size_t nh = 0;
#ifdef _OPENMP
  const int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt) reduction(+ : c_calls, c_gated, c_tri_tot, c_tri_skip)
#endif
  for (long long ci = 0; ci < (long long)n; ++ci) {
    const orc_cand617& C = cands[ci];
    const u128 base = ((u128)C.base[1] << 64) | C.base[0];
    const u32 kmax = C.fmax1 / C.mod1 + 1;
    std::vector<orc_hit617> local;
    for (u32 tt = 0; tt < C.nres1 * kmax; ++tt) {
      const u32 d = C.res[tt % C.nres1] + (tt / C.nres1) * C.mod1;
      if (d == 0 || d > C.fmax1) continue;
      const i128 Rs = (i128)base - (i128)pow6_u128(21ULL * d);
      if (Rs <= 0) continue;
      const u128 R = (u128)Rs;
      u32 hi4 = o617_iroot6_fix(R, kM42);
      if (hi4 > C.lim) hi4 = C.lim;
      if (hi4 < 1) continue;
      const u32 lo4 = o617_min_c_fix(R, hi4, kM42);
      if (lo4 > hi4) continue;
      // T = R/42^6 residues (once per d, reused per c4)
      const u32 q504 = (u32)((u64)(R % (u128)(504ULL * kM42)) / kM42 % 504);
      const u32 q247 = (u32)((u64)(R % 247) * PC.inv42_247 % 247);
      for (u32 c4 = lo4; c4 <= hi4; ++c4) {
        // visits of this c4 by the reference's c4 tiles of 2048 (gpu_run :960-968)
        const u64 mult = zmax <= 1 ? 1 : std::min<u64>((u64)zmax, (c4 - lo4) / 2048 + 1);
        const u32 t4504 = (q504 + 504 - G.p6504[c4 % 504]) % 504;
        const u32 t4247 = (q247 + 247 - G.p6247[c4 % 247]) % 247;
        if (use_tri) {
          c_tri_tot += mult;
          if (!t504[t4504] || !t247[t4247]) { c_tri_skip += mult; continue; }
        }
        const u128 c6 = pow6_u128(c4);
        if (c6 > (~(u128)0) / kM42) continue;
        const u128 m = c6 * kM42;
        if (m >= R) continue;
        const u128 R2 = R - m;
        u32 hi3 = o617_iroot6_fix(R2, kM42);
        const u32 capm = C.lim < c4 ? C.lim : c4;
        if (hi3 > capm) hi3 = capm;
        if (hi3 < 1) continue;
        const u32 lo3 = o617_min_c_fix(R2, hi3, kM42);
        const u64 tfp = ((u64)R2 >> 6 | (u64)(R2 >> 64) << 58) * PC.inv216;   // funnel_fp
        for (u32 c3 = lo3; c3 <= hi3; ++c3) {
          if (use_gate) {
            const u32 x = (t4504 + 504 - G.p6504[c3 % 504]) % 504;
            const u32 y = (t4247 + 247 - G.p6247[c3 % 247]) % 247;
            if (!(G.g504[x] && G.g247[y])) { c_gated += mult; continue; }
          }
          c_calls += mult;
          const u64 c3_2 = (u64)c3 * c3;
          const u64 key = tfp - c3_2 * c3_2 * c3_2;
          if (might_contain(*t, key))
            for (u64 k = 0; k < mult; ++k) local.push_back(orc_hit617{(u32)ci, 0, 0, c3, c4, d, key});
        }
      }
    }
    if (!local.empty()) {
#pragma omp critical(orc_hits617)
      {
        for (const auto& h : local) { if (nh < cap) hits[nh] = h; ++nh; }
      }
    }
  }
  counters[0] = c_calls; counters[1] = c_gated; counters[2] = 3 * c_calls;
  counters[3] = c_tri_tot; counters[4] = c_tri_skip;
  return nh;
}

size_t orc_617_verify(const orc_cand617* cands, const orc_hit617* hits, size_t nh, int N,
                      int planted, char* buf, size_t buflen, uint64_t stats[2]) {
  u64 n_exact = 0, n_false = 0;
  PairRecover pr(N);
  std::vector<std::pair<u32, u32>> pairs;
  std::vector<std::array<long long, 7>> reported;
  std::string text;
  size_t lines = 0;
  for (size_t k = 0; k < nh; ++k) {
    const orc_hit617& H = hits[k];
    const orc_cand617& C = cands[H.cand];
    const u128 q = ((u128)C.base[1] << 64) | C.base[0];
    pr.recover(H.fp, pairs);
    for (auto [a, b] : pairs) {
      const u128 g6 = pow6_u128(21ULL * H.e);
      bool exact = false;
      if (g6 <= q) {
        const u128 rhs = q - g6;
        exact = rhs % kM42 == 0 &&
                pow6_u128(a) + pow6_u128(b) + pow6_u128(H.c) + pow6_u128(H.d) == rhs / kM42;
      }
      if (!exact) { ++n_false; continue; }
      ++n_exact;
      char line[256];
      if (planted) {
        std::snprintf(line, sizeof line, "PLANT617 cand=%u e=%u a=%u b=%u c=%u d=%u\n", H.cand, H.e,
                      a, b, H.c, H.d);
        text += line;
        ++lines;
        continue;
      }
      std::array<long long, 7> t = {42LL * a, 42LL * b, 42LL * H.c, 42LL * H.d, 21LL * H.e,
                                    (long long)C.u, (long long)C.w};
      std::sort(t.begin(), t.end());
      bool bad = false;
      for (int i = 0; i < 6; ++i) if (t[i] == t[i + 1]) bad = true;
      if (bad || t[6] >= (long long)C.B || t[0] < 1) continue;
      i128 lhs = (i128)pow6_u128(C.B);
      for (long long x : t) { lhs -= (i128)pow6_u128((u64)x); if (lhs < 0) break; }
      if (lhs != 0) continue;
      if (std::find(reported.begin(), reported.end(), t) != reported.end()) continue;
      reported.push_back(t);
      long long g = std::gcd(t[0], t[1]);
      for (int i = 2; i < 7; ++i) g = std::gcd(g, t[i]);
      g = std::gcd(g, (long long)C.B);
      std::snprintf(line, sizeof line,
                    "SOLUTION cls=5 B=%u a1=%lld a2=%lld a3=%lld a4=%lld a5=%lld a6=%lld a7=%lld "
                    "(anchor=%u) gcd=%lld %s\n",
                    C.B, t[0], t[1], t[2], t[3], t[4], t[5], t[6], C.u, g,
                    g == 1 ? "primitive" : "NON-PRIMITIVE");
      text += line;
      ++lines;
    }
  }
  if (stats) { stats[0] = n_exact; stats[1] = n_false; }
  if (buf && buflen) {
    const size_t c = std::min(buflen - 1, text.size());
    std::memcpy(buf, text.data(), c);
    buf[c] = 0;
  }
  return lines;
}

}  // extern "C"

// ================================================ (6,1,7) Branch-A cls 1-4
namespace {

// exact floor sixth root (iroot6_i128, solve_617_v1.cu:192-201)
long long o617_iroot6(i128 n) {
  if (n <= 0) return 0;
  long long lo = 0, hi = 1;
  while ((i128)pow6_u128(hi) <= n) hi <<= 1;
  while (hi - lo > 1) {
    const long long mid = (lo + hi) >> 1;
    if ((i128)pow6_u128(mid) <= n) lo = mid; else hi = mid;
  }
  return lo;
}
// least c >= 1 with k c^6 >= Q (the estimate-and-fix loops of :773-776, :788-791)
long long o617_least(i128 Q, int k) {
  long long c = 1;
  while ((i128)k * (i128)pow6_u128(c) < Q) ++c;
  return c;
}

std::vector<long long> o617_seeds616(long long B, int cls) {   // :267-275
  if (cls == 4) {                                              // classes_d_cls4 (:256-264)
    const Roots& rt = roots();
    const long long t2 = mod_pow6(B, kM2) * mod_inv(mod_pow6(7, kM2), kM2) % kM2;
    const long long t3 = mod_pow6(B, kM3) * mod_inv(mod_pow6(7, kM3), kM3) % kM3;
    std::vector<long long> out;
    for (long long a : rt.r2[t2]) for (long long b : rt.r3[t3]) out.push_back(crt2(a, kM2, b, kM3));
    std::sort(out.begin(), out.end());
    return out;
  }
  return seeds_for_B(B, cls);
}
long long o617_mod616(int cls) {
  return cls == 1 ? 5489031744LL : cls == 2 ? 7529536LL : cls == 3 ? 85766121LL : kM2 * kM3;
}
bool o617_unit_ok616(long long u, int cls) {                   // :282-290
  switch (cls) {
    case 1: return (u & 1) && std::gcd(u, 42LL) == 1;
    case 2: return (u & 1) && (u % 3 == 0);
    case 3: return !(u & 1) && std::gcd(u, 21LL) == 1;
    case 4: return (u % 7 == 0);
  }
  return true;
}

// push_find5_cand + set_window4_gen (:766-803)
void o617_push_find5(orc_job617 J0, i128 Q, long long c5cap, std::vector<orc_job617>& out) {
  long long hi5 = std::min(o617_iroot6(Q), (long long)J0.lim);
  if (hi5 > c5cap) hi5 = c5cap;
  const long long lo5 = o617_least(Q, 5);
  if (lo5 > hi5) return;
  for (long long c5 = lo5; c5 <= hi5; ++c5) {
    const i128 Q4 = Q - (i128)pow6_u128(c5);
    if (Q4 < 4) continue;
    long long hi4 = std::min(o617_iroot6(Q4), (long long)J0.lim);
    if (hi4 > c5) hi4 = c5;
    const long long lo4 = o617_least(Q4, 4);
    if (lo4 > hi4) continue;
    orc_job617 J = J0;
    J.Q4[0] = (u64)(u128)Q4; J.Q4[1] = (u64)((u128)Q4 >> 64);
    J.c5 = (u32)c5; J.lo = (u32)lo4; J.hi = (u32)hi4;
    out.push_back(J);
  }
}

}  // namespace

extern "C" {

size_t orc_617_jobs(uint64_t Bu, int cls, orc_job617* out, size_t cap) {   // :807-884, full band
  const long long B = (long long)Bu;
  const long long lo = 1, hi = B - 1;
  const i128 B6 = (i128)pow6_u128(Bu);
  const u32 lim = (u32)((B - 1) / 42);
  const auto lift = [](const std::vector<long long>& res, long long m, long long maxv) {
    return lift617(res, m, maxv);
  };
  std::vector<long long> uvals;
  if (cls == 4) {
    for (long long x : lift(o617_seeds616(B, 4), kM2 * kM3, (B - 1) / 7)) {
      const long long u = 7 * x;
      if (u >= lo && u <= hi) uvals.push_back(u);
    }
  } else {
    const long long M = o617_mod616(cls);
    for (long long s : o617_seeds616(B, cls)) {
      long long u0 = s % M;
      if (u0 < lo) u0 += (lo - u0 + M - 1) / M * M;
      for (long long u = u0; u <= hi; u += M)
        if (o617_unit_ok616(u, cls)) uvals.push_back(u);
    }
  }
  std::sort(uvals.begin(), uvals.end());
  uvals.erase(std::unique(uvals.begin(), uvals.end()), uvals.end());
  std::vector<orc_job617> jobs;
  for (long long u : uvals) {
    const i128 u6 = (i128)pow6_u128((u64)u);
    if (u6 >= B6) continue;
    orc_job617 J0{};
    J0.B = (u32)B; J0.u = (u32)u; J0.cls = (u32)cls; J0.lim = lim;
    if (cls == 1) {
      const i128 R = B6 - u6;
      if (R % (i128)kM42 != 0) continue;
      const i128 Q0 = R / (i128)kM42;
      const long long wmax = std::min((long long)lim, o617_iroot6(Q0 - 5));
      for (long long w = 1; w <= wmax; ++w) {
        const i128 Q = Q0 - (i128)pow6_u128((u64)w);
        if (Q < 5) break;
        J0.w = (u32)(42 * w);
        o617_push_find5(J0, Q, w, jobs);
      }
    } else {
      long long f, vmod, vmax;
      std::vector<long long> vres;
      if (cls == 2) { f = 14; vres = classes_d_cls2(B); vmod = kM3; vmax = (B - 1) / 14; }
      else if (cls == 3) { f = 21; vres = classes_d_cls3(B, u); vmod = kM2; vmax = (B - 1) / 21; }
      else {
        f = 6;
        vres = roots().r7[mod_pow6(B, kM7) * mod_inv(mod_pow6(6, kM7), kM7) % kM7];
        vmod = kM7; vmax = (B - 1) / 6;
      }
      for (long long v : lift(vres, vmod, vmax)) {
        const i128 R = B6 - u6 - (i128)pow6_u128((u64)(f * v));
        if (R <= 0 || R % (i128)kM42 != 0) continue;
        const i128 Q = R / (i128)kM42;
        if (Q < 5) continue;
        J0.w = (u32)(f * v);
        o617_push_find5(J0, Q, lim, jobs);
      }
    }
  }
  for (size_t i = 0; i < jobs.size() && i < cap; ++i) out[i] = jobs[i];
  return jobs.size();
}

size_t orc_617_find4_run(const orc_table* t, const orc_job617* jobs, size_t n, int use_gate,
                         int use_tri, int ymax, int threads, orc_hit4x* hits, size_t cap,
                         uint64_t counters[5]) {   // k_find4 (:507-560)
  const Gate& G = gate();
  static const std::vector<uint8_t> t504 = tri_set(504), t247 = tri_set(247);
  u64 c_calls = 0, c_gated = 0, c_tri_tot = 0, c_tri_skip = 0;
  size_t nh = 0;
#ifdef _OPENMP
  const int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt) reduction(+ : c_calls, c_gated, c_tri_tot, c_tri_skip)
#endif
  for (long long ci = 0; ci < (long long)n; ++ci) {
    const orc_job617& J = jobs[ci];
    const u128 Q = ((u128)J.Q4[1] << 64) | J.Q4[0];
    const u32 q504 = (u32)(Q % 504), q247 = (u32)(Q % 247);
    std::vector<orc_hit4x> local;
    for (u32 c4 = J.lo; c4 <= J.hi; ++c4) {
      const u64 mult = ymax <= 1 ? 1 : std::min<u64>((u64)ymax, (c4 - J.lo) / 2048 + 1);
      const u32 t4504 = (q504 + 504 - G.p6504[c4 % 504]) % 504;
      const u32 t4247 = (q247 + 247 - G.p6247[c4 % 247]) % 247;
      if (use_tri) {
        c_tri_tot += mult;
        if (!t504[t4504] || !t247[t4247]) { c_tri_skip += mult; continue; }
      }
      const u128 c46 = pow6_u128(c4);
      if (c46 >= Q) continue;
      const u128 R2 = Q - c46;
      u32 hi3 = (u32)o617_iroot6((i128)R2);
      const u32 capm = J.lim < c4 ? J.lim : c4;
      if (hi3 > capm) hi3 = capm;
      if (hi3 < 1) continue;
      const u32 lo3 = (u32)o617_least((i128)R2, 3);
      const u64 tfp = J.Q4[0] - (u64)c46;
      for (u32 c3 = lo3; c3 <= hi3; ++c3) {
        if (use_gate) {
          const u32 x = (t4504 + 504 - G.p6504[c3 % 504]) % 504;
          const u32 y = (t4247 + 247 - G.p6247[c3 % 247]) % 247;
          if (!(G.g504[x] && G.g247[y])) { c_gated += mult; continue; }
        }
        c_calls += mult;
        const u64 c32 = (u64)c3 * c3;
        const u64 key = tfp - c32 * c32 * c32;
        if (might_contain(*t, key))
          for (u64 k = 0; k < mult; ++k) local.push_back(orc_hit4x{(u32)ci, c3, c4, 0, key});
      }
    }
    if (!local.empty()) {
#pragma omp critical(orc_hits4x)
      {
        for (const auto& h : local) { if (nh < cap) hits[nh] = h; ++nh; }
      }
    }
  }
  counters[0] = c_calls; counters[1] = c_gated; counters[2] = 3 * c_calls;
  counters[3] = c_tri_tot; counters[4] = c_tri_skip;
  return nh;
}

size_t orc_617_find4_verify(const orc_job617* jobs, const orc_hit4x* hits, size_t nh, int N,
                            char* buf, size_t buflen, uint64_t stats[2]) {   // verify_hit cls <= 4
  u64 n_exact = 0, n_false = 0;
  PairRecover pr(N);
  std::vector<std::pair<u32, u32>> pairs;
  std::vector<std::array<long long, 7>> reported;
  std::string text;
  size_t lines = 0;
  for (size_t k = 0; k < nh; ++k) {
    const orc_hit4x& H = hits[k];
    const orc_job617& J = jobs[H.job];
    const u128 q = ((u128)J.Q4[1] << 64) | J.Q4[0];
    pr.recover(H.fp, pairs);
    for (auto [a, b] : pairs) {
      if (pow6_u128(a) + pow6_u128(b) + pow6_u128(H.c3) + pow6_u128(H.c4) != q) { ++n_false; continue; }
      ++n_exact;
      std::array<long long, 7> t = {42LL * a, 42LL * b, 42LL * H.c3, 42LL * H.c4, 42LL * J.c5,
                                    (long long)J.w, (long long)J.u};
      std::sort(t.begin(), t.end());
      bool bad = false;
      for (int i = 0; i < 6; ++i) if (t[i] == t[i + 1]) bad = true;
      if (bad || t[6] >= (long long)J.B || t[0] < 1) continue;
      i128 lhs = (i128)pow6_u128(J.B);
      for (long long x : t) { lhs -= (i128)pow6_u128((u64)x); if (lhs < 0) break; }
      if (lhs != 0) continue;
      if (std::find(reported.begin(), reported.end(), t) != reported.end()) continue;
      reported.push_back(t);
      long long g = std::gcd(t[0], t[1]);
      for (int i = 2; i < 7; ++i) g = std::gcd(g, t[i]);
      g = std::gcd(g, (long long)J.B);
      char line[256];
      std::snprintf(line, sizeof line,
                    "SOLUTION cls=%u B=%u a1=%lld a2=%lld a3=%lld a4=%lld a5=%lld a6=%lld a7=%lld "
                    "(anchor=%u) gcd=%lld %s\n",
                    J.cls, J.B, t[0], t[1], t[2], t[3], t[4], t[5], t[6], J.u, g,
                    g == 1 ? "primitive" : "NON-PRIMITIVE");
      text += line;
      ++lines;
    }
  }
  if (stats) { stats[0] = n_exact; stats[1] = n_false; }
  if (buf && buflen) {
    const size_t c = std::min(buflen - 1, text.size());
    std::memcpy(buf, text.data(), c);
    buf[c] = 0;
  }
  return lines;
}

}  // extern "C"
