// host_math.cpp -- exact host arithmetic, residue rules and unit records.
//
// The unit rule and free-term residue classes restate
// fourcore_classes_v3.hpp:68-219; unit packing restates pack_unit5
// (fourcore_cls5_gpu_v4.cu:169-184) and adds the divisibility checks the
// device row arithmetic relies on.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "engine.hpp"

namespace s615 {

// ------------------------------------------------------------ 192-bit words
W3 pow6_w3(u64 x) {
  const u128 x2 = (u128)x * x;
  // x < 2^32 keeps x^2 < 2^64; for larger x compute in two steps.
  if ((u64)(x2 >> 64) == 0) {
    const u64 a = (u64)x2;
    const u128 x4 = (u128)a * a;
    const u128 lo = (u128)(u64)x4 * a;
    const u128 hi = (u128)(u64)(x4 >> 64) * a;
    W3 r;
    r.l[0] = (u64)lo;
    const u128 mid = (lo >> 64) + (u128)(u64)hi;
    r.l[1] = (u64)mid;
    r.l[2] = (u64)(hi >> 64) + (u64)(mid >> 64);
    return r;
  }
  W3 r{{1, 0, 0}};
  for (int i = 0; i < 6; ++i) r = mul_w3_u64(r, x);
  return r;
}

bool sub_w3(W3& a, const W3& b) {
  u64 br = 0;
  for (int i = 0; i < 3; ++i) {
    const u128 d = (u128)a.l[i] - b.l[i] - br;
    a.l[i] = (u64)d;
    br = (u64)(d >> 64) ? 1 : 0;
  }
  return br != 0;
}
void add_w3(W3& a, const W3& b) {
  u128 c = 0;
  for (int i = 0; i < 3; ++i) {
    c += (u128)a.l[i] + b.l[i];
    a.l[i] = (u64)c;
    c >>= 64;
  }
}
W3 mul_w3_u64(const W3& a, u64 m) {
  W3 r;
  u128 c = 0;
  for (int i = 0; i < 3; ++i) {
    c += (u128)a.l[i] * m;
    r.l[i] = (u64)c;
    c >>= 64;
  }
  return r;
}
bool zero_w3(const W3& a) { return (a.l[0] | a.l[1] | a.l[2]) == 0; }
bool eq_w3(const W3& a, const W3& b) {
  return a.l[0] == b.l[0] && a.l[1] == b.l[1] && a.l[2] == b.l[2];
}
u64 divmod_w3(W3& a, u64 m) {
  u128 r = 0;
  for (int i = 2; i >= 0; --i) {
    const u128 cur = (r << 64) | a.l[i];
    a.l[i] = (u64)(cur / m);
    r = cur % m;
  }
  return (u64)r;
}
u128 pow6_u128(u64 x) { const u128 a = (u128)x * x; return a * a * a; }
u128 inv_2adic_u128(u128 a) {
  u128 x = a;                       // correct to 3 bits for odd a
  for (int i = 0; i < 7; ++i) x *= (u128)2 - a * x;
  return x;
}

// ------------------------------------------------------------ residue rules
namespace {

long long mod_pow6(long long b, long long m) {
  long long r = 1;
  b %= m; if (b < 0) b += m;
  for (int i = 0; i < 6; ++i) r = (long long)((__int128)r * b % m);
  return r;
}
// Inverse of a modulo m (a coprime to m) by the extended Euclidean algorithm.
long long mod_inv(long long a, long long m) {
  long long r0 = m, r1 = ((a % m) + m) % m, s0 = 0, s1 = 1;
  while (r1) {
    const long long q = r0 / r1;
    long long t = r0 - q * r1; r0 = r1; r1 = t;
    t = s0 - q * s1; s0 = s1; s1 = t;
  }
  s0 %= m;
  return s0 < 0 ? s0 + m : s0;
}
long long crt_pair(long long r1, long long m1, long long r2, long long m2) {
  // m1, m2 coprime
  const long long inv = mod_inv(m1 % m2, m2);
  long long t = ((r2 - r1) % m2 + m2) % m2;
  t = (long long)((__int128)t * inv % m2);
  return r1 + m1 * t;
}

constexpr long long kM2 = 64, kM3 = 729, kM7 = 117649;

// Units a (coprime to the modulus) grouped by a^6 mod the modulus.
struct RootTable {
  std::vector<std::vector<u32>> by;
  explicit RootTable(long long m) : by((size_t)m) {
    for (long long a = 1; a < m; ++a)
      if (std::gcd(a, m) == 1) by[(size_t)mod_pow6(a, m)].push_back((u32)a);
  }
};
const RootTable& roots2() { static RootTable t(kM2); return t; }
const RootTable& roots3() { static RootTable t(kM3); return t; }
const RootTable& roots7() { static RootTable t(kM7); return t; }

bool unit_ok(u64 u, int cls) {
  switch (cls) {
    case 1: return (u & 1) && std::gcd(u, (u64)42) == 1;
    case 2: return (u & 1) && (u % 3 == 0) && (u % 9 != 0);
    case 3: return !(u & 1) && std::gcd(u, (u64)21) == 1;
    case 4: case 5: return (u % 6 == 0) && (u % 7 != 0);
  }
  return false;
}

}  // namespace

// Root lists as CSR arrays for the device: off[t]..off[t+1] index the units a
// with a^6 = t (mod m), ascending.  which: 2, 3 or 7 (moduli 2^6, 3^6, 7^6).
void root_csr(int which, std::vector<u32>& off, std::vector<u32>& roots) {
  const RootTable& t = which == 2 ? roots2() : which == 3 ? roots3() : roots7();
  off.assign(t.by.size() + 1, 0);
  roots.clear();
  for (size_t i = 0; i < t.by.size(); ++i) {
    off[i] = (u32)roots.size();
    roots.insert(roots.end(), t.by[i].begin(), t.by[i].end());
  }
  off[t.by.size()] = (u32)roots.size();
}
u32 inv_pow6_mod(u32 f, u32 m) { return (u32)mod_inv(mod_pow6(f, m), m); }

// (14e)^6 = B^6 (mod 3^6): e in the roots of B^6 * 14^-6.
std::vector<u32> e_residues(u64 B) {
  const long long t = mod_pow6((long long)(B % kM3), kM3) * mod_inv(mod_pow6(14, kM3), kM3) % kM3;
  return roots3().by[(size_t)t];
}
// (21d)^6 = B^6 - u^6 (mod 2^6).
std::vector<u32> d_residues(u64 B, u64 u) {
  long long rhs = (mod_pow6((long long)(B % kM2), kM2) - mod_pow6((long long)(u % kM2), kM2)) % kM2;
  if (rhs < 0) rhs += kM2;
  const long long t = rhs * mod_inv(mod_pow6(21, kM2), kM2) % kM2;
  return roots2().by[(size_t)t];
}

// Stage-1 units for one B over the full band (0,1)*B.
std::vector<u64> unit_candidates(u64 B, int cls) {
  std::vector<u64> out;
  if (B < 2 || cls < 1 || cls > 5) return out;
  const long long b2 = mod_pow6((long long)(B % kM2), kM2);
  const long long b3 = mod_pow6((long long)(B % kM3), kM3);
  const long long b7 = mod_pow6((long long)(B % kM7), kM7);
  std::vector<long long> seeds;
  long long M = kM7;
  const auto& s7 = roots7().by[(size_t)b7];
  if (cls == 1) {
    M = kM2 * kM3 * kM7;
    for (u32 a : roots2().by[(size_t)b2])
      for (u32 c : roots3().by[(size_t)b3]) {
        const long long s23 = crt_pair(a, kM2, c, kM3);
        for (u32 s : s7) seeds.push_back(crt_pair(s23, kM2 * kM3, s, kM7));
      }
  } else if (cls == 2) {
    M = kM2 * kM7;
    for (u32 a : roots2().by[(size_t)b2]) for (u32 s : s7) seeds.push_back(crt_pair(a, kM2, s, kM7));
  } else if (cls == 3) {
    M = kM3 * kM7;
    for (u32 c : roots3().by[(size_t)b3]) for (u32 s : s7) seeds.push_back(crt_pair(c, kM3, s, kM7));
  } else {
    for (u32 s : s7) seeds.push_back(s);
  }
  const u64 lo = 1, hi = B - 1;
  for (long long s : seeds) {
    u64 u = (u64)(s % M);
    if (u < lo) u += (lo - u + (u64)M - 1) / (u64)M * (u64)M;
    for (; u <= hi; u += (u64)M) if (unit_ok(u, cls)) out.push_back(u);
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

// gen_class_cands(cls=5), solve_617_v1.cu:885-906: u = 14u' with (14u')^6 =
// B^6 (mod 3^6) (the e rule of the (6,1,5) search), w = 6v' with (6v')^6 = B^6
// (mod 7^6); residues lifted to every value <= (B-1)/14, (B-1)/6; pairs with
// B^6 - u^6 - w^6 > 0, u ascending then w ascending.
std::vector<std::pair<u64, u64>> candidates617(u64 B) {
  std::vector<std::pair<u64, u64>> out;
  if (B < 2) return out;
  auto lift = [](const std::vector<u32>& res, u64 m, u64 maxv) {
    std::vector<u64> v;
    for (u32 r : res)
      for (u64 x = (r % m) ? r % m : m; x <= maxv; x += m) v.push_back(x);
    std::sort(v.begin(), v.end());
    return v;
  };
  const long long t7 = mod_pow6((long long)(B % kM7), kM7) * mod_inv(mod_pow6(6, kM7), kM7) % kM7;
  const auto us = lift(e_residues(B), (u64)kM3, (B - 1) / 14);
  const auto vs = lift(roots7().by[(size_t)t7], (u64)kM7, (B - 1) / 6);
  const u128 B6 = pow6_u128(B);
  for (u64 up : us) {
    const u64 u = 14 * up;
    if (u < 1 || u > B - 1) continue;
    const u128 u6 = pow6_u128(u);
    for (u64 vp : vs) {
      const u128 w6 = pow6_u128(6 * vp);
      if (u6 < B6 && w6 < B6 - u6) out.emplace_back(u, 6 * vp);
    }
  }
  return out;
}

// ---------------------------------------------- (6,1,7) classes 1-4 jobs
namespace {
using i128 = __int128;

u64 iroot6_i(i128 n) {   // exact floor sixth root, n >= 0
  if (n <= 0) return 0;
  const double x = (double)n;
  u64 a = (u64)std::pow(x, 1.0 / 6.0);
  while ((i128)pow6_u128(a + 1) <= n) ++a;
  while (a && (i128)pow6_u128(a) > n) --a;
  return a;
}
u64 least_k(i128 Q, int k) {   // least c >= 1 with k c^6 >= Q
  u64 c = (u64)std::pow((double)Q / k, 1.0 / 6.0);
  if (c < 1) c = 1;
  while ((i128)k * (i128)pow6_u128(c) < Q) ++c;
  while (c > 1 && (i128)k * (i128)pow6_u128(c - 1) >= Q) --c;
  return c;
}
std::vector<u64> lift_res(const std::vector<long long>& res, u64 m, u64 maxv) {
  std::vector<u64> v;
  for (long long r : res)
    for (u64 x = (u64)r % m ? (u64)r % m : m; x <= maxv; x += m) v.push_back(x);
  std::sort(v.begin(), v.end());
  return v;
}
// the c5 peel and the find4 window of one find5 target (push_find5_cand,
// set_window4_gen: c5 <= c5cap, c4 <= c5, 5 c5^6 >= Q, 4 c4^6 >= Q4)
void push_find5(const s615_unit& J0, i128 Q, u64 c5cap, std::vector<s615_unit>& out) {
  u64 hi5 = std::min<u64>(iroot6_i(Q), J0.lim);
  if (hi5 > c5cap) hi5 = c5cap;
  const u64 lo5 = least_k(Q, 5);
  for (u64 c5 = lo5; c5 <= hi5; ++c5) {
    const i128 Q4 = Q - (i128)pow6_u128(c5);
    if (Q4 < 4) continue;
    u64 hi4 = std::min<u64>(iroot6_i(Q4), J0.lim);
    if (hi4 > c5) hi4 = c5;
    const u64 lo4 = least_k(Q4, 4);
    if (lo4 > hi4) continue;
    s615_unit J = J0;
    J.base[0] = (u64)(u128)Q4;
    J.base[1] = (u64)((u128)Q4 >> 64);
    J.res_e = (u32)c5;
    J.fmax2 = (u32)lo4;
    J.fmax1 = (u32)hi4;
    out.push_back(J);
  }
}
}  // namespace

std::vector<s615_unit> jobs617(u64 B, int cls) {
  std::vector<s615_unit> out;
  if (B < 2 || cls < 1 || cls > 4) return out;
  const i128 B6 = (i128)pow6_u128(B);
  const u32 lim = (u32)((B - 1) / 42);
  const long long b2 = mod_pow6((long long)(B % kM2), kM2), b3 = mod_pow6((long long)(B % kM3), kM3);
  const long long b7 = mod_pow6((long long)(B % kM7), kM7);
  // anchors u (seeds616 / mod616 / unit_ok616, solve_617_v1.cu:267-290,826-848)
  std::vector<u64> us;
  if (cls == 4) {
    const long long t2 = b2 * mod_inv(mod_pow6(7, kM2), kM2) % kM2;
    const long long t3 = b3 * mod_inv(mod_pow6(7, kM3), kM3) % kM3;
    std::vector<long long> xs;
    for (u32 a : roots2().by[(size_t)t2]) for (u32 b : roots3().by[(size_t)t3]) xs.push_back(crt_pair(a, kM2, b, kM3));
    for (u64 x : lift_res(xs, (u64)(kM2 * kM3), (B - 1) / 7)) us.push_back(7 * x);
  } else {
    std::vector<long long> seeds;
    long long M = 0;
    if (cls == 1) {
      M = kM2 * kM3 * kM7;
      for (u32 a : roots2().by[(size_t)b2])
        for (u32 c : roots3().by[(size_t)b3]) {
          const long long s23 = crt_pair(a, kM2, c, kM3);
          for (u32 d : roots7().by[(size_t)b7]) seeds.push_back(crt_pair(s23, kM2 * kM3, d, kM7));
        }
    } else if (cls == 2) {
      M = kM2 * kM7;
      for (u32 a : roots2().by[(size_t)b2]) for (u32 d : roots7().by[(size_t)b7]) seeds.push_back(crt_pair(a, kM2, d, kM7));
    } else {
      M = kM3 * kM7;
      for (u32 c : roots3().by[(size_t)b3]) for (u32 d : roots7().by[(size_t)b7]) seeds.push_back(crt_pair(c, kM3, d, kM7));
    }
    for (long long sd : seeds)
      for (u64 u = (u64)(sd % M) ? (u64)(sd % M) : (u64)M; u <= B - 1; u += (u64)M) {
        const bool ok = cls == 1 ? ((u & 1) && std::gcd(u, (u64)42) == 1)
                      : cls == 2 ? ((u & 1) && u % 3 == 0)
                                 : (!(u & 1) && std::gcd(u, (u64)21) == 1);
        if (ok) us.push_back(u);
      }
  }
  std::sort(us.begin(), us.end());
  us.erase(std::unique(us.begin(), us.end()), us.end());
  for (u64 u : us) {
    const i128 u6 = (i128)pow6_u128(u);
    if (u6 >= B6) continue;
    s615_unit J0{};
    J0.cls = S615_CLS_617_FIND4; J0.kind = 0; J0.B = B; J0.u = u; J0.lim = lim; J0.res_d = (u32)cls;
    if (cls == 1) {   // Q0 = (B^6-u^6)/42^6; the sixth 42-term 42w with c5 <= w
      const i128 R = B6 - u6;
      if (R % (i128)kM42 != 0) continue;
      const i128 Q0 = R / (i128)kM42;
      const u64 wmax = std::min<u64>(lim, iroot6_i(Q0 - 5));
      for (u64 w = 1; w <= wmax; ++w) {
        const i128 Q = Q0 - (i128)pow6_u128(w);
        if (Q < 5) break;
        J0.w = (u32)(42 * w);
        push_find5(J0, Q, w, out);
      }
    } else {          // the sixth term f v over its residue classes
      u64 f = 0, vmod = 0, vmax = 0;
      std::vector<long long> vres;
      if (cls == 2) {
        f = 14; vmod = kM3; vmax = (B - 1) / 14;
        for (u32 v : e_residues(B)) vres.push_back(v);
      } else if (cls == 3) {
        f = 21; vmod = kM2; vmax = (B - 1) / 21;
        for (u32 v : d_residues(B, u)) vres.push_back(v);
      } else {
        f = 6; vmod = kM7; vmax = (B - 1) / 6;
        const long long t = b7 * mod_inv(mod_pow6(6, kM7), kM7) % kM7;
        for (u32 v : roots7().by[(size_t)t]) vres.push_back(v);
      }
      for (u64 v : lift_res(vres, vmod, vmax)) {
        const i128 R = B6 - u6 - (i128)pow6_u128(f * v);
        if (R <= 0 || R % (i128)kM42 != 0) continue;
        const i128 Q = R / (i128)kM42;
        if (Q < 5) continue;
        J0.w = (u32)(f * v);
        push_find5(J0, Q, lim, out);
      }
    }
  }
  return out;
}

// --------------------------------------------------------------- dev units
namespace {
constexpr u64 kMaxB = 40000000ULL;  // keeps d^3, (14e)^3 and the row values inside device words
constexpr u64 kMaxB617 = 2353973ULL; // largest B with B^6 < 2^127 (solve_617_v1.cu B_HARD_MAX)

// base - (14 e0)^6 divisible by 21^6, and V(e0) = d0^6 (mod 64) for every d0:
// then every grid point of the unit has 42^6 | R.
bool divisible_grid5(const W3& base, u32 e0, const u32* d0s, u32 nd) {
  W3 R = base;
  if (sub_w3(R, pow6_w3(14ULL * e0))) return true;  // row has no R>0 point
  if (divmod_w3(R, kM21) != 0) return false;
  for (u32 i = 0; i < nd; ++i) {
    const u64 d0 = d0s[i];
    const u64 d6m = ((d0 * d0 % 64) * (d0 * d0 % 64) % 64) * (d0 * d0 % 64) % 64;
    if ((R.l[0] & 63) != d6m) return false;
  }
  return true;
}

// 42^6 | base - (f d0)^6; every d = d0 (mod mod) then follows (the modulus
// supplies the prime powers that f^6 lacks).
bool divisible_row234(const W3& base, u32 f, u32 d0) {
  W3 R = base;
  if (sub_w3(R, pow6_w3((u64)f * d0))) return true;   // no R>0 row in this class
  return divmod_w3(R, kM42) == 0;
}
}  // namespace

int free_factor(int cls) { return cls == 2 ? 14 : cls == 3 ? 21 : cls == 4 ? 7 : 0; }

// free_d_cls234 (fourcore_classes_v3.hpp:188-209): residues, modulus, fmax.
std::vector<u32> d_residues_cls234(u64 B, u64 u, int cls, u32* mod, u32* fmax) {
  std::vector<u32> r;
  if (cls == 2) {
    const long long t = mod_pow6((long long)(B % kM3), kM3) * mod_inv(mod_pow6(14, kM3), kM3) % kM3;
    r = roots3().by[(size_t)t];
    *mod = (u32)kM3; *fmax = (u32)((B - 1) / 14);
  } else if (cls == 3) {
    r = d_residues(B, u);
    *mod = (u32)kM2; *fmax = (u32)((B - 1) / 21);
  } else if (cls == 4) {
    const long long t2 = mod_pow6((long long)(B % kM2), kM2) * mod_inv(mod_pow6(7, kM2), kM2) % kM2;
    const long long t3 = mod_pow6((long long)(B % kM3), kM3) * mod_inv(mod_pow6(7, kM3), kM3) % kM3;
    for (u32 a : roots2().by[(size_t)t2])
      for (u32 b : roots3().by[(size_t)t3]) r.push_back((u32)crt_pair(a, kM2, b, kM3));
    std::sort(r.begin(), r.end());
    *mod = (u32)(kM2 * kM3); *fmax = (u32)((B - 1) / 7);
  }
  return r;
}

// cls 7: the (6,1,7) class-5 candidate (gen_class_cands, solve_617_v1.cu:
// 885-906).  Every row d then has 42^6 | base - (21d)^6: mod 2^6 by the d
// residues (u, w even), mod 3^6 by u^6 = B^6 (w, 21d divisible by 3), mod 7^6
// by w^6 = B^6 (u, 21d divisible by 7).
static int make_dev_unit617(const s615_unit& in, DevUnit* out, bool* skip) {
  out->cls = S615_CLS_617;
  out->f = 21;
  out->mod1 = (u32)kM2;
  W3 base;
  if (in.kind == 0) {
    const u64 B = in.B, u = in.u, w = in.w;
    if (B < 2 || B > kMaxB617 || u == 0 || w == 0) return S615_E_FORMAT;
    if (u % 14 != 0 || w % 6 != 0) return S615_E_FORMAT;
    if (mod_pow6((long long)(u % kM3), kM3) != mod_pow6((long long)(B % kM3), kM3) ||
        mod_pow6((long long)(w % kM7), kM7) != mod_pow6((long long)(B % kM7), kM7))
      return S615_E_FORMAT;
    if (u >= B || w >= B) { *skip = true; return S615_OK; }
    base = pow6_w3(B);
    sub_w3(base, pow6_w3(u));
    if (sub_w3(base, pow6_w3(w)) || zero_w3(base)) { *skip = true; return S615_OK; }  // base <= 0
    const auto dr = d_residues(B, u);
    if (dr.empty()) { *skip = true; return S615_OK; }
    out->B = B; out->u = u; out->w = (u32)w;
    out->lim = (u32)((B - 1) / 42);
    out->fmax1 = (u32)((B - 1) / 21);
    out->nres1 = (u32)std::min<size_t>(dr.size(), 24);
    for (u32 i = 0; i < out->nres1; ++i) out->res1[i] = dr[i];
  } else if (in.kind == 1) {
    base = W3{{in.base[0], in.base[1], in.base[2]}};
    if (zero_w3(base) || base.l[2] != 0 || (base.l[1] >> 63) != 0) return S615_E_FORMAT;
    if (in.lim >= 65536 || (u64)in.fmax1 * 21 > kMaxB617) return S615_E_FORMAT;
    out->B = in.B; out->u = in.u; out->w = in.w;
    out->lim = in.lim;
    out->fmax1 = in.fmax1;
    out->nres1 = 1;
    out->res1[0] = in.res_d % (u32)kM2;
    if (!divisible_row234(base, 21, out->res1[0])) return S615_E_FORMAT;
  } else {
    return S615_E_FORMAT;
  }
  out->base_lo = base.l[0];
  out->base_hi = base.l[1];
  return S615_OK;
}

// floor(T^(1/6)) and the least c >= 1 with k c^6 >= T, exactly (T < 2^126).
static u32 iroot6_exact(u128 T) {
  const double x = (double)(u64)(T >> 64) * 18446744073709551616.0 + (double)(u64)T;
  u64 a = x < 1.0 ? 0 : (u64)std::pow(x, 1.0 / 6.0);
  while (pow6_u128(a + 1) <= T) ++a;
  while (a && pow6_u128(a) > T) --a;
  return (u32)a;
}
static u32 least_c_k(u128 T, u32 k) {
  const double x = (double)(u64)(T >> 64) * 18446744073709551616.0 + (double)(u64)T;
  u64 c = (u64)std::pow(x / k, 1.0 / 6.0);
  if (c < 1) c = 1;
  while ((u128)k * pow6_u128(c) < T) ++c;
  while (c > 1 && (u128)k * pow6_u128(c - 1) >= T) --c;
  return (u32)c;
}

// cls 1: the find4 unit of fourcore_find_v4 (expand_unit :172-176, make_cand
// mode 4 :415-419): T = (B^6 - u^6)/42^6 exact, c4 window [lo4, hi4] with
// hi4 = min(iroot6(T), lim), lo4 the least c with 4 c^6 >= T; an empty window
// is dropped like run_batch drops it (:486).
static int make_dev_unit1(const s615_unit& in, DevUnit* out, bool* skip) {
  out->cls = 1;
  out->f = 0;
  W3 R;
  u32 lim = 0;
  if (in.kind == 0) {
    const u64 B = in.B, u = in.u;
    if (B < 2 || B > kMaxB || u == 0) return S615_E_FORMAT;
    if (u >= B) { *skip = true; return S615_OK; }
    R = pow6_w3(B);
    sub_w3(R, pow6_w3(u));
    lim = (u32)((B - 1) / 42);
  } else if (in.kind == 1) {
    R = W3{{in.base[0], in.base[1], in.base[2]}};
    if (in.lim >= (1u << 21)) return S615_E_FORMAT;
    lim = in.lim;
  } else {
    return S615_E_FORMAT;
  }
  if (zero_w3(R) || divmod_w3(R, kM42) != 0 || R.l[2] != 0 || (R.l[1] >> 62) != 0)
    return S615_E_FORMAT;   // not a class-1 target, or T outside exact device range
  const u128 T = ((u128)R.l[1] << 64) | R.l[0];
  const u32 hi4 = std::min(iroot6_exact(T), lim);
  const u32 lo4 = least_c_k(T, 4);
  if (hi4 < 1 || lo4 > hi4) { *skip = true; return S615_OK; }
  out->B = in.B; out->u = in.u;
  out->lim = lim;
  out->base_lo = (u64)T;
  out->base_hi = (u64)(T >> 64);
  out->fmax1 = hi4;
  out->fmax2 = lo4;
  out->nres1 = 1;
  return S615_OK;
}

// cls 8: a (6,1,7) class 1-4 find4 job as jobs617 makes it (or a caller's
// own: base = Q4 < 2^126, window inside [1, lim], lim < 2^21).
static int make_dev_unit8(const s615_unit& in, DevUnit* out) {
  if (in.kind != 0 || in.base[2] != 0 || (in.base[1] >> 62) != 0) return S615_E_FORMAT;
  if (in.lim >= (1u << 21) || in.fmax2 < 1 || in.fmax1 < in.fmax2 || in.fmax1 > in.lim)
    return S615_E_FORMAT;
  out->cls = S615_CLS_617_FIND4;
  out->B = in.B; out->u = in.u; out->w = in.w;
  out->base_lo = in.base[0];
  out->base_hi = in.base[1];
  out->lim = in.lim;
  out->fmax1 = in.fmax1;
  out->fmax2 = in.fmax2;
  out->nres1 = 1;
  out->pad1 = in.res_e;   // c5
  out->pad2 = in.res_d;   // the (6,1,7) class
  return S615_OK;
}

// kind 2: one reduced-T job of fourcore_find_v4 (job_from_bin :598-608 with
// make_cand :401-425).  lim defaults to (B-1)/42 and stays <= (kMaxB-1)/42,
// so 3 lim^6 < 2^121 and 4 lim^6 < 2^122: a find3 job with T >= 2^121 or a
// find4 job with T >= 2^122 has an empty window and is dropped, as run_batch
// drops it (:486); other empty find3 windows come out empty on the device.
// cls 2-4: a one-row unit (kClsJobRow) whose row value is T;
// cls 5 (find2): the same row with W = T + 1 and the window [1, 1], so the
// gate tests W - 1^6 = T and the key is T mod 2^64.  When T + 1 >= 2^121, W is
// T + 1 reduced mod 15561 * 2^64 (15561 = 9 * 7 * 13 * 19), which keeps the key
// and every gate residue.  cls 1: the class-1 find4 unit with T given.
static int make_dev_job(const s615_unit& in, DevUnit* out, bool* skip) {
  if (in.cls < 1 || in.cls > 5 || in.base[2] != 0) return S615_E_FORMAT;
  const u128 T = ((u128)in.base[1] << 64) | in.base[0];
  const u64 lim = in.lim ? in.lim : (in.B ? (in.B - 1) / 42 : 0);
  if (lim > (kMaxB - 1) / 42) return S615_E_FORMAT;
  out->B = in.B; out->u = in.u;
  out->lim = (u32)lim;
  if (in.cls == 1) {
    if (T == 0 || (T >> 122) != 0) { *skip = true; return S615_OK; }
    const u32 hi4 = std::min(iroot6_exact(T), (u32)lim);
    const u32 lo4 = least_c_k(T, 4);
    if (hi4 < 1 || lo4 > hi4) { *skip = true; return S615_OK; }
    out->cls = 1;
    out->base_lo = (u64)T;
    out->base_hi = (u64)(T >> 64);
    out->fmax1 = hi4;
    out->fmax2 = lo4;
    out->nres1 = 1;
    return S615_OK;
  }
  u128 W;
  if (in.cls == 5) {
    const u128 M = (u128)15561 << 64;
    W = (T >> 121) == 0 && T + 1 < ((u128)1 << 121) ? T + 1 : (T % M + 1) % M;
    if (W == 0) W = M;
    out->w = 1;
  } else {
    // the device row computes the c3 window; an empty one searches nothing
    if (T == 0 || (T >> 121) != 0) { *skip = true; return S615_OK; }
    W = T;
  }
  out->cls = kClsJobRow;
  out->f = 0;            // row x = 0: the row value is (base >> 6) / 21^6 = W
  out->mod1 = 1;
  out->fmax1 = 1;
  out->nres1 = 1;
  out->res1[0] = 1;
  const u128 base = W * (u128)kM42;   // mod 2^128
  out->base_lo = (u64)base;
  out->base_hi = (u64)(base >> 64);
  return S615_OK;
}

int make_dev_unit(const s615_unit& in, u32 id, DevUnit* out, bool* skip) {
  std::memset(out, 0, sizeof *out);
  *skip = false;
  const u32 cls = in.cls;
  if (in.kind == S615_KIND_JOB) {
    const int s = make_dev_job(in, out, skip);
    out->id = id;
    return s;
  }
  if (cls == S615_CLS_617_FIND4) {
    const int s = make_dev_unit8(in, out);
    out->id = id;
    return s;
  }
  if (cls == 1) {
    const int s = make_dev_unit1(in, out, skip);
    out->id = id;
    return s;
  }
  if (cls == S615_CLS_617) {
    const int s = make_dev_unit617(in, out, skip);
    out->id = id;
    return s;
  }
  if (cls < 2 || cls > 5) return S615_E_FORMAT;
  W3 base;
  out->cls = cls;
  out->f = (u32)free_factor((int)cls);
  if (in.kind == 0) {
    const u64 B = in.B, u = in.u;
    if (B < 2 || B > kMaxB || u == 0) return S615_E_FORMAT;
    if (u >= B) { *skip = true; return S615_OK; }   // base <= 0: the reference drops it
    base = pow6_w3(B);
    sub_w3(base, pow6_w3(u));
    out->B = B; out->u = u;
    out->lim = (u32)((B - 1) / 42);
    if (cls == 5) {
      const auto er = e_residues(B);
      const auto dr = d_residues(B, u);
      if (er.empty() || dr.empty()) { *skip = true; return S615_OK; }
      out->mod1 = kModE;
      out->fmax1 = (u32)((B - 1) / 14);
      out->fmax2 = (u32)((B - 1) / 21);
      out->nres1 = (u32)std::min<size_t>(er.size(), 12);
      out->nres2 = (u32)std::min<size_t>(dr.size(), 12);
      for (u32 i = 0; i < out->nres1; ++i) out->res1[i] = er[i];
      for (u32 i = 0; i < out->nres2; ++i) out->res2[i] = dr[i];
      // With both residue classes non-empty, R = 0 (mod 2^6) holds by the d
      // rule and R = 0 (mod 3^6) by the e rule once 3 | u; R = 0 (mod 7^6)
      // needs u^6 = B^6 (mod 7^6).  Stage-1 units satisfy both
      // (classes_v3.hpp:102-135).
      if (u % 3 != 0 || mod_pow6((long long)(u % kM7), kM7) != mod_pow6((long long)(B % kM7), kM7))
        return S615_E_FORMAT;
    } else {
      u32 mod = 0, fmax = 0;
      const auto dr = d_residues_cls234(B, u, (int)cls, &mod, &fmax);
      if (dr.empty()) { *skip = true; return S615_OK; }
      out->mod1 = mod;
      out->fmax1 = fmax;
      out->nres1 = (u32)std::min<size_t>(dr.size(), 24);
      for (u32 i = 0; i < out->nres1; ++i) out->res1[i] = dr[i];
      for (u32 i = 0; i < out->nres1; ++i)
        if (!divisible_row234(base, out->f, out->res1[i])) return S615_E_FORMAT;
    }
  } else if (in.kind == 1) {
    base = W3{{in.base[0], in.base[1], in.base[2]}};
    // base < 2^152, like a Stage-1 unit's B^6 - u^6 at the largest B (kMaxB^6 < 2^151.6):
    // the row values V = (base - x^6) / 21^6 stay below 2^126
    if (zero_w3(base) || (in.base[2] >> 24) != 0) return S615_E_FORMAT;
    out->B = in.B; out->u = in.u;
    out->lim = in.lim;
    out->nres1 = 1;
    if (cls == 5) {
      if ((u64)in.fmax1 * 14 > kMaxB || (u64)in.fmax2 * 21 > kMaxB) return S615_E_FORMAT;
      out->mod1 = kModE;
      out->fmax1 = in.fmax1; out->fmax2 = in.fmax2;
      out->nres2 = 1;
      out->res1[0] = in.res_e % kModE;
      out->res2[0] = in.res_d % kModD;
      if (!divisible_grid5(base, out->res1[0], out->res2, 1)) return S615_E_FORMAT;
    } else {
      const u32 mod = cls == 2 ? (u32)kM3 : cls == 3 ? (u32)kM2 : (u32)(kM2 * kM3);
      if ((u64)in.fmax1 * out->f > kMaxB) return S615_E_FORMAT;
      out->mod1 = mod;
      out->fmax1 = in.fmax1;
      out->res1[0] = in.res_d % mod;
      if (!divisible_row234(base, out->f, out->res1[0])) return S615_E_FORMAT;
    }
  } else {
    return S615_E_FORMAT;
  }
  out->base_lo = base.l[0];
  out->base_hi = base.l[1];
  out->id = id;
  return S615_OK;
}

// ------------------------------------------------------------ gate patterns
// Admissible values mod q: sums of two sixth powers mod q (the factors of the
// reference's mod-504 and mod-247 bitmaps, fourcore_cls5_gpu_v4.cu:124-137).
static std::vector<u8> pair_sums_mod(u32 q) {
  std::vector<u8> ok(q, 0);
  for (u32 i = 0; i < q; ++i)
    for (u32 j = 0; j < q; ++j) ok[(mod_pow6(i, q) + mod_pow6(j, q)) % q] = 1;
  return ok;
}

// shape 0: cls5 columns, x = s + 64 i, value (W - x^6)/64;
// shape 1: find3 columns, x = s + i, value W - x^6.
void gate_patterns(bool gated, int shape, u32 out[kPatWords]) {
  const u32 step = shape == 0 ? 64 : 1, scale = shape == 0 ? 64 : 1;
  for (int qi = 0; qi < 4; ++qi) {
    const u32 q = (u32)kPatQ[qi];
    const auto ok = pair_sums_mod(q);
    std::vector<u8> okw(q, 0);   // admissible (W - x^6) mod q
    for (u32 t = 0; t < q; ++t) if (ok[t]) okw[(scale * t) % q] = 1;
    for (u32 a = 0; a < q; ++a)
      for (u32 s = 0; s < q; ++s) {
        u32 w = 0;
        for (u32 i = 0; i < 32; ++i) {
          const u32 x = (s + step * i) % q;
          const u32 v = (u32)(((long long)a - mod_pow6(x, q)) % q + q) % q;
          if (!gated || okw[v]) w |= 1u << i;
        }
        out[kPatBase[qi] + a * q + s] = w;
      }
  }
}

// Sharp pattern blocks: for q in kSharpQ, the same construction as
// gate_patterns (shape 0: x = s + 64 i, value (W - x^6)/64; shape 1: x = s + i,
// value W - x^6), always gated.
void gate_patterns_sharp(int shape, u32 out[kSharpWords]) {
  const u32 step = shape == 0 ? 64 : 1, scale = shape == 0 ? 64 : 1;
  for (int qi = 0; qi < 7; ++qi) {
    const u32 q = (u32)kSharpQ[qi];
    const auto ok = pair_sums_mod(q);
    std::vector<u8> okw(q, 0);   // admissible (W - x^6) mod q
    for (u32 t = 0; t < q; ++t) if (ok[t]) okw[(scale * t) % q] = 1;
    for (u32 a = 0; a < q; ++a)
      for (u32 s = 0; s < q; ++s) {
        u32 w = 0;
        for (u32 i = 0; i < 32; ++i) {
          const u32 x = (s + step * i) % q;
          const u32 v = (u32)(((long long)a - mod_pow6(x, q)) % q + q) % q;
          if (okw[v]) w |= 1u << i;
        }
        out[kSharpBase[qi] + a * q + s] = w;
      }
  }
}

u64 pair_sums_mask64() {
  const auto ok = pair_sums_mod(64);
  u64 m = 0;
  for (u32 t = 0; t < 64; ++t) if (ok[t]) m |= 1ULL << t;
  return m;
}

// Triple-sum gate block (build_tri_set, solve_617_v1.cu:334-345): bit x of
// the first bitmap is set iff x = a^6 + b^6 + c^6 (mod 504) for some a, b, c;
// likewise mod 247; then the tables c^6 mod 504 and mod 247 as u16 pairs.
void tri_tables(u32 out[kTriWords]) {
  std::memset(out, 0, kTriWords * sizeof(u32));
  auto tri = [](u32 m, u32* bits) {
    std::vector<u8> sp(m, 0), p2(m, 0);
    for (u32 i = 0; i < m; ++i) sp[(size_t)mod_pow6(i, m)] = 1;
    for (u32 a = 0; a < m; ++a) if (sp[a]) for (u32 c = 0; c < m; ++c) if (sp[c]) p2[(a + c) % m] = 1;
    for (u32 a = 0; a < m; ++a) if (p2[a]) for (u32 c = 0; c < m; ++c) if (sp[c]) {
      const u32 x = (a + c) % m;
      bits[x >> 5] |= 1u << (x & 31);
    }
  };
  tri(504, out + kTriT504);
  tri(247, out + kTriT247);
  u16* p6 = reinterpret_cast<u16*>(out + kTriP504);
  for (u32 c = 0; c < 504; ++c) p6[c] = (u16)mod_pow6(c, 504);
  for (u32 c = 0; c < 247; ++c) p6[504 + c] = (u16)mod_pow6(c, 247);
}

// The reference's bitmaps equal the CRT product of the five factor sets.
bool gate_product_matches() {
  std::vector<u8> g504(504, 0), g247(247, 0);
  for (int i = 0; i < 504; ++i) for (int j = i; j < 504; ++j) g504[(mod_pow6(i, 504) + mod_pow6(j, 504)) % 504] = 1;
  for (int i = 0; i < 247; ++i) for (int j = i; j < 247; ++j) g247[(mod_pow6(i, 247) + mod_pow6(j, 247)) % 247] = 1;
  const auto s8 = pair_sums_mod(8), s9 = pair_sums_mod(9), s7 = pair_sums_mod(7);
  const auto s13 = pair_sums_mod(13), s19 = pair_sums_mod(19);
  int c504 = 0, c247 = 0;
  for (int t = 0; t < 504; ++t) {
    c504 += g504[t];
    if (g504[t] != (s8[t % 8] && s9[t % 9] && s7[t % 7])) return false;
  }
  for (int t = 0; t < 247; ++t) {
    c247 += g247[t];
    if (g247[t] != (s13[t % 13] && s19[t % 19])) return false;
  }
  // admissible T mod 8 must be exactly {0,1,2}: the kernel encodes it as 0x7
  if (!(s8[0] && s8[1] && s8[2]) || s8[3] || s8[4] || s8[5] || s8[6] || s8[7]) return false;
  return c504 == 27 && c247 == 50;
}

}  // namespace s615
