// cli_617.cpp -- s615_617, a drop-in for solve_617_v1 restricted to what this
// engine builds: Branch A (7 does not divide B), classes 1-5.
//
// Same positional arguments, options, stderr progress lines, stdout SOLUTION
// lines, summary and exit codes as solve_617_v1.cu:1686-2046 for
//   s615_617 B_min B_max [classes] [u_lo] [u_hi] --branch-a-only [options]
// The table is built on the device (or loaded), candidates come from
// s615_617_candidates (class 5) and s615_617_jobs (classes 1-4: the c5
// expansion into find4 jobs), the search is s615_run and the identities
// s615_verify.
// The summary's exact / fp-false counts expand every raw hit into its pairs
// the way expand_xor_hits does (:1019-1036): all i <= j <= N with
// i^6 + j^6 = fp (mod 2^64); exact = pairs that satisfy the identity.
#include <algorithm>
#include <array>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <set>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/s615.h"

namespace {

using Clock = std::chrono::steady_clock;
using u64 = unsigned long long;
using u128 = unsigned __int128;
constexpr long long kHardMax = 2353973;   // B^6 < 2^127 (solve_617_v1.cu:146)
constexpr int kNSoftMax = 120000;         // fourcore_xor_store.hpp:122
constexpr u64 kM42 = 5489031744ULL;

u128 pow6(u64 x) { const u128 a = (u128)x * x; return a * a * a; }

void usage(const char* a0) {
  std::fprintf(stderr,
      "usage: %s <B_min> <B_max> [classes] [u_lo] [u_hi] [options]\n"
      "  (6,1,7): a1^6+..+a7^6 = B^6, primitive; Branch A (7 does not divide B), classes 1-5.\n"
      "  classes: \"all\" (default) or e.g. \"1,3\" (Branch B is not built by this engine);\n"
      "  u band as fractions of B.\n"
      "  options: --branch-a-only (required) --chunk K --device K --r R --hit-cap N\n"
      "           --save-table F --load-table F --bench [K] --quiet\n"
      "           --no-gate --no-tri-gate --check-known [--known-file F]\n"
      "           %s --selftest\n", a0, a0);
}

// PairRecover (fourcore_xor_store.hpp:23-51) for counting expanded records.
struct Pairs {
  int N = 0;
  std::unordered_map<u64, std::vector<unsigned>> by;
  explicit Pairs(int n) : N(n) {
    by.reserve((size_t)n * 2);
    for (unsigned i = 1; i <= (unsigned)n; ++i) by[(u64)pow6(i)].push_back(i);
  }
  template <class F> void each(u64 fp, F f) const {
    for (unsigned i = 1; i <= (unsigned)N; ++i) {
      auto it = by.find(fp - (u64)pow6(i));
      if (it == by.end()) continue;
      for (unsigned j : it->second)
        if (j >= i) f(i, j);
    }
  }
};

struct Known { long long B; };

std::vector<Known> load_known(const char* path) {   // load_known617 (:1259-1276)
  std::vector<Known> out;
  FILE* f = std::fopen(path, "r");
  if (!f) { std::fprintf(stderr, "[check-known] cannot open %s\n", path); return out; }
  char line[512];
  while (std::fgets(line, sizeof line, f)) {
    if (line[0] == '#' || line[0] == '\n') continue;
    long long B = 0;
    if (std::sscanf(line, "%lld", &B) != 1 || B <= 0) continue;
    out.push_back({B});
  }
  std::fclose(f);
  std::fprintf(stderr, "[check-known] loaded %zu entries from %s\n", out.size(), path);
  return out;
}

int check_known(const std::set<long long>& found, const std::vector<Known>& known, long long lo,
                long long hi) {   // check_known_diff (:1277-1301)
  std::set<long long> expect;
  for (const auto& k : known)
    if (k.B >= lo && k.B <= hi) expect.insert(k.B);
  int missing = 0, extra = 0;
  for (long long b : expect)
    if (!found.count(b)) {
      ++missing;
      std::fprintf(stderr, "[check-known] MISSING B=%lld (regression — known solution not recovered!)\n", b);
    }
  for (long long b : found)
    if (!expect.count(b)) {
      ++extra;
      std::fprintf(stderr, "[check-known] *** CANDIDATE NEW B=%lld (not in database — verify independently) ***\n", b);
    }
  std::fprintf(stderr, "[check-known] range [%lld,%lld]: expected=%zu found=%zu missing=%d new-candidates=%d %s\n",
               lo, hi, expect.size(), found.size(), missing, extra,
               missing == 0 ? (extra == 0 ? "PASS" : "PASS (with new candidates)") : "FAIL");
  return missing == 0 ? 0 : 1;
}

// Plants in the shape of the reference's selftest (:1564-1602): base =
// (21d)^6 + 42^6 (c1^6+..+c4^6) with c4 and c3 inside the searched windows.
int selftest(int device) {
  const int hs = s615_selftest_host();
  if (hs) { std::fprintf(stderr, "SELFTEST FAIL (host) check %d\n", hs); return 1; }
  std::fprintf(stderr, "[selftest] host math OK\n");
  s615_ctx* ctx = nullptr;
  if (s615_open(device, 0, &ctx)) {
    std::fprintf(stderr, "[selftest] no GPU — host part only, PASS\n");
    return 0;
  }
  const int N = 4096;
  int tid = 0;
  if (s615_build_table(ctx, N, 48, S615_LAYOUT_AUTO, &tid)) { s615_close(ctx); return 1; }
  std::vector<s615_unit> u;
  std::vector<std::array<unsigned, 5>> want;
  unsigned long long x = 0x617617617ULL;
  auto rnd = [&](unsigned m) { x = x * 6364136223846793005ULL + 1442695040888963407ULL; return (unsigned)((x >> 33) % m); };
  while (u.size() < 256) {
    unsigned c[4];
    for (int k = 0; k < 4; ++k) c[k] = 1 + rnd(N);
    std::sort(c, c + 4);
    if (c[0] == c[1] || c[1] == c[2] || c[2] == c[3]) continue;
    const u128 T = pow6(c[0]) + pow6(c[1]) + pow6(c[2]) + pow6(c[3]);
    if (3 * pow6(c[3]) < T || 3 * pow6(c[2]) < T - pow6(c[3])) continue;
    const unsigned d = 1 + rnd(280);
    const u128 base = pow6(21ULL * d) + (u128)kM42 * T;
    s615_unit p{};
    p.cls = S615_CLS_617; p.kind = 1; p.B = 42ULL * N + 1; p.u = 14; p.w = 6;
    p.base[0] = (u64)base; p.base[1] = (u64)(base >> 64);
    p.fmax1 = d; p.res_d = d % 64; p.lim = N;
    u.push_back(p);
    want.push_back({d, c[0], c[1], c[2], c[3]});
  }
  std::vector<s615_hit> hits(1 << 16);
  size_t nh = 0;
  s615_counters ctr{};
  int s = s615_run(ctx, tid, u.data(), u.size(), 0, hits.data(), hits.size(), &nh, &ctr);
  std::vector<s615_solution> sol(4096);
  size_t ns = 0;
  if (!s) s = s615_verify(ctx, u.data(), u.size(), hits.data(), nh, N, sol.data(), sol.size(), &ns);
  std::vector<char> got(u.size(), 0);
  for (size_t k = 0; k < ns && k < sol.size(); ++k) {
    const s615_solution& S = sol[k];
    unsigned cs[4] = {S.c1, S.c2, S.c3, S.c4};
    std::sort(cs, cs + 4);
    const auto& w = want[S.unit];
    if (S.d == w[0] && cs[0] == w[1] && cs[1] == w[2] && cs[2] == w[3] && cs[3] == w[4]) got[S.unit] = 1;
  }
  int cnt = 0;
  for (char g : got) cnt += g;
  std::fprintf(stderr, "[plant] find4 (cls5 shape): %d/%zu\n", cnt, u.size());
  s615_close(ctx);
  if (s || cnt != (int)u.size()) { std::fprintf(stderr, "SELFTEST FAIL (GPU)\n"); return 1; }
  std::fprintf(stderr, "SELFTEST PASS\n");
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  std::vector<std::string> pos;
  long long chunk = 8192, bench_chunks = 0;
  int device = 0, r = 48;
  size_t hit_cap = 1u << 20;
  std::string save_table, load_table, known_file = "617-solutions-clean.txt";
  bool opt_selftest = false, quiet = false, no_gate = false, no_tri = false, check = false;
  bool branch_a_only = false;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--selftest") opt_selftest = true;
    else if (a == "--quiet") quiet = true;
    else if (a == "--no-gate") no_gate = true;
    else if (a == "--no-tri-gate") no_tri = true;
    else if (a == "--no-defer-gate-load") {}   // a launch-shape option of the reference kernel
    else if (a == "--check-known") check = true;
    else if (a == "--branch-a-only") branch_a_only = true;
    else if (a == "--known-file" && i + 1 < argc) known_file = argv[++i];
    else if (a == "--chunk" && i + 1 < argc) chunk = std::atoll(argv[++i]);
    else if (a == "--device" && i + 1 < argc) device = std::atoi(argv[++i]);
    else if (a == "--r" && i + 1 < argc) r = std::atoi(argv[++i]);
    else if (a == "--hit-cap" && i + 1 < argc) hit_cap = (size_t)std::atol(argv[++i]);
    else if (a == "--save-table" && i + 1 < argc) save_table = argv[++i];
    else if (a == "--load-table" && i + 1 < argc) load_table = argv[++i];
    else if (a == "--bench") bench_chunks = (i + 1 < argc && argv[i + 1][0] != '-') ? std::atoll(argv[++i]) : 4;
    else if (a == "--slots-log2") {
      if (i + 1 < argc && argv[i + 1][0] != '-') ++i;
      std::fprintf(stderr, "[617] --slots-log2 ignored (packed xor replaces OA table)\n");
    }
    else if (a == "--branch-b-only" || a == "--xcheck" || a == "--branch-b-lim") {
      std::fprintf(stderr, "%s: Branch B and --xcheck are not built by this engine\n", a.c_str());
      return 1;
    }
    else if (!a.empty() && a[0] == '-') { std::fprintf(stderr, "unknown option %s\n", a.c_str()); return 1; }
    else pos.push_back(a);
  }
  if (opt_selftest) return selftest(device);
  if (pos.size() < 2 && bench_chunks > 0) { pos.push_back("1"); pos.push_back("10000"); }
  if (pos.size() < 2) { usage(argv[0]); return 1; }
  const long long B_min = std::atoll(pos[0].c_str()), B_max = std::atoll(pos[1].c_str());
  std::vector<int> classes{1, 2, 3, 4, 5};   // the reference's "all" (:1767-1772)
  if (pos.size() >= 3 && pos[2] != "all") {
    classes.clear();
    for (char c : pos[2]) if (c >= '1' && c <= '5') classes.push_back(c - '0');
    if (classes.empty()) classes = {1, 2, 3, 4, 5};
  }
  if (!branch_a_only) {
    std::fprintf(stderr, "Branch B is not built by this engine: pass --branch-a-only\n");
    return 1;
  }
  const double u_lo = pos.size() >= 4 ? std::atof(pos[3].c_str()) : 0.0;
  const double u_hi = pos.size() >= 5 ? std::atof(pos[4].c_str()) : 1.0;
  if (B_max > kHardMax) { std::fprintf(stderr, "B_max capped at %lld (i128: B^6 < 2^127)\n", kHardMax); return 1; }
  if (chunk < 1) chunk = 1;
  std::vector<Known> known;
  if (check) known = load_known(known_file.c_str());

  const int N = (int)(B_max / 42);
  if (N < 4) { std::fprintf(stderr, "B_max too small for Branch A\n"); return 1; }
  s615_ctx* ctx = nullptr;
  if (s615_open(device, 0, &ctx)) { std::fprintf(stderr, "CUDA error: no usable device %d\n", device); return 1; }
  int tid = 0;
  bool loaded = false;
  if (!load_table.empty()) loaded = s615_load_table(ctx, load_table.c_str(), N, S615_LAYOUT_AUTO, &tid) == S615_OK;
  if (!loaded) {
    if (N > kNSoftMax) {
      std::fprintf(stderr, "[617] N=%d > soft max %d (~B=%lld) — raise cap or shard\n", N, kNSoftMax,
                   (long long)kNSoftMax * 42LL);
      s615_close(ctx);
      return 1;
    }
    if (s615_build_table(ctx, N, r, S615_LAYOUT_AUTO, &tid)) {
      std::fprintf(stderr, "[617] FATAL: xor build failed\n");
      s615_close(ctx);
      return 1;
    }
  }
  if (!save_table.empty()) s615_save_table(ctx, tid, save_table.c_str());
  int fpr = 0;
  if (s615_fpr_smoke(ctx, tid, &fpr) || fpr > 8) {
    std::fprintf(stderr, "[617] FATAL: xor FPR smoke too high (%d) — refuse to search\n", fpr);
    s615_close(ctx);
    return 1;
  }
  const Pairs pr(N);
  const unsigned flags = (no_gate ? S615_F_NO_GATE : 0u) | (no_tri ? S615_F_NO_TRI : 0u);
  const size_t kBatchCap = 6000000;   // BRANCH_A_BATCH_CAP (:1896)

  long solutions = 0;
  long long st_cands[6] = {0}, st_exact[6] = {0}, st_false[6] = {0};
  u64 st_probes[6] = {0}, st_calls[6] = {0}, st_gated[6] = {0}, st_tri_skip[6] = {0}, st_tri_tot[6] = {0};
  double st_ms[6] = {0};
  std::set<std::array<long long, 7>> reported;
  std::set<long long> found_B;
  std::vector<s615_hit> hits(hit_cap);
  long long chunks_done = 0;
  int rc = 0;

  for (long long c0 = B_min; c0 <= B_max && !rc; c0 += chunk) {
    const long long c1 = std::min(B_max, c0 + chunk - 1);
    std::vector<long long> Bl;
    for (long long B = std::max(c0, 11LL); B <= c1; ++B)
      if ((B & 1) && B % 3 && B % 7) Bl.push_back(B);
    if (!quiet) std::fprintf(stderr, "[chunk] B %lld..%lld: Branch A (%zu values)\n", c0, c1, Bl.size());
    for (int cls : classes) {
      std::vector<s615_unit> batch;
      auto flush = [&]() -> int {
        if (batch.empty()) return 0;
        size_t nh = 0;
        s615_counters c{};
        const auto t0 = Clock::now();
        int s = s615_run(ctx, tid, batch.data(), batch.size(), flags, hits.data(), hits.size(), &nh, &c);
        st_ms[cls] += std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
        if (s == S615_E_OVERFLOW)
          std::fprintf(stderr, "!! hit buffer overflow at B<=%lld — rerun with larger --hit-cap\n", c1);
        else if (s) { std::fprintf(stderr, "[617] run failed: %s\n", s615_strerror(s)); return 1; }
        st_cands[cls] += (long long)batch.size();
        st_probes[cls] += 3 * c.probes; st_calls[cls] += c.probes; st_gated[cls] += c.gated;
        st_tri_skip[cls] += 32 * c.tri_skipped; st_tri_tot[cls] += 32 * c.tri_total;   // per thread
        const size_t kept = std::min(nh, hits.size());
        for (size_t k = 0; k < kept; ++k) {   // expanded (hit, pair) records, as expand_xor_hits
          const s615_hit& H = hits[k];
          const s615_unit& U = batch[H.unit];
          pr.each(H.fp, [&](unsigned a, unsigned b) {
            bool ex = false;
            if (U.cls == S615_CLS_617_FIND4) {   // the find4 identity against Q4
              const u128 q4 = ((u128)U.base[1] << 64) | U.base[0];
              ex = pow6(a) + pow6(b) + pow6(H.e) + pow6(H.c4) == q4;
            } else {
              const u128 q = pow6(U.B) - pow6(U.u) - pow6(U.w);
              const u128 g6 = pow6(21ULL * H.d);
              if (g6 <= q) {
                const u128 rhs = q - g6;
                ex = rhs % kM42 == 0 && pow6(a) + pow6(b) + pow6(H.e) + pow6(H.c4) == rhs / kM42;
              }
            }
            ex ? ++st_exact[cls] : ++st_false[cls];
          });
        }
        std::vector<s615_solution> sol(4 * kept + 64);
        size_t ns = 0;
        s = s615_verify(ctx, batch.data(), batch.size(), hits.data(), kept, N, sol.data(), sol.size(), &ns);
        if (s) { std::fprintf(stderr, "[617] verify failed: %s\n", s615_strerror(s)); return 1; }
        for (size_t k = 0; k < ns; ++k) {
          const s615_solution& S = sol[k];
          std::array<long long, 7> t;
          for (int i = 0; i < 7; ++i) t[i] = S.a[i];
          if (!reported.insert(t).second) continue;
          const unsigned pcls = S.cls == S615_CLS_617_FIND4 ? S.d : 5u;
          std::printf("SOLUTION cls=%u B=%llu a1=%lld a2=%lld a3=%lld a4=%lld a5=%lld a6=%lld a7=%lld (anchor=%llu) gcd=%lld %s\n",
                      pcls, (u64)S.B, t[0], t[1], t[2], t[3], t[4], t[5], t[6], (u64)S.u, (long long)S.gcd,
                      S.gcd == 1 ? "primitive" : "NON-PRIMITIVE");
          std::fflush(stdout);
          std::fprintf(stderr, "%llu\tSOLUTION\tcls=%u\n", (u64)S.B, pcls);
          ++solutions;
          found_B.insert((long long)S.B);
        }
        batch.clear();
        return 0;
      };
      std::vector<s615_unit> tmp;
      for (long long B : Bl) {
        size_t n = 0;
        if (cls == 5) {
          s615_617_candidates((uint64_t)B, nullptr, 0, &n);
          tmp.resize(n);
          if (n) s615_617_candidates((uint64_t)B, tmp.data(), n, &n);
        } else {
          s615_617_jobs((uint64_t)B, cls, nullptr, 0, &n);
          tmp.resize(n);
          if (n) s615_617_jobs((uint64_t)B, cls, tmp.data(), n, &n);
        }
        const long long lo = std::max(1LL, (long long)(u_lo * B)), hi = std::min(B - 1, (long long)(u_hi * B));
        for (const s615_unit& x : tmp) {
          if ((long long)x.u < lo || (long long)x.u > hi) continue;   // band applies to the u term
          batch.push_back(x);
          if (batch.size() >= kBatchCap && (rc = flush())) break;
        }
        if (rc) break;
      }
      if (!rc) rc = flush();
      if (rc) break;
      if (!quiet && st_cands[cls])
        std::fprintf(stderr, "[chunk] cls%d done: cum cands=%lld probes=%.2e sol=%ld\n", cls, st_cands[cls],
                     (double)st_probes[cls], solutions);
    }
    if (!quiet) {
      std::fprintf(stderr, "B %lld..%lld | cands", c0, c1);
      for (int cls : classes) std::fprintf(stderr, " c%d=%lld", cls, st_cands[cls]);
      std::fprintf(stderr, " | probes");
      for (int cls : classes) std::fprintf(stderr, " c%d=%.2e", cls, (double)st_probes[cls]);
      std::fprintf(stderr, " | sol=%ld\n", solutions);
    }
    if (bench_chunks > 0 && ++chunks_done >= bench_chunks) break;
  }
  s615_close(ctx);
  if (rc) return 1;
  std::fprintf(stderr, "---- summary ----\n");
  for (int cls : classes)
    if (st_cands[cls]) {
      std::fprintf(stderr, "cls%d: cands=%lld probes=%.4e kernel=%.1fs rate=%.2e probes/s exact=%lld fp-false=%lld gate-kill=%.2f%%",
                   cls, st_cands[cls], (double)st_probes[cls], st_ms[cls] / 1e3,
                   st_probes[cls] / std::max(1e-9, st_ms[cls] / 1e3), st_exact[cls], st_false[cls],
                   100.0 * (double)st_gated[cls] / std::max(1.0, (double)(st_gated[cls] + st_calls[cls])));
      if (st_tri_tot[cls])
        std::fprintf(stderr, " tri-skip=%.2f%% (%llu/%llu c4)",
                     100.0 * (double)st_tri_skip[cls] / (double)st_tri_tot[cls], st_tri_skip[cls], st_tri_tot[cls]);
      std::fprintf(stderr, "\n");
    }
  std::fprintf(stderr, "total solutions: %ld (unique B=%zu)\n", solutions, found_B.size());
  if (check && !known.empty()) return check_known(found_B, known, B_min, B_max);
  return 0;
}
