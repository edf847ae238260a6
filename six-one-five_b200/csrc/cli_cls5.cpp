// cli_cls5.cpp -- s615_cls5, a drop-in for fourcore_cls5_gpu_v4.
//
// Same flags, semantics, stdout lines and exit codes as
// fourcore_cls5_gpu_v4.cu:596-709 (usage, argument parsing, --check-table,
// acquire_xor_filter's FATAL paths, the SOLUTION and "---- done" lines).
// Extra flags: --dump-survivors F (one "B u d e fp" line per raw filter hit,
// reference naming: d is the x21 term, e the x14 term), --plain (one unit per
// launch), --layout packed|wide, --batch K (units per device batch),
// --plant COUNT[:SEED] (adds planted targets in the reference's plant shape,
// solve_516_v3.cu:1130-1170, and reports how many were recovered) and
// --serve (reads .buc lines from stdin and runs them through the serving
// loop as they arrive, printing SOLUTION lines as their requests finish) and
// --journal F (a restart journal: every finished chunk or request is
// committed to F with its raw hits and solutions; a rerun with the same F
// prints the recorded SOLUTION lines again and searches only the units that
// are not committed yet).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/s615.h"

namespace {

using Clock = std::chrono::steady_clock;
constexpr int kNSoftMax = 120000;   // fourcore_xor_store.hpp:122
// With pair-space shards each build holds one shard's keys; the set's limit
// is HBM (a packed r=48 set at N = 240,000, B ~ 10.08M, is ~210 GB).
constexpr int kNShardMax = 240000;

void usage() {
  std::printf(
      "usage: s615_cls5 [--selftest-host]\n"
      "   or: s615_cls5 --units FILE.buc [--r BITS]\n"
      "                 [--N K] [--quiet|--no-quiet] [--no-gate]\n"
      "                 [--stop-first] [--device K]\n"
      "                 [--load-table F] [--save-table F]\n"
      "                 [--allow-rebuild] [--dump-survivors F] [--plain]\n"
      "                 [--layout packed|wide] [--batch K] [--plant COUNT[:SEED]]\n"
      "                 [--shards S [--save-shards PREFIX]] [--load-shards F0,F1,..]\n"
      "                 [--journal F]\n"
      "   or: s615_cls5 --serve --N K [--load-table F] [--r BITS] [--batch K]\n"
      "                 [--journal F] < units.buc\n"
      "   or: s615_cls5 --check-table --N K --load-table F\n"
      "                 [--r BITS] [--save-table F] [--allow-rebuild]\n"
      "  --load-table F: packed xor from xor_build_save / --save-table.\n"
      "  --save-table F: write packed xor after build or successful load.\n"
      "  --allow-rebuild: if --load-table fails, build on the device (default: FATAL).\n"
      "  --check-table: load + FPR smoke only.\n"
      "  --shards S: build the table as S pair-space shards (a probe asks only its\n"
      "      key's shard); lifts the soft cap to N <= 240000 as HBM allows.\n"
      "  --journal F: commit finished units to F; a rerun resumes from it.\n");
}

int selftest_host() {
  std::printf("[selftest-host] cls5 engine (row identity, gate factors, exact remainder)\n");
  const int s = s615_selftest_host();
  if (s != 0) {
    std::printf("FAIL check %d\n", s);
    return 1;
  }
  std::printf("[selftest-host] PASS\n");
  return 0;
}

struct Line { int cls; unsigned long long B, u; };

using u64 = unsigned long long;
using u128 = unsigned __int128;
struct W3 { u64 l[3]; };
W3 pow6_w3(u64 x) {   // x < 2^32
  const u128 x2 = (u128)x * x, x4 = x2 * x2;
  const u128 lo = (u128)(u64)x4 * (u64)x2, hi = (u128)(u64)(x4 >> 64) * (u64)x2;
  const u128 mid = (lo >> 64) + (u128)(u64)hi;
  return W3{{(u64)lo, (u64)mid, (u64)(hi >> 64) + (u64)(mid >> 64)}};
}
void add_w3(W3& a, const W3& b) {
  u128 c = 0;
  for (int i = 0; i < 3; ++i) { c += (u128)a.l[i] + b.l[i]; a.l[i] = (u64)c; c >>= 64; }
}
W3 mul_w3(const W3& a, u64 m) {
  W3 r;
  u128 c = 0;
  for (int i = 0; i < 3; ++i) { c += (u128)a.l[i] * m; r.l[i] = (u64)c; c >>= 64; }
  return r;
}

// Planted class-5 targets: base = (14e)^6 + (21d)^6 + 42^6 (c1^6 + c2^6), one
// residue per axis and fmax = the planted value, c1 < c2 <= N.
struct Plant { unsigned e, d, c1, c2; };
std::vector<Plant> make_plants(int count, u64 seed, u64 B_max, int N, std::vector<s615_unit>& out) {
  std::vector<Plant> ps;
  u64 x = seed * 0x9E3779B97F4A7C15ULL + 615;
  auto rnd = [&](u64 m) { x = x * 6364136223846793005ULL + 1442695040888963407ULL; return (x >> 17) % m; };
  while ((int)ps.size() < count) {
    Plant p;
    p.e = 1 + (unsigned)rnd((B_max - 1) / 14);
    p.d = 1 + (unsigned)rnd((B_max - 1) / 21);
    p.c1 = 1 + (unsigned)rnd(N);
    p.c2 = 1 + (unsigned)rnd(N);
    if (p.c1 >= p.c2) continue;
    W3 base = pow6_w3(14ULL * p.e);
    add_w3(base, pow6_w3(21ULL * p.d));
    W3 core = pow6_w3(p.c1);
    add_w3(core, pow6_w3(p.c2));
    add_w3(base, mul_w3(core, 5489031744ULL));   // 42^6
    s615_unit U{};
    U.cls = 5; U.kind = 1;
    for (int i = 0; i < 3; ++i) U.base[i] = base.l[i];
    U.fmax1 = p.e; U.fmax2 = p.d; U.res_e = p.e % 729; U.res_d = p.d % 64; U.lim = (unsigned)N;
    if (s615_unit_status(&U) != S615_OK) continue;
    out.push_back(U);
    ps.push_back(p);
  }
  return ps;
}

void print_solution(const s615_solution& S) {   // fourcore_cls5_gpu_v4.cu:533-536
  std::printf("SOLUTION cls=5 B=%llu u=%llu a1=%lld a2=%lld a3=%lld a4=%lld a5=%lld gcd=%lld %s\n",
              (unsigned long long)S.B, (unsigned long long)S.u, (long long)S.a[0], (long long)S.a[1],
              (long long)S.a[2], (long long)S.a[3], (long long)S.a[4], (long long)S.gcd,
              S.gcd == 1 ? "primitive" : "NON-PRIMITIVE");
}

// Opens the journal and reports what it holds; nullptr (with a message) on error.
s615_journal* open_journal(const std::string& path) {
  s615_journal* j = nullptr;
  const int s = s615_journal_open(path.c_str(), &j);
  if (s) {
    std::fprintf(stderr, "[journal] cannot open %s: %s\n", path.c_str(), s615_strerror(s));
    return nullptr;
  }
  size_t nu = 0, nh = 0, ns = 0;
  s615_journal_stats(j, &nu, &nh, &ns);
  std::fprintf(stderr, "[journal] %s: %zu committed units, %zu raw hits, %zu solutions\n", path.c_str(),
               nu, nh, ns);
  return j;
}

// The journal's recorded solutions of kind 0, printed again (a resumed run's
// stdout then holds every SOLUTION line of the campaign); returns how many.
unsigned long long replay_solutions(s615_journal* j) {
  size_t n = 0;
  s615_journal_solutions(j, nullptr, 0, &n);
  std::vector<s615_solution> v(n);
  if (n) s615_journal_solutions(j, v.data(), v.size(), &n);
  unsigned long long k = 0;
  for (const s615_solution& S : v)
    if (S.kind == 0) { print_solution(S); ++k; }
  return k;
}

bool load_buc5(const char* path, std::vector<Line>& out) {  // fourcore_cls5_gpu_v4.cu:155-167
  FILE* f = std::fopen(path, "r");
  if (!f) return false;
  char buf[256];
  while (std::fgets(buf, sizeof buf, f)) {
    int cls;
    unsigned long long B, u;
    if (std::sscanf(buf, "%d %llu %llu", &cls, &B, &u) != 3) continue;
    if (cls != 5) continue;
    out.push_back({cls, B, u});
  }
  std::fclose(f);
  return !out.empty();
}

std::vector<std::string> split_commas(const std::string& v) {
  std::vector<std::string> out;
  size_t a = 0;
  while (a <= v.size()) {
    const size_t b = v.find(',', a);
    const std::string part = v.substr(a, b == std::string::npos ? std::string::npos : b - a);
    if (!part.empty()) out.push_back(part);
    if (b == std::string::npos) break;
    a = b + 1;
  }
  return out;
}

// A pair-space shard set: loaded from its shard files in order, or built on
// the device one shard at a time (and saved as <prefix>.shard<k>of<S>).
bool acquire_shards(s615_ctx* ctx, int N, int r, int shards, const std::string& load,
                    const std::string& save_prefix, int layout, int& tid) {
  int s = 0;
  if (!load.empty()) {
    const auto files = split_commas(load);
    std::vector<const char*> paths;
    for (const auto& f : files) paths.push_back(f.c_str());
    s = s615_load_table_shards(ctx, paths.data(), (int)paths.size(), N, layout, &tid);
    if (s) {
      std::fprintf(stderr, "[cls5-gpu] FATAL: --load-shards: %s\n", s615_strerror(s));
      return false;
    }
  } else {
    s = s615_build_table_sharded(ctx, N, r, shards, layout, &tid);
    if (s) {
      std::fprintf(stderr, "[cls5-gpu] FATAL: sharded xor build failed: %s\n", s615_strerror(s));
      return false;
    }
  }
  s615_table_info info;
  s615_get_table_info(ctx, tid, &info);
  std::fprintf(stderr, "[xor] N=%u keys=%llu cells=%llu r=%u in %u pair-space shards (%.2f GB in HBM)\n",
               info.hdr.N, (unsigned long long)info.hdr.n_keys, (unsigned long long)info.hdr.m_cells,
               info.hdr.r, info.hdr.shard_count, info.device_bytes / 1e9);
  if (!save_prefix.empty()) {
    for (unsigned k = 0; k < info.hdr.shard_count; ++k) {
      const std::string path = save_prefix + ".shard" + std::to_string(k) + "of" +
                               std::to_string(info.hdr.shard_count);
      if ((s = s615_save_table_shard(ctx, tid, (int)k, path.c_str()))) {
        std::fprintf(stderr, "[xor] cannot save %s: %s\n", path.c_str(), s615_strerror(s));
        return false;
      }
      std::fprintf(stderr, "[xor] saved %s\n", path.c_str());
    }
  }
  return true;
}

// acquire_xor_filter (fourcore_cls5_gpu_v4.cu:568-594) on the device.
bool acquire(s615_ctx* ctx, int N, int& r, const std::string& load, const std::string& save,
             bool allow_rebuild, int layout, int& tid) {
  bool loaded = false;
  if (!load.empty()) {
    const int s = s615_load_table(ctx, load.c_str(), N, layout, &tid);
    if (s == S615_E_FPR_SMOKE) {
      std::fprintf(stderr, "[cls5-gpu] FATAL: xor FPR smoke too high — refuse to search\n");
      return false;
    }
    loaded = s == S615_OK;
    if (!loaded) {
      std::fprintf(stderr, "[xor] cannot use %s: %s\n", load.c_str(), s615_strerror(s));
      if (!allow_rebuild) {
        std::fprintf(stderr,
                     "[cls5-gpu] FATAL: --load-table failed (see [xor] lines above). Fix N/path, or "
                     "pass --allow-rebuild to build the table on the device.\n");
        return false;
      }
      std::fprintf(stderr, "[cls5-gpu] --load-table failed; --allow-rebuild: building xor on device...\n");
    }
  }
  if (!loaded) {
    const int s = s615_build_table(ctx, N, r, layout, &tid);
    if (s) {
      std::fprintf(stderr, "[cls5-gpu] FATAL: xor build failed: %s\n", s615_strerror(s));
      return false;
    }
  }
  s615_table_info info;
  s615_get_table_info(ctx, tid, &info);
  r = (int)info.hdr.r;
  std::fprintf(stderr, "[xor] N=%u keys=%llu cells=%llu r=%u seed=0x%llx (%.2f GB in HBM)\n",
               info.hdr.N, (unsigned long long)info.hdr.n_keys, (unsigned long long)info.hdr.m_cells,
               info.hdr.r, (unsigned long long)info.hdr.mix_seed, info.device_bytes / 1e9);
  if (!save.empty()) {
    const int s = s615_save_table(ctx, tid, save.c_str());
    if (s) {
      std::fprintf(stderr, "[xor] cannot save %s: %s\n", save.c_str(), s615_strerror(s));
      return false;
    }
    std::fprintf(stderr, "[xor] saved %s\n", save.c_str());
  }
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  std::setvbuf(stdout, nullptr, _IOLBF, 0);
  std::setvbuf(stderr, nullptr, _IOLBF, 0);
  std::string units_path, load_table, save_table, dump_path, load_shards, save_shards, journal_path;
  int device = 0, N_override = 0, xor_r = 48, layout = S615_LAYOUT_AUTO, shards = 1;
  size_t batch = 1 << 16;
  bool do_host = false, quiet = true, use_gate = true, stop_first = false;
  bool allow_rebuild = false, check_table = false, plain = false, serve = false;
  int plant_count = 0;
  u64 plant_seed = 0;
  for (int i = 1; i < argc; ++i) {
    const std::string s = argv[i];
    auto next = [&]() { return (i + 1 < argc) ? std::string(argv[++i]) : std::string(); };
    if (s == "--selftest-host") do_host = true;
    else if (s == "--units") units_path = next();
    else if (s == "--max-table-gb") (void)next();   // accepted and ignored, like the reference
    else if (s == "--S") (void)next();              // accepted and ignored, like the reference
    else if (s == "--r") xor_r = std::atoi(next().c_str());
    else if (s == "--N") N_override = std::atoi(next().c_str());
    else if (s == "--quiet") quiet = true;
    else if (s == "--no-quiet") quiet = false;
    else if (s == "--no-gate") use_gate = false;
    else if (s == "--stop-first") stop_first = true;
    else if (s == "--device") device = std::atoi(next().c_str());
    else if (s == "--load-table") load_table = next();
    else if (s == "--save-table") save_table = next();
    else if (s == "--allow-rebuild") allow_rebuild = true;
    else if (s == "--shards") shards = std::atoi(next().c_str());
    else if (s == "--load-shards") load_shards = next();
    else if (s == "--save-shards") save_shards = next();
    else if (s == "--check-table") check_table = true;
    else if (s == "--dump-survivors") dump_path = next();
    else if (s == "--plain") plain = true;
    else if (s == "--serve") serve = true;
    else if (s == "--journal") journal_path = next();
    else if (s == "--plant") {
      const std::string v = next();
      plant_count = std::atoi(v.c_str());
      const size_t c = v.find(':');
      if (c != std::string::npos) plant_seed = std::strtoull(v.c_str() + c + 1, nullptr, 10);
    }
    else if (s == "--batch") batch = (size_t)std::max(1, std::atoi(next().c_str()));
    else if (s == "--layout") {
      const std::string v = next();
      layout = v == "packed" ? S615_LAYOUT_PACKED : v == "wide" ? S615_LAYOUT_WIDE : S615_LAYOUT_AUTO;
    } else if (s == "-h" || s == "--help") { usage(); return 0; }
    else { std::fprintf(stderr, "unknown %s\n", s.c_str()); usage(); return 1; }
  }
  if (do_host || argc == 1) return selftest_host();
  if (xor_r < 8 || xor_r > 64) { std::fprintf(stderr, "--r must be 8..64\n"); return 1; }
  if (!load_shards.empty()) shards = std::max<int>(2, (int)split_commas(load_shards).size());
  if (shards != 1 && (shards < 2 || shards > 64)) {
    std::fprintf(stderr, "--shards must be 2..64\n");
    return 1;
  }
  const int n_cap = shards > 1 ? kNShardMax : kNSoftMax;
  auto get_table = [&](s615_ctx* c, int N, int& r, int& tid) {
    if (shards > 1) return acquire_shards(c, N, r, shards, load_shards, save_shards, layout, tid);
    return acquire(c, N, r, load_table, save_table, allow_rebuild, layout, tid);
  };

  if (check_table) {
    if (N_override <= 0) { std::fprintf(stderr, "--check-table needs --N\n"); return 1; }
    if (N_override > n_cap) {
      std::fprintf(stderr, "N=%d exceeds soft xor cap %d\n", N_override, n_cap);
      return 1;
    }
  } else if (serve) {
    if (N_override <= 0) { std::fprintf(stderr, "--serve needs --N\n"); return 1; }
  } else if (units_path.empty()) {
    usage();
    return 1;
  }

  s615_ctx* ctx = nullptr;
  int s = s615_open(device, 0, &ctx);
  if (s) { std::fprintf(stderr, "CUDA device %d: %s\n", device, s615_strerror(s)); return 1; }
  size_t free_b = 0, total_b = 0;
  s615_mem_info(ctx, &free_b, &total_b);
  std::fprintf(stderr, "[cls5-gpu] device=%d free=%.1f / total=%.1f GB\n", device, free_b / 1e9,
               total_b / 1e9);

  if (check_table) {
    int tid = 0;
    if (!get_table(ctx, N_override, xor_r, tid)) {
      s615_close(ctx);
      return 1;
    }
    s615_table_info info;
    s615_get_table_info(ctx, tid, &info);
    std::fprintf(stderr, "[cls5-gpu] --check-table OK N=%d r=%d packed=%.3f GB\n", N_override, xor_r,
                 (double)(info.hdr.m_cells * info.hdr.r / 8 + 8) / 1e9);
    s615_close(ctx);
    return 0;
  }

  if (serve) {   // units stream in on stdin; one request per --batch lines (or at EOF)
    int tid = 0;
    if (!get_table(ctx, N_override, xor_r, tid)) {
      s615_close(ctx);
      return 1;
    }
    const unsigned flags = use_gate ? 0u : S615_F_NO_GATE;
    if ((s = s615_serve_start(ctx, 2, 0))) {
      std::fprintf(stderr, "[cls5-gpu] serve: %s\n", s615_strerror(s));
      s615_close(ctx);
      return 1;
    }
    std::vector<s615_unit> pend;
    size_t submitted = 0, finished = 0, n_units = 0, resumed = 0;
    unsigned long long sols = 0, calls = 0, probes = 0;
    std::vector<s615_result> res(64);
    s615_journal* jr = nullptr;
    std::map<uint64_t, std::vector<s615_unit>> inflight;   // ticket -> units (journal)
    bool jfail = false;
    if (!journal_path.empty()) {
      if (!(jr = open_journal(journal_path))) {
        s615_serve_stop(ctx);
        s615_close(ctx);
        return 1;
      }
      sols += replay_solutions(jr);
    }
    auto drain = [&](int wait_ms) {
      size_t k = 0;
      s615_poll(ctx, res.data(), res.size(), &k, wait_ms);
      for (size_t i = 0; i < k; ++i) {
        const s615_result& R = res[i];
        if (R.status) std::fprintf(stderr, "[cls5-gpu] request %llu: %s\n", (u64)R.ticket, s615_strerror(R.status));
        for (u64 j = 0; j < R.n_solutions; ++j) {
          const s615_solution& S = R.solutions[j];
          if (S.kind != 0) continue;
          print_solution(S);
          ++sols;
        }
        if (jr && R.status == S615_OK) {   // commit the request once it is reported
          const auto& us = inflight[R.ticket];
          if (s615_journal_append(jr, us.data(), us.size(), R.hits, R.n_hits, R.solutions,
                                  R.n_solutions) != S615_OK) {
            std::fprintf(stderr, "[journal] append failed\n");
            jfail = true;
          }
        }
        inflight.erase(R.ticket);
        if (!quiet)
          std::fprintf(stderr, "[cls5-gpu] request %llu: %llu units, %.1f ms\n", (u64)R.ticket,
                       (u64)R.n_units, R.latency_ms);
        s615_release(ctx, R.ticket);
        ++finished;
      }
    };
    auto submit = [&]() {
      if (pend.empty()) return;
      uint64_t t = 0;
      if (s615_submit(ctx, tid, pend.data(), pend.size(), flags, &t) == S615_OK) {
        ++submitted;
        if (jr) inflight[t] = pend;
      }
      n_units += pend.size();
      pend.clear();
    };
    const auto t0 = Clock::now();
    char buf[256];
    while (std::fgets(buf, sizeof buf, stdin)) {
      int cls;
      u64 B, u;
      if (std::sscanf(buf, "%d %llu %llu", &cls, &B, &u) != 3 || cls != 5) continue;
      s615_unit U{};
      U.cls = 5; U.B = B; U.u = u;
      if (s615_unit_status(&U) != S615_OK) continue;
      if (jr && s615_journal_has(jr, &U) == 1) { ++resumed; continue; }
      pend.push_back(U);
      if (pend.size() >= batch) submit();
      drain(0);
    }
    submit();
    while (finished < submitted) drain(100);
    s615_serve_stop(ctx);
    (void)calls; (void)probes;
    if (jr) {
      std::fprintf(stderr, "[journal] %zu units already committed, %zu searched now\n", resumed, n_units);
      if (s615_journal_close(jr) != S615_OK) jfail = true;
    }
    std::printf("---- done cls5-gpu serve: solutions=%llu units=%zu requests=%zu time=%.1fs ----\n", sols,
                n_units + resumed, submitted, std::chrono::duration<double>(Clock::now() - t0).count());
    s615_close(ctx);
    return jfail ? 1 : 0;
  }

  std::vector<Line> lines;
  if (!load_buc5(units_path.c_str(), lines)) {
    std::fprintf(stderr, "no cls5 units in %s\n", units_path.c_str());
    s615_close(ctx);
    return 1;
  }
  std::vector<s615_unit> units;
  units.reserve(lines.size());
  unsigned need = 0;
  for (const Line& L : lines) {
    s615_unit U{};
    U.cls = 5; U.kind = 0; U.B = L.B; U.u = L.u;
    const int st = s615_unit_status(&U);
    if (st == 1) continue;
    if (st != S615_OK) {
      std::fprintf(stderr, "[cls5-gpu] unit B=%llu u=%llu rejected: %s\n", L.B, L.u, s615_strerror(st));
      continue;
    }
    need = std::max(need, (unsigned)((L.B - 1) / 42));
    units.push_back(U);
  }
  std::fprintf(stderr, "[cls5-gpu] packed %zu/%zu units from %s\n", units.size(), lines.size(),
               units_path.c_str());
  if (units.empty()) { s615_close(ctx); return 1; }
  const int N = N_override > 0 ? N_override : (int)need;
  if (N > n_cap) {
    std::fprintf(stderr, "N=%d exceeds soft xor cap %d%s\n", N, n_cap,
                 shards > 1 ? "" : " (past it: --shards S)");
    s615_close(ctx);
    return 1;
  }
  std::fprintf(stderr, "[cls5-gpu] N=%d r=%d\n", N, xor_r);
  std::vector<Plant> plants;
  const size_t n_stage1 = units.size();
  if (plant_count > 0) {
    u64 bmax = 0;
    for (size_t i = 0; i < n_stage1; ++i) bmax = std::max<u64>(bmax, units[i].B);
    plants = make_plants(plant_count, plant_seed, bmax, N, units);
    std::fprintf(stderr, "[plant] %d planted targets after %zu units\n", plant_count, n_stage1);
  }
  std::vector<char> plant_got(plants.size(), 0);
  int tid = 0;
  if (!get_table(ctx, N, xor_r, tid)) {
    s615_close(ctx);
    return 1;
  }

  FILE* dump = nullptr;
  if (!dump_path.empty()) {
    dump = std::fopen(dump_path.c_str(), "w");
    if (!dump) { std::fprintf(stderr, "cannot open %s\n", dump_path.c_str()); s615_close(ctx); return 1; }
  }
  const unsigned flags = (use_gate ? 0u : S615_F_NO_GATE) | (plain ? S615_F_PLAIN : 0u);
  unsigned long long tot_calls = 0, tot_gated = 0, tot_probes = 0, sols = 0;
  // With a journal, committed units are skipped (their solutions printed
  // again) and the rest are searched in order; `order` holds the indices into
  // `units` still to search, kept contiguous in `work`.
  s615_journal* jr = nullptr;
  std::vector<s615_unit> work;
  std::vector<size_t> order;
  if (!journal_path.empty()) {
    if (!(jr = open_journal(journal_path))) { s615_close(ctx); return 1; }
    sols += replay_solutions(jr);
    size_t n = 0;
    s615_journal_solutions(jr, nullptr, 0, &n);
    std::vector<s615_solution> old(n);
    if (n) s615_journal_solutions(jr, old.data(), n, &n);
    size_t nu = 0;
    s615_journal_units(jr, nullptr, 0, &nu);
    std::vector<s615_unit> jus(nu);
    if (nu) s615_journal_units(jr, jus.data(), nu, &nu);
    for (const s615_solution& S : old) {   // plants recovered before the restart
      if (S.kind != 1) continue;
      for (size_t pi = 0; pi < plants.size(); ++pi) {
        const Plant& P = plants[pi];
        if (!std::memcmp(&jus[S.unit], &units[n_stage1 + pi], sizeof(s615_unit)) && S.e == P.e &&
            S.d == P.d && S.c1 == P.c1 && S.c2 == P.c2)
          plant_got[pi] = 1;
      }
    }
    for (size_t i = 0; i < units.size(); ++i)
      if (s615_journal_has(jr, &units[i]) != 1) order.push_back(i);
    std::fprintf(stderr, "[journal] %zu of %zu units already committed; searching %zu\n",
                 units.size() - order.size(), units.size(), order.size());
  } else {
    order.resize(units.size());
    for (size_t i = 0; i < units.size(); ++i) order[i] = i;
  }
  work.reserve(order.size());
  for (size_t i : order) work.push_back(units[i]);
  const auto t0 = Clock::now();
  std::vector<s615_hit> hits;
  std::vector<s615_solution> solv;
  size_t chunk_no = 0;
  for (size_t off = 0; off < work.size(); off += batch, ++chunk_no) {
    const size_t n = std::min(batch, work.size() - off);
    size_t cap = std::max<size_t>(hits.size(), 1 << 16), nh = 0;
    s615_counters c{};
    for (;;) {
      hits.resize(cap);
      s = s615_cls5_run(ctx, tid, work.data() + off, n, flags, hits.data(), cap, &nh, &c);
      if (s == S615_E_OVERFLOW && nh > cap) { cap = nh + nh / 4; continue; }
      break;
    }
    if (s) {
      std::fprintf(stderr, "[cls5-gpu] run failed: %s\n", s615_strerror(s));
      s615_close(ctx);
      return 1;
    }
    tot_calls += c.calls; tot_gated += c.gated; tot_probes += c.probes;
    if (dump)
      for (size_t k = 0; k < nh; ++k) {
        const s615_unit& U = work[off + hits[k].unit];
        std::fprintf(dump, "%llu %llu %u %u %llu\n", (unsigned long long)U.B, (unsigned long long)U.u,
                     hits[k].d, hits[k].e, (unsigned long long)hits[k].fp);
      }
    size_t ns = 0;
    if (nh) {
      size_t scap = std::max<size_t>(16, nh);
      for (;;) {   // one hit can verify to several pairs: grow the buffer until it holds them
        solv.resize(scap);
        s = s615_cls5_verify(ctx, work.data() + off, n, hits.data(), nh, N, solv.data(), scap, &ns);
        if (s == S615_E_OVERFLOW && ns > scap) { scap = ns; continue; }
        break;
      }
      if (s) {
        std::fprintf(stderr, "[cls5-gpu] verify failed: %s\n", s615_strerror(s));
        s615_close(ctx);
        return 1;
      }
      for (size_t k = 0; k < ns; ++k) {
        const s615_solution& S = solv[k];
        if (S.kind == 1) {   // a recovered plant: its exact planted (e, d, c1, c2)?
          const size_t ui = order[off + S.unit];
          const size_t pi = ui - n_stage1;
          if (ui >= n_stage1 && pi < plants.size()) {
            const Plant& P = plants[pi];
            if (S.e == P.e && S.d == P.d && S.c1 == P.c1 && S.c2 == P.c2) plant_got[pi] = 1;
          }
          continue;
        }
        if (S.kind != 0) continue;
        print_solution(S);
        ++sols;
        if (stop_first) break;
      }
    }
    if (jr && s615_journal_append(jr, work.data() + off, n, hits.data(), nh, solv.data(), ns) != S615_OK) {
      std::fprintf(stderr, "[journal] append failed\n");
      s615_journal_close(jr);
      s615_close(ctx);
      return 1;
    }
    const double sec = std::chrono::duration<double>(Clock::now() - t0).count();
    if (!quiet || chunk_no % 2 == 0 || off + n >= units.size()) {
      const double gate_pct = tot_calls ? 100.0 * (double)tot_gated / (double)tot_calls : 0.0;
      std::fprintf(stderr, "[cls5-gpu] units=%zu/%zu calls=%llu probes=%llu gate=%.1f%% sols=%llu %.1fs\n",
                   units.size() - work.size() + off + n, units.size(), tot_calls, tot_probes, gate_pct,
                   sols, sec);
    }
    if (stop_first && sols) break;
  }
  if (jr && s615_journal_close(jr) != S615_OK) {
    std::fprintf(stderr, "[journal] close failed\n");
    s615_close(ctx);
    return 1;
  }
  if (dump) std::fclose(dump);
  if (!plants.empty()) {
    size_t got = 0;
    for (char g : plant_got) got += g;
    std::fprintf(stderr, "[plant] recovered %zu/%zu\n", got, plants.size());
  }
  const double sec = std::chrono::duration<double>(Clock::now() - t0).count();
  std::printf("---- done cls5-gpu: solutions=%llu units=%zu calls=%llu probes=%llu time=%.1fs ----\n",
              sols, units.size(), tot_calls, tot_probes, sec);
  s615_close(ctx);
  return 0;
}
