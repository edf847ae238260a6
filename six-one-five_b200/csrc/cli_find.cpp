// cli_find.cpp -- s615_find, a drop-in for fourcore_find_v4's job and unit modes.
//
// Same flags, stdout lines and exit codes as fourcore_find_v4.cu:896-1227 for
// --jobs FILE.but|.bbj (reduced-T jobs; .bbj streamed), --units FILE.buc
// (stream-expand of Stage-1 units into jobs), --selftest-gpu (planted
// find2 / find3 / find4 jobs on an N = 40 table, :808-892) and
// --selftest-host.  The search runs on the engine (s615_run + s615_verify
// with kind 2 units).  Extra flags: --load-table F (a table file instead of
// the device build), --shards S / --load-shards F0,F1,.. (a pair-space shard
// set, past the single-table cap) and --emit-jobs F (with --units: write the expanded jobs
// as a .bbj or text job file instead of searching, the hunt tool's
// --expand --emit, fourcore_hunt_v3.cpp:347-447).  The per-batch "[gate]"
// line counts a whole engine batch (every find mode together).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/s615.h"

namespace {

constexpr int kNSoftMax = 120000;   // kXorNSoftMax of the reference's store
constexpr int kNShardMax = 240000;  // with pair-space shards, as HBM allows

// Table options beyond the reference's: a file, or a pair-space shard set
// (built on the device, or loaded from its shard files in order).
struct TableOpts {
  std::string load;
  int shards = 1;
  std::vector<std::string> shard_files;
};

void usage() {
  std::printf(
      "usage: s615_find [--selftest-host] [--selftest-gpu]\n"
      "   or: s615_find --jobs FILE.but|.bbj [options]\n"
      "   or: s615_find --units FILE.buc [options]   (stream-expand)\n"
      "   or: s615_find --units FILE.buc --emit-jobs FILE.bbj|FILE.but [--max-expand N]\n"
      " options: --N n --r BITS (xor rank, default 48) --batch N --max-expand N\n"
      "          --max-table-gb G (ignored) --S (ignored) --load-table F\n"
      "          --shards S | --load-shards F0,F1,.. (pair-space shard set; N <= 240000)\n"
      "          --quiet --no-quiet --no-gate --stop-first --device K\n"
      "  .buc: cls B u\n"
      "  .but: ASCII jobs | .bbj: binary jobs (36 B/job; streamed)\n");
}

struct Run {
  s615_ctx* ctx = nullptr;
  int tid = -1, N = 0;
  unsigned flags = 0;
  bool quiet = false;
  std::vector<s615_hit> hits = std::vector<s615_hit>(1 << 20);
  std::vector<s615_solution> sols = std::vector<s615_solution>(1 << 16);

  // One engine batch: search, verify, print; returns the exact matches
  // (kind 0 and kind 2 records: the reference's `sols`), or -1 on error.
  long long batch(const std::vector<s615_unit>& jobs) {
    if (jobs.empty()) return 0;
    size_t nh = 0;
    s615_counters c{};
    int s = s615_run(ctx, tid, jobs.data(), jobs.size(), flags, hits.data(), hits.size(), &nh, &c);
    if (s == S615_E_OVERFLOW) {
      hits.resize(nh + nh / 4 + 1024);
      s = s615_run(ctx, tid, jobs.data(), jobs.size(), flags, hits.data(), hits.size(), &nh, &c);
    }
    if (s) {
      std::fprintf(stderr, "[find] run failed: %s\n", s615_strerror(s));
      return -1;
    }
    if (!quiet && c.calls)
      std::fprintf(stderr, "[gate] batch n=%zu calls=%llu gated=%llu probes=%llu gate=%.1f%%\n",
                   jobs.size(), (unsigned long long)c.calls, (unsigned long long)c.gated,
                   (unsigned long long)c.probes, 100.0 * (double)c.gated / (double)c.calls);
    size_t ns = 0;
    s = s615_verify(ctx, jobs.data(), jobs.size(), hits.data(), nh, N, sols.data(), sols.size(), &ns);
    if (s == S615_E_OVERFLOW) {
      sols.resize(ns + 64);
      s = s615_verify(ctx, jobs.data(), jobs.size(), hits.data(), nh, N, sols.data(), sols.size(), &ns);
    }
    if (s) {
      std::fprintf(stderr, "[find] verify failed: %s\n", s615_strerror(s));
      return -1;
    }
    for (size_t i = 0; i < ns; ++i) {   // report_solution (fourcore_find_v4.cu:427-457)
      const s615_solution& S = sols[i];
      if (S.kind != 0) continue;
      std::printf("SOLUTION cls=%u B=%llu u=%llu a1=%lld a2=%lld a3=%lld a4=%lld a5=%lld gcd=%lld %s\n",
                  S.cls, (unsigned long long)S.B, (unsigned long long)S.u, (long long)S.a[0],
                  (long long)S.a[1], (long long)S.a[2], (long long)S.a[3], (long long)S.a[4],
                  (long long)S.gcd, S.gcd == 1 ? "primitive" : "NON-PRIMITIVE");
      std::fflush(stdout);
      std::fprintf(stderr, "%llu\tSOLUTION\tcls=%u\n", (unsigned long long)S.B, S.cls);
    }
    return (long long)ns;
  }
};

bool start(Run& R, int device, int N, int r, const TableOpts& T) {
  int s = s615_open(device, 0, &R.ctx);
  if (s) {
    std::fprintf(stderr, "[find] cannot open device %d: %s\n", device, s615_strerror(s));
    return false;
  }
  R.N = N;
  if (!T.shard_files.empty()) {
    std::vector<const char*> paths;
    for (const auto& f : T.shard_files) paths.push_back(f.c_str());
    s = s615_load_table_shards(R.ctx, paths.data(), (int)paths.size(), N, S615_LAYOUT_WIDE, &R.tid);
  } else if (T.shards > 1) {
    s = s615_build_table_sharded(R.ctx, N, r, T.shards, S615_LAYOUT_WIDE, &R.tid);
  } else {
    s = T.load.empty() ? s615_build_table(R.ctx, N, r, S615_LAYOUT_WIDE, &R.tid)
                       : s615_load_table(R.ctx, T.load.c_str(), N, S615_LAYOUT_WIDE, &R.tid);
  }
  if (s) {
    std::fprintf(stderr, "[find] FATAL: xor table: %s\n", s615_strerror(s));
    return false;
  }
  return true;
}

uint32_t job_lim(const s615_unit& J) {
  return J.lim ? J.lim : (uint32_t)((J.B > 0 ? J.B - 1 : 0) / 42);
}

// selftest_gpu (fourcore_find_v4.cu:808-892): exact T matches of one planted
// job per find mode, checked without the (6,1,5) identity (fake B).
int selftest_gpu(int device) {
  std::printf("[selftest-gpu] tiny xor store + planted find2/find3/find4\n");
  const int N = 40;
  Run R;
  R.quiet = true;
  if (!start(R, device, N, 48, TableOpts{})) return 1;
  auto p6 = [](unsigned long long x) { return x * x * x * x * x * x; };
  struct Plant { int mode; uint32_t cls; uint64_t B; uint32_t f1, f2; unsigned long long T; };
  const Plant plants[3] = {
      {2, 5, 999999, 1, 1, p6(3) + p6(4)},
      {3, 2, 999998, 1, 0, p6(3) + p6(4) + p6(5)},
      {4, 1, 999997, 0, 0, p6(3) + p6(4) + p6(5) + p6(6)}};
  unsigned long long total = 0;
  for (const Plant& P : plants) {
    s615_unit J{};
    J.cls = P.cls; J.kind = S615_KIND_JOB; J.B = P.B; J.u = 1;
    J.res_d = P.f1; J.res_e = P.f2; J.lim = N;
    J.base[0] = P.T;
    size_t nh = 0;
    s615_counters c{};
    int s = s615_run(R.ctx, R.tid, &J, 1, 0, R.hits.data(), R.hits.size(), &nh, &c);
    size_t ns = 0;
    if (!s) s = s615_verify(R.ctx, &J, 1, R.hits.data(), nh, N, R.sols.data(), R.sols.size(), &ns);
    if (s) {
      std::printf("FAIL find%d plant: %s\n", P.mode, s615_strerror(s));
      s615_close(R.ctx);
      return 1;
    }
    std::printf("  find%d plant exact_hits=%zu (raw nh=%zu)\n", P.mode, ns, nh);
    if (!ns) {
      std::printf("FAIL find%d plant\n", P.mode);
      s615_close(R.ctx);
      return 1;
    }
    total += ns;
  }
  s615_close(R.ctx);
  std::printf("[selftest-gpu] PASS (exact=%llu)\n", total);
  return 0;
}

bool load_buc(const char* path, std::vector<s615_unit>& units) {
  FILE* f = std::fopen(path, "r");
  if (!f) return false;
  char buf[256];
  while (std::fgets(buf, sizeof buf, f)) {   // load_units_buc (fourcore_find_v4.cu:147-161)
    int cls;
    unsigned long long B, u;
    if (std::sscanf(buf, "%d %llu %llu", &cls, &B, &u) != 3) continue;
    s615_unit U{};
    U.cls = (uint32_t)cls; U.B = B; U.u = u;
    units.push_back(U);
  }
  std::fclose(f);
  return !units.empty();
}

}  // namespace

int main(int argc, char** argv) {
  std::setvbuf(stdout, nullptr, _IOLBF, 0);
  std::setvbuf(stderr, nullptr, _IOLBF, 0);
  std::string units_path, jobs_path, emit;
  TableOpts topt;
  int N = 0, device = 0, r = 48, quiet_flag = -1;
  unsigned long long max_expand = 0, batch = 1ULL << 20;
  bool use_gate = true, stop_first = false, do_host = false, do_gpu = false;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto next = [&]() { return i + 1 < argc ? std::string(argv[++i]) : std::string(); };
    if (a == "--selftest-host") do_host = true;
    else if (a == "--selftest-gpu") do_gpu = true;
    else if (a == "--units") units_path = next();
    else if (a == "--jobs") jobs_path = next();
    else if (a == "--N") N = std::atoi(next().c_str());
    else if (a == "--r") r = std::atoi(next().c_str());
    else if (a == "--batch") batch = std::strtoull(next().c_str(), nullptr, 10);
    else if (a == "--max-expand") max_expand = std::strtoull(next().c_str(), nullptr, 10);
    else if (a == "--max-table-gb" || a == "--S") (void)next();
    else if (a == "--quiet") quiet_flag = 1;
    else if (a == "--no-quiet") quiet_flag = 0;
    else if (a == "--no-gate") use_gate = false;
    else if (a == "--stop-first") stop_first = true;
    else if (a == "--device") device = std::atoi(next().c_str());
    else if (a == "--load-table") topt.load = next();
    else if (a == "--shards") topt.shards = std::atoi(next().c_str());
    else if (a == "--load-shards") {
      const std::string v = next();
      size_t p = 0;
      while (p <= v.size()) {
        const size_t q = v.find(',', p);
        const std::string f = v.substr(p, q == std::string::npos ? std::string::npos : q - p);
        if (!f.empty()) topt.shard_files.push_back(f);
        if (q == std::string::npos) break;
        p = q + 1;
      }
    }
    else if (a == "--emit-jobs") emit = next();
    else if (a == "-h" || a == "--help") { usage(); return 0; }
    else { std::fprintf(stderr, "unknown arg %s\n", a.c_str()); usage(); return 1; }
  }
  if (do_host) {
    std::printf("[selftest-host] engine host checks\n");
    const int s = s615_selftest_host();
    if (s) { std::printf("FAIL check %d\n", s); return 1; }
    std::printf("[selftest-host] PASS\n");
    if (!do_gpu) return 0;
  }
  if (do_gpu) return selftest_gpu(device);
  if (r < 8 || r > 64) { std::fprintf(stderr, "--r must be 8..64\n"); return 1; }
  if (topt.shards != 1 && (topt.shards < 2 || topt.shards > 64)) {
    std::fprintf(stderr, "--shards must be 2..64\n");
    return 1;
  }
  const int n_cap = (topt.shards > 1 || !topt.shard_files.empty()) ? kNShardMax : kNSoftMax;
  if (batch < 1) batch = 1;
  if (batch > (1ULL << 24)) batch = 1ULL << 24;
  const bool quiet = quiet_flag == 1;

  Run R;
  R.quiet = quiet;
  R.flags = use_gate ? 0u : S615_F_NO_GATE;
  unsigned long long sols = 0, jobs_done = 0, fail_t = 0;

  // ---- binary jobs: streamed (stream_jobs_bbj, fourcore_find_v4.cu:634-679) ----
  if (!jobs_path.empty()) {
    s615_jobs_file* f = nullptr;
    s615_jobs_info info{};
    int s = s615_jobs_open(jobs_path.c_str(), &f, &info);
    if (s) {
      if (s == S615_E_IO) std::perror(jobs_path.c_str());
      std::fprintf(stderr, info.binary || s == S615_E_FORMAT ? "bad .bbj %s\n" : "failed to load %s\n",
                   jobs_path.c_str());
      return 1;
    }
    std::vector<s615_unit> all;   // text jobs load all first (:1161-1170)
    if (info.binary) {
      if (!info.n_jobs) { std::fprintf(stderr, "empty .bbj\n"); s615_jobs_close(f, nullptr); return 1; }
      const int need = info.max_B ? (int)((info.max_B - 1) / 42) : 0;
      if (N <= 0 || N < need) N = need;
    } else {
      std::vector<s615_unit> buf(1 << 16);
      size_t k = 0;
      while (!(s = s615_jobs_next(f, buf.data(), buf.size(), &k)) && k)
        all.insert(all.end(), buf.begin(), buf.begin() + (long)k);
      s615_jobs_close(f, &info);
      f = nullptr;
      if (info.bad_lines) std::fprintf(stderr, "[jobs] skipped %llu bad lines\n", (unsigned long long)info.bad_lines);
      if (s || all.empty()) { std::fprintf(stderr, "failed to load %s\n", jobs_path.c_str()); return 1; }
      std::fprintf(stderr, "[jobs] loaded %zu from %s (ASCII)\n", all.size(), jobs_path.c_str());
      uint32_t need = 0;
      for (const auto& J : all) need = std::max(need, job_lim(J));
      if (N <= 0 || N < (int)need) N = (int)need;
    }
    if (N > n_cap) {
      std::fprintf(stderr, "[fatal] N=%d exceeds soft xor cap %d\n", N, n_cap);
      if (f) s615_jobs_close(f, nullptr);
      return 1;
    }
    if (!start(R, device, N, r, topt)) { if (f) s615_jobs_close(f, nullptr); return 1; }
    if (info.binary) {
      std::fprintf(stderr, "[bbj] stream %s n_jobs=%llu B=[%u,%u]\n", jobs_path.c_str(),
                   (unsigned long long)info.n_jobs, info.min_B, info.max_B);
      std::vector<s615_unit> buf(batch), take;
      size_t k = 0;
      bool bad = false;
      while (!(s = s615_jobs_next(f, buf.data(), buf.size(), &k)) && k) {
        take.clear();
        for (size_t i = 0; i < k; ++i) {
          if ((int)job_lim(buf[i]) > N) {
            std::fprintf(stderr, "[bbj] job lim=%u > N=%d — skip\n", job_lim(buf[i]), N);
            continue;
          }
          take.push_back(buf[i]);
        }
        jobs_done += take.size();
        const long long got = R.batch(take);
        if (got < 0) { bad = true; break; }
        sols += (unsigned long long)got;
        std::fprintf(stderr, "[progress] bbj %llu/%llu sols=%llu\n", jobs_done,
                     (unsigned long long)info.n_jobs, sols);
        if (stop_first && sols) break;
      }
      s615_jobs_close(f, nullptr);
      s615_close(R.ctx);
      if (bad || s) return 1;
      std::printf("---- done: solutions=%llu jobs=%llu failT=0 (bbj stream) ----\n", sols, jobs_done);
      return 0;
    }
    for (size_t off = 0; off < all.size(); off += batch) {   // process_jobs (:571-596)
      const std::vector<s615_unit> piece(all.begin() + (long)off,
                                         all.begin() + (long)std::min<size_t>(all.size(), off + batch));
      const long long got = R.batch(piece);
      if (got < 0) { s615_close(R.ctx); return 1; }
      sols += (unsigned long long)got;
      if (stop_first && sols) break;
    }
    s615_close(R.ctx);
    std::printf("---- done: solutions=%llu jobs=%zu failT=0 ----\n", sols, all.size());
    return 0;
  }

  // ---- Stage-1 units: stream-expand (stream_units_expand, :681-760) ----
  if (!units_path.empty()) {
    std::vector<s615_unit> units;
    if (!load_buc(units_path.c_str(), units)) {
      std::fprintf(stderr, "failed to load %s\n", units_path.c_str());
      return 1;
    }
    uint32_t need = 0;
    for (const auto& U : units) need = std::max(need, (uint32_t)((U.B > 0 ? U.B - 1 : 0) / 42));
    if (N <= 0 || N < (int)need) N = (int)need;
    if (N > n_cap) {
      std::fprintf(stderr, "[fatal] N=%d exceeds soft xor cap %d\n", N, n_cap);
      return 1;
    }
    const bool emitting = !emit.empty();
    if (!emitting) {
      std::fprintf(stderr, "[units] %zu from %s — stream-expand (max_expand=%llu) N=%d\n", units.size(),
                   units_path.c_str(), max_expand, N);
      if (!start(R, device, N, r, topt)) return 1;
    }
    std::vector<s615_unit> pending, emitted, tmp;
    bool cap = false, bad = false;
    for (size_t ui = 0; ui < units.size() && !cap && !bad; ++ui) {
      size_t n = 0;
      uint64_t ft = 0;
      int s = s615_expand_unit(&units[ui], nullptr, 0, &n, &ft);
      if (s == S615_E_ARG) continue;   // a class or B the expansion does not take
      tmp.resize(std::max<size_t>(n, 1));
      s = s615_expand_unit(&units[ui], tmp.data(), tmp.size(), &n, &ft);
      if (s) { bad = true; break; }
      fail_t += ft;
      for (size_t i = 0; i < n; ++i) {
        if (max_expand && jobs_done >= max_expand) { cap = true; break; }
        if ((int)job_lim(tmp[i]) > N) continue;
        (emitting ? emitted : pending).push_back(tmp[i]);
        ++jobs_done;
        if (!emitting && pending.size() >= batch) {
          const long long got = R.batch(pending);
          pending.clear();
          if (got < 0) { bad = true; break; }
          sols += (unsigned long long)got;
          if (stop_first && sols) { cap = true; break; }
        }
      }
      if (!emitting && ((ui + 1) % 100 == 0 || ui + 1 == units.size()))
        std::fprintf(stderr, "[stream-units] %zu/%zu jobs=%llu failT=%llu sols=%llu\n", ui + 1,
                     units.size(), jobs_done, fail_t, sols);
    }
    if (emitting) {
      if (bad) return 1;
      const int s = s615_jobs_write(emit.c_str(), emitted.data(), emitted.size());
      if (s) { std::fprintf(stderr, "[emit] %s: %s\n", emit.c_str(), s615_strerror(s)); return 1; }
      std::fprintf(stderr, "[emit] %llu jobs -> %s (failT=%llu)%s\n", jobs_done, emit.c_str(), fail_t,
                   cap ? " (hit --max-expand)" : "");
      return 0;
    }
    if (!bad && !(stop_first && sols)) {
      const long long got = R.batch(pending);
      if (got < 0) bad = true;
      else sols += (unsigned long long)got;
    }
    s615_close(R.ctx);
    if (bad) return 1;
    std::printf("---- done: solutions=%llu jobs=%llu failT=%llu (units stream) ----\n", sols, jobs_done,
                fail_t);
    return 0;
  }
  std::fprintf(stderr, "no --jobs / --units\n");
  usage();
  return 1;
}
