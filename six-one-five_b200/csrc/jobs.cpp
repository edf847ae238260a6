// jobs.cpp -- reduced-T jobs: expand_unit and the .but / .bbj job files.
//
// A job is one reduced target T of fourcore_find_v4 (its Job{cls, B, u,
// free1, free2, T}, fourcore_find_v4.cu:91-97): what is left of B^6 after the
// anchor u and the free terms are peeled, divided by 42^6.  expand_unit
// (:164-205) makes them from Stage-1 units; the binary file layout is
// fourcore_job_bin.hpp:16-46 and the text one load_jobs_but (:125-145).  Jobs
// enter the engine as kind 2 units (include/s615.h).
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "engine.hpp"

namespace s615 {
namespace {

constexpr uint32_t kBbjMagic = 0x4a424346u;   // 'FCJB' little-endian
constexpr uint32_t kBbjVersion = 2;
constexpr size_t kBbjHeader = 32, kBbjRecord = 36;

bool is_bbj(const char* path) {
  const size_t n = std::strlen(path);
  if (n < 4) return false;
  const char* e = path + n - 4;
  return e[0] == '.' && std::tolower((unsigned char)e[1]) == 'b' &&
         std::tolower((unsigned char)e[2]) == 'b' && std::tolower((unsigned char)e[3]) == 'j';
}

template <class T> void put(uint8_t* p, T v) { std::memcpy(p, &v, sizeof v); }
template <class T> T get(const uint8_t* p) { T v; std::memcpy(&v, p, sizeof v); return v; }

s615_unit make_job(uint32_t cls, uint64_t B, uint64_t u, uint64_t f1, uint64_t f2, uint64_t tlo,
                   uint64_t thi) {
  s615_unit J{};
  J.cls = cls;
  J.kind = S615_KIND_JOB;
  J.B = B;
  J.u = u;
  J.res_d = (uint32_t)f1;
  J.res_e = (uint32_t)f2;
  J.base[0] = tlo;
  J.base[1] = thi;
  return J;
}

// T = (B^6 - u^6 - sum of terms^6) / 42^6 as compute_T_gmp (D = 42),
// compute_T_peel1_gmp and compute_T_peel2_gmp (fourcore_gmp.hpp:34-62): false
// when the difference is not positive or not divisible, or T >= 2^128.
bool job_T(u64 B, u64 u, const u64* terms, int nt, u128* T) {
  if (u >= B) return false;
  W3 R = pow6_w3(B);
  if (sub_w3(R, pow6_w3(u))) return false;
  for (int i = 0; i < nt; ++i)
    if (sub_w3(R, pow6_w3(terms[i]))) return false;
  if (zero_w3(R) || divmod_w3(R, kM42) != 0 || R.l[2] != 0) return false;
  *T = ((u128)R.l[1] << 64) | R.l[0];
  return true;
}

// for_each_free (fourcore_classes_v3.hpp:224-232): x = r + k mod <= fmax, x != 0.
template <class Fn>
void each_free(const std::vector<u32>& res, u64 mod, u64 fmax, Fn&& fn) {
  if (mod == 0 || fmax < 1) return;
  for (u32 r : res)
    for (u64 x = r; x <= fmax; x += mod)
      if (x) fn(x);
}

}  // namespace
}  // namespace s615

using namespace s615;

struct s615_jobs_file {
  FILE* fp = nullptr;
  s615_jobs_info info{};
  uint64_t read = 0;
};

extern "C" {

int s615_expand_unit(const s615_unit* unit, s615_unit* out, size_t cap, size_t* n,
                     uint64_t* fail_t) {
  if (!unit || !n || (cap && !out)) return S615_E_ARG;
  const s615_unit& U = *unit;
  if (U.kind != 0 || U.cls < 1 || U.cls > 5 || U.B < 2 || U.B > 40000000ULL) return S615_E_ARG;
  const u64 B = U.B, u = U.u;
  size_t k = 0;
  uint64_t fails = 0;
  u128 T = 0;
  auto push = [&](u64 f1, u64 f2, u128 t) {
    if (t == 0) return;
    if (k < cap) out[k] = make_job(U.cls, B, u, f1, f2, (u64)t, (u64)(t >> 64));
    ++k;
  };
  if (U.cls == 1) {                                  // :172-176
    if (job_T(B, u, nullptr, 0, &T)) push(0, 0, T);
    else ++fails;
  } else if (U.cls <= 4) {                           // :178-189
    u32 mod = 0, fmax = 0;
    const auto dr = d_residues_cls234(B, u, (int)U.cls, &mod, &fmax);
    const u64 f = (u64)free_factor((int)U.cls);
    each_free(dr, mod, fmax, [&](u64 d) {
      const u64 t1 = f * d;
      if (job_T(B, u, &t1, 1, &T)) push(d, 0, T);
      else ++fails;
    });
  } else {                                           // :190-203, e outer
    const auto er = e_residues(B);
    const auto dr = d_residues(B, u);
    each_free(er, kModE, (B - 1) / 14, [&](u64 e) {
      each_free(dr, kModD, (B - 1) / 21, [&](u64 d) {
        const u64 t2[2] = {21 * d, 14 * e};
        if (job_T(B, u, t2, 2, &T)) push(d, e, T);
        else ++fails;
      });
    });
  }
  *n = k;
  if (fail_t) *fail_t = fails;
  return k > cap ? S615_E_OVERFLOW : S615_OK;
}

int s615_jobs_open(const char* path, s615_jobs_file** out, s615_jobs_info* info) {
  if (!path || !out) return S615_E_ARG;
  *out = nullptr;
  const bool bin = is_bbj(path);
  FILE* fp = std::fopen(path, bin ? "rb" : "r");
  if (!fp) return S615_E_IO;
  s615_jobs_file* f = new s615_jobs_file();
  f->fp = fp;
  f->info.binary = bin ? 1u : 0u;
  if (bin) {   // read_header + header_ok (fourcore_job_bin.hpp:48-50, 86-89)
    uint8_t h[kBbjHeader];
    if (std::fread(h, 1, sizeof h, fp) != sizeof h || get<uint32_t>(h) != kBbjMagic ||
        get<uint32_t>(h + 4) != kBbjVersion || get<uint32_t>(h + 16) != kBbjRecord) {
      std::fclose(fp);
      delete f;
      return S615_E_FORMAT;
    }
    f->info.n_jobs = get<uint64_t>(h + 8);
    f->info.min_B = get<uint32_t>(h + 20);
    f->info.max_B = get<uint32_t>(h + 24);
  }
  if (info) *info = f->info;
  *out = f;
  return S615_OK;
}

int s615_jobs_next(s615_jobs_file* f, s615_unit* out, size_t cap, size_t* n) {
  if (!f || !n || (cap && !out)) return S615_E_ARG;
  size_t k = 0;
  if (f->info.binary) {
    // blocks of records read whole (up to 2^22 at a time), each decoded by up
    // to 16 threads when it is large
    std::vector<uint8_t> buf;
    while (k < cap) {
      const size_t want = std::min<size_t>(cap - k, 1u << 22);
      buf.resize(want * kBbjRecord);
      const size_t got = std::fread(buf.data(), kBbjRecord, want, f->fp);
      auto decode = [&](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; ++i) {
          // JobBinRec {u8 cls, 3 pad, u32 B, u, free1, free2, u64 T_lo, T_hi}
          const uint8_t* r = buf.data() + i * kBbjRecord;
          out[k + i] = make_job(r[0], get<uint32_t>(r + 4), get<uint32_t>(r + 8),
                                get<uint32_t>(r + 12), get<uint32_t>(r + 16),
                                get<uint64_t>(r + 20), get<uint64_t>(r + 28));
        }
      };
      const size_t nt = got < (1u << 16) ? 1
                        : std::min<size_t>({16, got >> 16,
                                            std::max(1u, std::thread::hardware_concurrency())});
      if (nt <= 1) {
        decode(0, got);
      } else {
        std::vector<std::thread> th;
        for (size_t t = 0; t < nt; ++t) th.emplace_back(decode, got * t / nt, got * (t + 1) / nt);
        for (auto& x : th) x.join();
      }
      k += got;
      if (got < want) break;
    }
  } else {
    char line[256];
    while (k < cap && std::fgets(line, sizeof line, f->fp)) {
      int cls = 0;
      unsigned long long B, u, f1, f2, tlo, thi;
      if (std::sscanf(line, "%d %llu %llu %llu %llu %llu %llu", &cls, &B, &u, &f1, &f2, &tlo,
                      &thi) != 7) {
        ++f->info.bad_lines;
        continue;
      }
      out[k++] = make_job((uint32_t)cls, B, u, f1, f2, tlo, thi);
    }
  }
  f->read += k;
  *n = k;
  return std::ferror(f->fp) ? S615_E_IO : S615_OK;
}

int s615_jobs_close(s615_jobs_file* f, s615_jobs_info* info) {
  if (!f) return S615_E_ARG;
  if (info) *info = f->info;
  std::fclose(f->fp);
  delete f;
  return S615_OK;
}

int s615_jobs_write(const char* path, const s615_unit* jobs, size_t n) {
  if (!path || (n && !jobs)) return S615_E_ARG;
  uint32_t lo = 0, hi = 0;
  for (size_t i = 0; i < n; ++i) {
    const s615_unit& J = jobs[i];
    if (J.kind != S615_KIND_JOB || J.cls > 255 || J.base[2] != 0) return S615_E_ARG;
    if (J.B > 0xFFFFFFFFull || J.u > 0xFFFFFFFFull) return S615_E_ARG;   // u32 record fields
    lo = i ? std::min(lo, (uint32_t)J.B) : (uint32_t)J.B;
    hi = std::max(hi, (uint32_t)J.B);
  }
  const bool bin = is_bbj(path);
  FILE* fp = std::fopen(path, bin ? "wb" : "w");
  if (!fp) return S615_E_IO;
  bool ok = true;
  if (bin) {   // write_header (fourcore_job_bin.hpp:52-59) with the final count
    uint8_t h[kBbjHeader] = {};
    put<uint32_t>(h, kBbjMagic);
    put<uint32_t>(h + 4, kBbjVersion);
    put<uint64_t>(h + 8, (uint64_t)n);
    put<uint32_t>(h + 16, (uint32_t)kBbjRecord);
    put<uint32_t>(h + 20, lo);
    put<uint32_t>(h + 24, hi);
    ok = std::fwrite(h, 1, sizeof h, fp) == sizeof h;
    for (size_t i = 0; ok && i < n; ++i) {   // write_rec (:69-81)
      const s615_unit& J = jobs[i];
      uint8_t r[kBbjRecord] = {};
      r[0] = (uint8_t)J.cls;
      put<uint32_t>(r + 4, (uint32_t)J.B);
      put<uint32_t>(r + 8, (uint32_t)J.u);
      put<uint32_t>(r + 12, J.res_d);
      put<uint32_t>(r + 16, J.res_e);
      put<uint64_t>(r + 20, J.base[0]);
      put<uint64_t>(r + 28, J.base[1]);
      ok = std::fwrite(r, 1, sizeof r, fp) == sizeof r;
    }
  } else {   // the --expand --emit line (fourcore_hunt_v3.cpp:260)
    for (size_t i = 0; ok && i < n; ++i) {
      const s615_unit& J = jobs[i];
      ok = std::fprintf(fp, "%u %llu %llu %u %u %llu %llu\n", J.cls, (unsigned long long)J.B,
                        (unsigned long long)J.u, J.res_d, J.res_e, (unsigned long long)J.base[0],
                        (unsigned long long)J.base[1]) > 0;
    }
  }
  if (std::fclose(fp) != 0) ok = false;
  return ok ? S615_OK : S615_E_IO;
}

}  // extern "C"
