// journal.cpp -- restart journal of a search campaign.
//
// The reference keeps no progress record: a restarted run redoes its whole
// band (fourcore_runbook_v3.md:162-170).  The journal is an append-only text
// file of committed blocks, one per finished request (serving loop) or chunk
// of units (batch CLI):
//
//   B <n_units> <n_hits> <n_sols>
//   U cls kind B u base0 base1 base2 fmax1 fmax2 res_e res_d lim w      x n_units
//   H unit a b d e c4 fp                                                 x n_hits
//   S unit kind cls c3 B u d e c1 c2 c4 w a0 .. a6 gcd                   x n_sols
//   C <n_units> <fnv1a-64 of the block's lines above, hex>
//
// Unit indices in H and S lines refer to the block's own U lines.  A block
// counts only once its C line is complete and its checksum matches, so a
// block torn by a crash is ignored (its units are searched again) and opening
// the journal cuts the file back to the last committed block before anything
// is appended.  Appends are flushed and fsync'd before they return.
#include <fcntl.h>
#include <unistd.h>

#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_set>
#include <vector>

#include "../../include/s615.h"

namespace {

struct UnitKey {
  std::string s;
  bool operator==(const UnitKey& o) const { return s == o.s; }
};
struct UnitKeyHash {
  size_t operator()(const UnitKey& k) const { return std::hash<std::string>()(k.s); }
};

std::string unit_line(const s615_unit& u) {
  char buf[512];
  std::snprintf(buf, sizeof buf,
                "U %u %u %" PRIu64 " %" PRIu64 " %" PRIu64 " %" PRIu64 " %" PRIu64 " %u %u %u %u %u %u\n",
                u.cls, u.kind, u.B, u.u, u.base[0], u.base[1], u.base[2], u.fmax1, u.fmax2, u.res_e,
                u.res_d, u.lim, u.w);
  return buf;
}

std::string hit_line(const s615_hit& h) {
  char buf[256];
  std::snprintf(buf, sizeof buf, "H %u %u %u %u %u %u %" PRIu64 "\n", h.unit, h.a, h.b, h.d, h.e,
                h.c4, h.fp);
  return buf;
}

std::string sol_line(const s615_solution& s) {
  char buf[768];
  std::snprintf(buf, sizeof buf,
                "S %u %u %u %u %" PRIu64 " %" PRIu64 " %u %u %u %u %u %u %" PRId64 " %" PRId64
                " %" PRId64 " %" PRId64 " %" PRId64 " %" PRId64 " %" PRId64 " %" PRId64 "\n",
                s.unit, s.kind, s.cls, s.c3, s.B, s.u, s.d, s.e, s.c1, s.c2, s.c4, s.w, s.a[0],
                s.a[1], s.a[2], s.a[3], s.a[4], s.a[5], s.a[6], s.gcd);
  return buf;
}

uint64_t fnv1a(const std::string& text) {
  uint64_t h = 1469598103934665603ULL;
  for (unsigned char c : text) {
    h ^= c;
    h *= 1099511628211ULL;
  }
  return h;
}

bool parse_unit(const char* l, s615_unit* u) {
  std::memset(u, 0, sizeof *u);
  return std::sscanf(l, "U %u %u %" SCNu64 " %" SCNu64 " %" SCNu64 " %" SCNu64 " %" SCNu64
                        " %u %u %u %u %u %u",
                     &u->cls, &u->kind, &u->B, &u->u, &u->base[0], &u->base[1], &u->base[2],
                     &u->fmax1, &u->fmax2, &u->res_e, &u->res_d, &u->lim, &u->w) == 13;
}

bool parse_sol(const char* l, s615_solution* s) {
  std::memset(s, 0, sizeof *s);
  return std::sscanf(l, "S %u %u %u %u %" SCNu64 " %" SCNu64 " %u %u %u %u %u %u %" SCNd64
                        " %" SCNd64 " %" SCNd64 " %" SCNd64 " %" SCNd64 " %" SCNd64 " %" SCNd64
                        " %" SCNd64,
                     &s->unit, &s->kind, &s->cls, &s->c3, &s->B, &s->u, &s->d, &s->e, &s->c1,
                     &s->c2, &s->c4, &s->w, &s->a[0], &s->a[1], &s->a[2], &s->a[3], &s->a[4],
                     &s->a[5], &s->a[6], &s->gcd) == 20;
}

}  // namespace

struct s615_journal {
  FILE* f = nullptr;
  std::unordered_set<UnitKey, UnitKeyHash> done;
  std::vector<s615_solution> sols;   // unit index = position in `units`
  std::vector<s615_unit> units;      // every committed unit, in file order
  size_t n_hits = 0;
};

extern "C" {

int s615_journal_open(const char* path, s615_journal** out) {
  if (!path || !out) return S615_E_ARG;
  *out = nullptr;
  auto* j = new s615_journal();
  long valid_end = 0;
  if (FILE* r = std::fopen(path, "r")) {
    // read committed blocks; stop at the first incomplete or corrupt one
    std::vector<std::string> lines;
    char buf[1024];
    while (std::fgets(buf, sizeof buf, r)) lines.emplace_back(buf);
    std::fclose(r);
    size_t i = 0;
    long pos = 0;
    while (i < lines.size()) {
      size_t nu = 0, nh = 0, ns = 0;
      if (std::sscanf(lines[i].c_str(), "B %zu %zu %zu", &nu, &nh, &ns) != 3) break;
      const size_t end = i + 1 + nu + nh + ns;   // index of the C line
      if (end >= lines.size()) break;
      std::string body;
      long bytes = 0;
      for (size_t k = i; k < end; ++k) {
        body += lines[k];
        bytes += (long)lines[k].size();
      }
      size_t cu = 0;
      uint64_t sum = 0;
      const std::string& c = lines[end];
      if (c.empty() || c.back() != '\n' ||
          std::sscanf(c.c_str(), "C %zu %" SCNx64, &cu, &sum) != 2 || cu != nu || sum != fnv1a(body))
        break;
      std::vector<s615_unit> us(nu);
      std::vector<s615_solution> ss(ns);
      bool ok = true;
      for (size_t k = 0; k < nu && ok; ++k) ok = parse_unit(lines[i + 1 + k].c_str(), &us[k]);
      for (size_t k = 0; k < ns && ok; ++k) {
        ok = parse_sol(lines[i + 1 + nu + nh + k].c_str(), &ss[k]) && ss[k].unit < nu;
      }
      if (!ok) break;
      const uint32_t base = (uint32_t)j->units.size();
      for (const s615_unit& u : us) {
        j->done.insert(UnitKey{unit_line(u)});
        j->units.push_back(u);
      }
      for (s615_solution& s : ss) {
        s.unit += base;
        j->sols.push_back(s);
      }
      j->n_hits += nh;
      pos += bytes + (long)c.size();
      i = end + 1;
    }
    valid_end = pos;
    // cut a torn or corrupt tail so that new blocks follow the last good one
    if (truncate(path, valid_end) != 0) {
      delete j;
      return S615_E_IO;
    }
  }
  j->f = std::fopen(path, "a");
  if (!j->f) {
    delete j;
    return S615_E_IO;
  }
  *out = j;
  return S615_OK;
}

int s615_journal_has(const s615_journal* j, const s615_unit* unit) {
  if (!j || !unit) return S615_E_ARG;
  return j->done.count(UnitKey{unit_line(*unit)}) ? 1 : 0;
}

int s615_journal_stats(const s615_journal* j, size_t* units, size_t* hits, size_t* solutions) {
  if (!j) return S615_E_ARG;
  if (units) *units = j->units.size();
  if (hits) *hits = j->n_hits;
  if (solutions) *solutions = j->sols.size();
  return S615_OK;
}

int s615_journal_solutions(const s615_journal* j, s615_solution* out, size_t cap, size_t* n) {
  if (!j || !n || (cap && !out)) return S615_E_ARG;
  *n = j->sols.size();
  if (cap < j->sols.size()) return S615_E_OVERFLOW;
  if (!j->sols.empty()) std::memcpy(out, j->sols.data(), j->sols.size() * sizeof(s615_solution));
  return S615_OK;
}

int s615_journal_units(const s615_journal* j, s615_unit* out, size_t cap, size_t* n) {
  if (!j || !n || (cap && !out)) return S615_E_ARG;
  *n = j->units.size();
  if (cap < j->units.size()) return S615_E_OVERFLOW;
  if (!j->units.empty()) std::memcpy(out, j->units.data(), j->units.size() * sizeof(s615_unit));
  return S615_OK;
}

int s615_journal_append(s615_journal* j, const s615_unit* units, size_t n, const s615_hit* hits,
                        size_t n_hits, const s615_solution* sols, size_t n_sols) {
  if (!j || !j->f || (n && !units) || (n_hits && !hits) || (n_sols && !sols)) return S615_E_ARG;
  for (size_t k = 0; k < n_hits; ++k)
    if (hits[k].unit >= n) return S615_E_ARG;
  for (size_t k = 0; k < n_sols; ++k)
    if (sols[k].unit >= n) return S615_E_ARG;
  char head[96];
  std::snprintf(head, sizeof head, "B %zu %zu %zu\n", n, n_hits, n_sols);
  std::string body = head;
  for (size_t k = 0; k < n; ++k) body += unit_line(units[k]);
  for (size_t k = 0; k < n_hits; ++k) body += hit_line(hits[k]);
  for (size_t k = 0; k < n_sols; ++k) body += sol_line(sols[k]);
  char tail[96];
  std::snprintf(tail, sizeof tail, "C %zu %016" PRIx64 "\n", n, fnv1a(body));
  body += tail;
  if (std::fwrite(body.data(), 1, body.size(), j->f) != body.size() || std::fflush(j->f) != 0 ||
      fsync(fileno(j->f)) != 0)
    return S615_E_IO;
  const uint32_t base = (uint32_t)j->units.size();
  for (size_t k = 0; k < n; ++k) {
    j->done.insert(UnitKey{unit_line(units[k])});
    j->units.push_back(units[k]);
  }
  for (size_t k = 0; k < n_sols; ++k) {
    s615_solution s = sols[k];
    s.unit += base;
    j->sols.push_back(s);
  }
  j->n_hits += n_hits;
  return S615_OK;
}

int s615_journal_close(s615_journal* j) {
  if (!j) return S615_E_ARG;
  int s = S615_OK;
  if (j->f && std::fclose(j->f) != 0) s = S615_E_IO;
  delete j;
  return s;
}

}  // extern "C"
