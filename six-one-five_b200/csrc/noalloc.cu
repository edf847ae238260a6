// noalloc.cu -- s615_cls5_run_noalloc: the class-5 sieve run with no device
// allocation.
//
// Some callers cannot allocate device memory at the point where they want to
// search units: a process whose free HBM is already owned by another
// allocator (a framework's caching pool, a co-resident service), a serving
// thread that must not pay cudaMalloc's latency and implicit device
// synchronisation, or a plugin whose host forbids new device allocations.
// This entry point runs the same sieve kernel as s615_cls5_run, but the
// device-side unit records, work items, counters, queue cursor and hit buffer
// live in one fixed array declared below, sized for kMaxUnits units.  The
// table must already be resident (loading or building it allocates once).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <cstddef>
#include <mutex>

#include "engine.hpp"

namespace s615 {

namespace {

constexpr size_t kMaxUnits = 4096;
constexpr size_t kMaxItems = 65536;
constexpr size_t kMaxHits = 16384;

struct Scratch {
  DevUnit units[kMaxUnits];
  u64 items[kMaxItems];
  s615_hit hits[kMaxHits];
  Cls5Counters ctr;
  u32 work;
};
// launch_peel clears 8 bytes of work counters between passes over a shard set
static_assert(offsetof(Scratch, work) + 8 <= sizeof(Scratch), "work counters");

// The scratch: every GPU that loads the library holds these ~1.9 MB until the
// process exits.  All calls share it; it keeps the last call's contents.
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(Scratch)];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
Scratch* g_ptr[kMaxDevices] = {};

// Device address of the scratch for the current device, looked up once per
// device (the array's name is only a host-side stand-in).
int scratch_for(int device, Scratch** out) {
  if (device < 0 || device >= kMaxDevices) return S615_E_ARG;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return S615_E_DEVICE;
    }
    g_ptr[device] = static_cast<Scratch*>(p);
  }
  *out = g_ptr[device];
  return S615_OK;
}

}  // namespace

}  // namespace s615

using namespace s615;

extern "C" int s615_cls5_run_noalloc(s615_ctx* ctx, int table_id, const s615_unit* units, size_t n,
                                     unsigned flags, s615_hit* hits, size_t hit_cap, size_t* n_hits,
                                     s615_counters* counters) {
  if (!ctx || (n && !units) || (flags & ~S615_F_NO_GATE)) return S615_E_ARG;
  if (n > kMaxUnits) return S615_E_ARG;
  if (serving_blocks(ctx)) return S615_E_BUSY;   // the request loop owns the context
  auto it = ctx->tables.find(table_id);
  if (it == ctx->tables.end()) return S615_E_NOTABLE;
  S615_CU(cudaSetDevice(ctx->device));
  Scratch* S = nullptr;
  int s = scratch_for(ctx->device, &S);
  if (s) return s;
  cudaStream_t st = ctx->stream;

  // Rows per work item, by the rule s615_run uses: the autotuned choice for
  // this batch size if there is one, else 64 rows, or 32 / 16 when 64-row
  // items would give fewer than about 40 warps per SM.  A size whose items
  // would not fit the scratch falls back to longer items.
  u64 items_at[3] = {0, 0, 0};   // items with 64, 32 and 16 rows
  for (size_t i = 0; i < n; ++i) {
    if (units[i].cls != 5) return S615_E_FORMAT;
    DevUnit d;
    bool skip = false;
    if ((s = make_dev_unit(units[i], (u32)i, &d, &skip))) return s;
    if (skip) continue;
    for (u32 ie = 0; ie < d.nres1; ++ie) {
      u32 jmin = 0, jend = 0;
      class_rows(d.res1[ie], d.mod1, d.fmax1, &jmin, &jend);
      const u32 rows = jend > jmin ? jend - jmin : 0;
      for (int k = 0; k < 3; ++k) items_at[k] += (rows + (kItemRows >> k) - 1) / (kItemRows >> k);
    }
  }
  u32 bucket = 0;
  while (bucket < 39 && (2ull << bucket) <= n) ++bucket;
  const auto& tuned = ctx->tune[bucket];
  u32 unit_rows = kItemRows;
  if (tuned.item_rows) {
    unit_rows = tuned.item_rows;
  } else {
    const u64 want_items = (u64)ctx->num_sms * 40;
    while (unit_rows > 16 && items_at[unit_rows == 64 ? 0 : 1] < want_items) unit_rows /= 2;
  }
  while (unit_rows < kItemRows &&
         items_at[unit_rows == 32 ? 1 : unit_rows == 16 ? 2 : 0] > kMaxItems)
    unit_rows *= 2;

  // Unit records and work items, staged through small stack buffers (the
  // pageable copies have consumed a buffer by the time they return).
  DevUnit ustage[32];
  u64 istage[256];
  size_t nu = 0, ni = 0, us = 0, is = 0;
  auto flush_units = [&]() -> int {
    if (!us) return S615_OK;
    S615_CU(cudaMemcpyAsync(S->units + nu - us, ustage, us * sizeof(DevUnit),
                            cudaMemcpyHostToDevice, st));
    us = 0;
    return S615_OK;
  };
  auto flush_items = [&]() -> int {
    if (!is) return S615_OK;
    S615_CU(cudaMemcpyAsync(S->items + ni - is, istage, is * sizeof(u64), cudaMemcpyHostToDevice, st));
    is = 0;
    return S615_OK;
  };
  for (size_t i = 0; i < n; ++i) {
    DevUnit d;
    bool skip = false;
    if ((s = make_dev_unit(units[i], (u32)i, &d, &skip))) return s;
    if (skip) continue;
    for (u32 ie = 0; ie < d.nres1; ++ie) {
      u32 jmin = 0, jend = 0;
      class_rows(d.res1[ie], d.mod1, d.fmax1, &jmin, &jend);
      const u32 rows = jend > jmin ? jend - jmin : 0;
      for (u32 c = 0; c * unit_rows < rows; ++c) {
        if (ni == kMaxItems) return S615_E_ARG;
        istage[is++] = make_item((u32)nu, ie, c);
        ++ni;
        if (is == sizeof istage / sizeof istage[0] && (s = flush_items())) return s;
      }
    }
    ustage[us++] = d;
    ++nu;
    if (us == sizeof ustage / sizeof ustage[0] && (s = flush_units())) return s;
  }
  if ((s = flush_units()) || (s = flush_items())) return s;

  // Counters and the queue cursor must start at zero on every call.
  S615_CU(cudaMemsetAsync(&S->ctr, 0, sizeof S->ctr, st));
  S615_CU(cudaMemsetAsync(&S->work, 0, sizeof S->work, st));
  s615_batch b;   // a view of the scratch; its vectors stay empty
  b.n_units = nu;
  b.n_items = ni;
  b.n_main = ni;   // class 5 only: every item is for k_peel
  b.d_units = S->units;
  b.d_items = S->items;
  b.d_hits = S->hits;
  b.hit_cap = (u32)kMaxHits;
  b.d_ctr = &S->ctr;
  b.d_work = &S->work;
  b.item_rows = unit_rows;
  b.blocks_per_sm = tuned.blocks_per_sm;
  if ((s = launch_peel(ctx, view_of(it->second), &b, flags, st, 0))) return s;

  Cls5Counters c{};
  S615_CU(cudaMemcpyAsync(&c, &S->ctr, sizeof c, cudaMemcpyDeviceToHost, st));
  S615_CU(cudaStreamSynchronize(st));
  const size_t nh = (size_t)c.hits;
  const size_t take = std::min(nh, std::min(hit_cap, kMaxHits));
  if (take && hits) {
    S615_CU(cudaMemcpyAsync(hits, S->hits, take * sizeof(s615_hit), cudaMemcpyDeviceToHost, st));
    S615_CU(cudaStreamSynchronize(st));
  }
  if (n_hits) *n_hits = nh;
  if (counters) {
    counters->calls = c.calls;
    counters->probes = c.probes;
    counters->pos = c.pos;
    counters->gated = c.pos - c.probes;
    counters->hits = c.hits;
    counters->tri_total = 0;
    counters->tri_skipped = 0;
  }
  return (nh > kMaxHits || nh > hit_cap) ? S615_E_OVERFLOW : S615_OK;
}
