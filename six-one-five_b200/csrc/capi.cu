// capi.cu -- the C ABI (include/s615.h): context, tables, cls5 runs, verify.
//
// Host orchestration replacing run_cls5_gpu / acquire_xor_filter
// (fourcore_cls5_gpu_v4.cu:412-594) and the table I/O of
// fourcore_xor_store.hpp:54-181.  Differences by design: every call returns a
// status instead of exiting; the table stays resident across calls; a whole
// batch of units is one persistent launch instead of one launch and one
// device-wide sync per 16 units; a full hit buffer is reported
// (S615_E_OVERFLOW) instead of silently truncated.
#include <cuda_runtime.h>
#include <sched.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <random>
#include <thread>
#include <vector>

#include "engine.hpp"

using namespace s615;

namespace s615 {

int cuda_status(cudaError_t e) {
  if (e == cudaErrorMemoryAllocation) return S615_E_OOM;
  return e == cudaSuccess ? S615_OK : S615_E_DEVICE;
}

// A failed allocation gives back s615_run's kept batch, if it holds one that
// no run is using, and tries once more.
int dev_alloc(s615_ctx* ctx, void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) bytes = 16;
  for (int attempt = 0;; ++attempt) {
    // reserve the bytes against the budget first, so that threads allocating
    // at once cannot overrun it together
    bool reserved = false;
    size_t cur = ctx->used.load();
    while (!ctx->budget || cur + bytes <= ctx->budget) {
      if (ctx->used.compare_exchange_weak(cur, cur + bytes)) {
        reserved = true;
        break;
      }
    }
    if (reserved) {
      if (cudaMalloc(p, bytes) == cudaSuccess) return S615_OK;
      cudaGetLastError();
      *p = nullptr;
      ctx->used.fetch_sub(bytes);
    }
    if (attempt > 0 || !release_run_batch(ctx)) return S615_E_OOM;
  }
}

void dev_free(s615_ctx* ctx, void* p, size_t bytes) {
  if (!p) return;
  if (bytes == 0) bytes = 16;
  cudaFree(p);
  size_t cur = ctx->used.load();
  while (!ctx->used.compare_exchange_weak(cur, cur - std::min(cur, bytes))) {
  }
}

bool release_run_batch(s615_ctx* ctx) {
  bool any = false;
  if (ctx->run_batch && !ctx->run_busy) {
    s615_batch* b = ctx->run_batch;
    ctx->run_batch = nullptr;
    s615_batch_free(ctx, b);
    any = true;
  }
  {
    std::lock_guard<std::mutex> lock(ctx->pool_mu);
    any = any || !ctx->pool.empty();
  }
  pool_release(ctx);
  return any;
}

// Batch buffers.  A freed batch's device buffers go to a pool on the context
// (at most kPoolBytes and kPoolBuffers), and the next batch takes the
// smallest pooled buffer that holds its request and is at most twice as large,
// so a caller that prepares and frees batch after batch allocates and frees
// no device memory once the pool holds its sizes.  The pool is given back
// with s615_run's kept batch: when a table is built or loaded, when an
// allocation runs out of room, and on s615_close.
constexpr size_t kPoolBytes = size_t(8) << 30;
constexpr size_t kPoolBuffers = 64;

int pool_get(s615_ctx* ctx, size_t bytes, void** p, size_t* got) {
  {
    std::lock_guard<std::mutex> lock(ctx->pool_mu);   // never held across dev_alloc
    size_t best = 0;
    for (size_t i = 0; i < ctx->pool.size(); ++i) {
      const size_t sz = ctx->pool[i].second;
      if (sz >= bytes && sz <= 2 * std::max<size_t>(bytes, 4096) &&
          (best == 0 || sz < ctx->pool[best - 1].second))
        best = i + 1;
    }
    if (best) {
      *p = ctx->pool[best - 1].first;
      *got = ctx->pool[best - 1].second;
      ctx->pool_bytes -= *got;
      ctx->pool.erase(ctx->pool.begin() + (best - 1));
      return S615_OK;
    }
  }
  *got = bytes;
  return dev_alloc(ctx, p, bytes);
}

void pool_put(s615_ctx* ctx, void* p, size_t bytes) {
  if (!p) return;
  {
    std::lock_guard<std::mutex> lock(ctx->pool_mu);
    if (ctx->pool.size() < kPoolBuffers && ctx->pool_bytes + bytes <= kPoolBytes) {
      ctx->pool.emplace_back(p, bytes);
      ctx->pool_bytes += bytes;
      return;
    }
  }
  dev_free(ctx, p, bytes);
}

void pool_release(s615_ctx* ctx) {
  std::vector<std::pair<void*, size_t>> all;
  {
    std::lock_guard<std::mutex> lock(ctx->pool_mu);
    all.swap(ctx->pool);
    ctx->pool_bytes = 0;
  }
  for (auto& e : all) dev_free(ctx, e.first, e.second);
}

void* stage_get(HostStage& s, size_t bytes) {
  if (bytes <= s.bytes) return s.p;
  stage_free(s);
  const size_t want = std::max<size_t>(bytes + bytes / 4, size_t(1) << 20);
  if (cudaMallocHost(&s.p, want) == cudaSuccess) {
    s.pinned = true;
  } else {
    cudaGetLastError();
    s.p = ::operator new(want, std::nothrow);
    s.pinned = false;
    if (!s.p) return nullptr;
  }
  s.bytes = want;
  return s.p;
}

void stage_free(HostStage& s) {
  if (s.p) {
    if (s.pinned) cudaFreeHost(s.p);
    else ::operator delete(s.p);
  }
  s = HostStage{};
}

bool gate_product_matches();

}  // namespace s615

namespace {

void free_table(s615_ctx* ctx, DevTable& t) {
  for (DevTable& p : t.parts) free_table(ctx, p);
  t.parts.clear();
  dev_free(ctx, t.d_views, t.d_views ? sizeof(TableView) * 64 : 0);
  t.d_views = nullptr;
  dev_free(ctx, t.d_cells, t.bytes);
  t.d_cells = nullptr;
  t.bytes = 0;
}

// Device bytes of a table or of every shard of a set.
size_t table_bytes(const DevTable& t) {
  size_t b = t.bytes;
  for (const DevTable& p : t.parts) b += p.bytes;
  return b;
}

// A shard set over parts (shards 0..S-1 of one N and r): header totals, the
// parts' views uploaded for the routed probe.
int make_set(s615_ctx* ctx, std::vector<DevTable>&& parts, u32 S, u32 lo, DevTable* out) {
  DevTable t;
  t.hdr = parts[0].hdr;
  t.hdr.n_keys = 0;
  t.hdr.m_cells = 0;
  t.hdr.mix_seed = kShardSeed;   // a set's header carries the routing seed
  t.hdr.shard_count = S;
  t.hdr.shard_index = lo;   // the first shard held
  t.hdr.shard_mode = 0;
  t.shard_lo = lo;
  for (const DevTable& p : parts) {
    t.hdr.n_keys += p.hdr.n_keys;
    t.hdr.m_cells += p.hdr.m_cells;
  }
  t.layout = parts[0].layout;
  t.cell_bytes = parts[0].cell_bytes;
  t.parts = std::move(parts);
  std::vector<TableView> views(S);   // shards not held keep an empty view
  for (size_t i = 0; i < t.parts.size(); ++i) views[lo + i] = view_of(t.parts[i]);
  void* d = nullptr;
  int s = dev_alloc(ctx, &d, sizeof(TableView) * 64);   // S <= 64
  if (s) { free_table(ctx, t); return s; }
  t.d_views = d;
  if (cudaMemcpy(d, views.data(), views.size() * sizeof(TableView), cudaMemcpyHostToDevice) !=
      cudaSuccess) {
    free_table(ctx, t);
    return S615_E_DEVICE;
  }
  *out = std::move(t);
  return S615_OK;
}

DevTable* find_table(s615_ctx* ctx, int id) {
  auto it = ctx->tables.find(id);
  return it == ctx->tables.end() ? nullptr : &it->second;
}

int add_table(s615_ctx* ctx, DevTable t, int* id) {
  const int k = ctx->next_table++;
  ctx->tables[k] = t;
  if (id) *id = k;
  return S615_OK;
}

bool header_ok(const s615_header& h) {  // store_header.hpp:39-42 plus kind == Xor
  return h.magic == kMagic && h.version == kVersion && h.shard_count >= 1 &&
         h.shard_index < h.shard_count && h.r > 0 && h.r <= 64 && h.kind == 1;
}

// Choose the HBM layout of a table with m cells of r bits.
int pick_layout(s615_ctx* ctx, int want, u64 m, u32 r, int* cell_bytes) {
  *cell_bytes = r <= 32 ? 4 : 8;
  if (want == S615_LAYOUT_PACKED) { *cell_bytes = 0; return S615_LAYOUT_PACKED; }
  if (want == S615_LAYOUT_WIDE) return S615_LAYOUT_WIDE;
  release_run_batch(ctx);   // a table needs the room more than s615_run's kept buffers
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const size_t wide = m * (size_t)(*cell_bytes) + packed_bytes(m, r) + ((size_t)4 << 30);
  const size_t room = std::min(free_b, ctx->budget ? ctx->budget - std::min(ctx->budget, ctx->used.load()) : free_b);
  if (wide <= room) return S615_LAYOUT_WIDE;
  *cell_bytes = 0;
  return S615_LAYOUT_PACKED;
}

// Turn a device buffer holding packed bytes into the chosen layout.
int finish_upload(s615_ctx* ctx, DevTable& t, void* d_packed, size_t packed_alloc, int layout,
                  int cell_bytes) {
  if (layout == S615_LAYOUT_PACKED) {
    t.layout = S615_LAYOUT_PACKED; t.cell_bytes = 0;
    t.d_cells = d_packed; t.bytes = packed_alloc;
    return S615_OK;
  }
  void* wide = nullptr;
  const size_t wb = t.hdr.m_cells * (size_t)cell_bytes;
  int s = dev_alloc(ctx, &wide, wb);
  if (s) { dev_free(ctx, d_packed, packed_alloc); return s; }
  s = launch_unpack(ctx, static_cast<const u8*>(d_packed), t.hdr.m_cells, t.hdr.r, wide, cell_bytes,
                    ctx->stream);
  const cudaError_t e = cudaStreamSynchronize(ctx->stream);
  dev_free(ctx, d_packed, packed_alloc);
  if (s || e != cudaSuccess) { dev_free(ctx, wide, wb); return s ? s : cuda_status(e); }
  t.layout = S615_LAYOUT_WIDE; t.cell_bytes = cell_bytes;
  t.d_cells = wide; t.bytes = wb;
  return S615_OK;
}

}  // namespace

// ======================================================================= ABI
namespace s615 {

int l2_window(s615_ctx* ctx, const TableView& tv, unsigned flags, cudaLaunchAttribute* attr) {
  if ((flags & S615_F_NO_L2_WINDOW) || !ctx->l2_persist_max || !ctx->l2_window_max) return 0;
  const void* base = nullptr;
  size_t bytes = 0;
  if (tv.shards <= 1 && tv.cells && tv.bytes && tv.bytes <= ctx->l2_persist_max &&
      tv.bytes <= ctx->l2_window_max) {
    base = tv.cells;   // the whole table stays in L2
    bytes = tv.bytes;
  } else {
    base = ctx->d_pat;   // only the gate patterns (the table streams through L2)
    bytes = (4 * kPatWords + kTriWords + 2 * kSharpWords) * sizeof(u32);
  }
  if (ctx->l2_limit < bytes) {   // reserve the set-aside once (this process only)
    const size_t want = ctx->l2_persist_max;
    if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    ctx->l2_limit = want;
  }
  attr->id = cudaLaunchAttributeAccessPolicyWindow;
  attr->val.accessPolicyWindow.base_ptr = const_cast<void*>(base);
  attr->val.accessPolicyWindow.num_bytes = bytes;
  attr->val.accessPolicyWindow.hitRatio = 1.0f;
  attr->val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
  attr->val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
  return 1;
}

}  // namespace s615

extern "C" {

const char* s615_strerror(int s) {
  switch (s) {
    case S615_OK: return "ok";
    case S615_E_ARG: return "bad argument";
    case S615_E_IO: return "i/o error";
    case S615_E_FORMAT: return "bad format";
    case S615_E_N_MISMATCH: return "table N mismatch";
    case S615_E_FPR_SMOKE: return "xor FPR smoke too high";
    case S615_E_OOM: return "out of device memory / HBM budget";
    case S615_E_DEVICE: return "CUDA error";
    case S615_E_TIMEOUT: return "device wait timed out";
    case S615_E_OVERFLOW: return "result buffer overflow";
    case S615_E_BUILD: return "xor peel stalled for every seed";
    case S615_E_NOTABLE: return "unknown table id";
    case S615_E_BUSY: return "context is serving";
  }
  return "unknown status";
}

int s615_open(int device, size_t hbm_budget, s615_ctx** out) {
  if (!out) return S615_E_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return S615_E_DEVICE;
  }
  std::unique_ptr<s615_ctx> ctx(new s615_ctx());
  ctx->device = device;
  S615_CU(cudaSetDevice(device));
  S615_CU(cudaFree(nullptr));
  S615_CU(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  S615_CU(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device));
  int l2p = 0, l2w = 0;
  if (cudaDeviceGetAttribute(&l2p, cudaDevAttrMaxPersistingL2CacheSize, device) != cudaSuccess ||
      cudaDeviceGetAttribute(&l2w, cudaDevAttrMaxAccessPolicyWindowSize, device) != cudaSuccess) {
    cudaGetLastError();
    l2p = l2w = 0;
  }
  ctx->l2_persist_max = (size_t)(l2p > 0 ? l2p : 0);
  ctx->l2_window_max = (size_t)(l2w > 0 ? l2w : 0);
  size_t free_b = 0, total_b = 0;
  S615_CU(cudaMemGetInfo(&free_b, &total_b));
  ctx->budget = hbm_budget ? hbm_budget : total_b;
  // gate pattern sets: [gate cls5 | open cls5 | gate find3 | open find3],
  // then the triple-sum gate block of the (6,1,7) kernel
  std::vector<u32> pat(4 * kPatWords + kTriWords + 2 * kSharpWords);
  gate_patterns(true, 0, pat.data());
  gate_patterns(false, 0, pat.data() + kPatWords);
  gate_patterns(true, 1, pat.data() + 2 * kPatWords);
  gate_patterns(false, 1, pat.data() + 3 * kPatWords);
  tri_tables(pat.data() + 4 * kPatWords);
  gate_patterns_sharp(0, pat.data() + 4 * kPatWords + kTriWords);
  gate_patterns_sharp(1, pat.data() + 4 * kPatWords + kTriWords + kSharpWords);
  void* p = nullptr;
  const int s = dev_alloc(ctx.get(), &p, pat.size() * sizeof(u32));
  if (s) return s;
  ctx->d_pat = static_cast<u32*>(p);
  ctx->d_tri = ctx->d_pat + 4 * kPatWords;
  ctx->d_sharp = ctx->d_tri + kTriWords;
  ctx->p64 = pair_sums_mask64();
  S615_CU(cudaMemcpy(ctx->d_pat, pat.data(), pat.size() * sizeof(u32), cudaMemcpyHostToDevice));
  *out = ctx.release();
  return S615_OK;
}

int s615_close(s615_ctx* ctx) {
  if (!ctx) return S615_E_ARG;
  cudaSetDevice(ctx->device);
  server_destroy(ctx);
  ctx->run_busy = false;
  release_run_batch(ctx);
  stage_free(ctx->unit_stage);
  for (int k = 0; k < 4; ++k) dev_free(ctx, ctx->arena[k], ctx->arena_cap[k]);
  dev_free(ctx, ctx->d_roots, ctx->roots_bytes);
  for (auto& kv : ctx->tables) free_table(ctx, kv.second);
  ctx->tables.clear();
  dev_free(ctx, ctx->d_pat, (4 * kPatWords + kTriWords + 2 * kSharpWords) * sizeof(u32));
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return S615_OK;
}

uint64_t s615_launch_count(s615_ctx* ctx) { return ctx ? ctx->launches : 0; }

int s615_checked_build(void) {
#ifdef S615_CHECKED
  return 1;
#else
  return 0;
#endif
}

int s615_check_flags(s615_ctx* ctx, uint32_t* flags) {
  if (!ctx || !flags) return S615_E_ARG;
  cudaSetDevice(ctx->device);
  S615_CU(cudaDeviceSynchronize());   // the kernels that may have set a flag are done
  *flags = check_take_peel() | check_take_peel617() | check_take_table() | check_take_xor_build();
  return S615_OK;
}

int s615_set_budget(s615_ctx* ctx, size_t hbm_budget) {
  if (!ctx) return S615_E_ARG;
  if (serving_blocks(ctx)) return S615_E_BUSY;
  size_t free_b = 0, total_b = 0;
  cudaSetDevice(ctx->device);
  S615_CU(cudaMemGetInfo(&free_b, &total_b));
  ctx->budget = hbm_budget ? hbm_budget : total_b;
  return S615_OK;
}

int s615_get_table_info(s615_ctx* ctx, int id, s615_table_info* info) {
  if (!ctx || !info) return S615_E_ARG;
  DevTable* t = find_table(ctx, id);
  if (!t) return S615_E_NOTABLE;
  info->hdr = t->hdr;
  info->layout = t->layout;
  info->cell_bytes = t->cell_bytes;
  info->device_bytes = table_bytes(*t);
  return S615_OK;
}

int s615_free_table(s615_ctx* ctx, int id) {
  if (!ctx) return S615_E_ARG;
  if (serving_blocks(ctx)) return S615_E_BUSY;
  DevTable* t = find_table(ctx, id);
  if (!t) return S615_E_NOTABLE;
  cudaSetDevice(ctx->device);
  free_table(ctx, *t);
  ctx->tables.erase(id);
  return S615_OK;
}

int s615_xor_query_dev(s615_ctx* ctx, int id, const uint64_t* d_keys, size_t n, uint8_t* d_out,
                       void* stream) {
  if (!ctx) return S615_E_ARG;
  DevTable* t = find_table(ctx, id);
  if (!t) return S615_E_NOTABLE;
  return launch_xor_query(ctx, view_of(*t), d_keys, n, d_out,
                          stream ? static_cast<cudaStream_t>(stream) : ctx->stream);
}

int s615_xor_query(s615_ctx* ctx, int id, const uint64_t* keys, size_t n, uint8_t* out) {
  if (!ctx || (n && (!keys || !out))) return S615_E_ARG;
  DevTable* t = find_table(ctx, id);
  if (!t) return S615_E_NOTABLE;
  if (n == 0) return S615_OK;
  cudaSetDevice(ctx->device);
  const size_t chunk = std::min<size_t>(n, (size_t)1 << 26);
  void *dk = nullptr, *dout = nullptr;
  int s = dev_alloc(ctx, &dk, chunk * 8);
  if (s) return s;
  if ((s = dev_alloc(ctx, &dout, chunk))) { dev_free(ctx, dk, chunk * 8); return s; }
  const TableView tv = view_of(*t);
  for (size_t off = 0; off < n && !s; off += chunk) {
    const size_t c = std::min(chunk, n - off);
    cudaError_t e = cudaMemcpyAsync(dk, keys + off, c * 8, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) s = launch_xor_query(ctx, tv, static_cast<const u64*>(dk), c,
                                               static_cast<u8*>(dout), ctx->stream);
    if (e == cudaSuccess && !s) e = cudaMemcpyAsync(out + off, dout, c, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && !s) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) s = cuda_status(e);
  }
  dev_free(ctx, dk, chunk * 8);
  dev_free(ctx, dout, chunk);
  return s;
}

// xor_fpr_smoke (fourcore_xor_store.hpp:54-65): 200k keys x <- x*phi + 1 from
// 0x123456789abcdef0 through the device query; the number of hits.
int s615_fpr_smoke(s615_ctx* ctx, int id, int* hits) {
  if (!ctx || !hits) return S615_E_ARG;
  DevTable* t = find_table(ctx, id);
  if (!t) return S615_E_NOTABLE;
  *hits = 200000;
  if (t->parts.empty() && (t->hdr.m_cells < 3 || t->hdr.r == 0 || !t->d_cells)) return S615_OK;
  const size_t n = 200000;
  std::vector<u64> keys(n);
  u64 x = 0x123456789abcdef0ULL;
  for (size_t i = 0; i < n; ++i) { x = x * kPhi + 1; keys[i] = x; }
  std::vector<u8> out(n);
  const int s = s615_xor_query(ctx, id, keys.data(), n, out.data());
  if (s) return s;
  int c = 0;
  for (u8 v : out) c += v;
  *hits = c;
  return S615_OK;
}

// Refuse more than 16 hits (fourcore_cls5_gpu_v4.cu:576-579).
static int smoke_table(s615_ctx* ctx, int id) {
  int hits = 0;
  const int s = s615_fpr_smoke(ctx, id, &hits);
  if (s) return s;
  return hits > 16 ? S615_E_FPR_SMOKE : S615_OK;
}

// Read one table file into HBM (header checks, streamed upload, layout).
static int load_part(s615_ctx* ctx, const char* path, int expected_N, int layout, DevTable* out) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return S615_E_IO;
  DevTable& t = *out;
  if (std::fread(&t.hdr, sizeof t.hdr, 1, f) != 1) { std::fclose(f); return S615_E_IO; }
  if (!header_ok(t.hdr)) { std::fclose(f); return S615_E_FORMAT; }
  if (expected_N > 0 && (int)t.hdr.N != expected_N) { std::fclose(f); return S615_E_N_MISMATCH; }
  const u64 len = packed_bytes(t.hdr.m_cells, t.hdr.r);
  const size_t alloc = ((len + 7) / 8 + 1) * 8;
  int cell_bytes = 0;
  const int lay = pick_layout(ctx, layout, t.hdr.m_cells, t.hdr.r, &cell_bytes);
  void* d = nullptr;
  int s = dev_alloc(ctx, &d, alloc);
  if (s) { std::fclose(f); return s; }
  cudaMemsetAsync(d, 0, alloc, ctx->stream);
  // Stream the file through two pinned staging buffers.
  const size_t stage = (size_t)64 << 20;
  void* pin[2] = {nullptr, nullptr};
  cudaEvent_t ev[2];
  bool ok = cudaMallocHost(&pin[0], stage) == cudaSuccess && cudaMallocHost(&pin[1], stage) == cudaSuccess;
  cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
  cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
  u64 done = 0;
  int k = 0;
  while (ok && done < len) {
    const size_t c = (size_t)std::min<u64>(stage, len - done);
    cudaEventSynchronize(ev[k]);
    if (std::fread(pin[k], 1, c, f) != c) { ok = false; s = S615_E_IO; break; }
    if (cudaMemcpyAsync(static_cast<u8*>(d) + done, pin[k], c, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) {
      ok = false; s = S615_E_DEVICE; break;
    }
    cudaEventRecord(ev[k], ctx->stream);
    done += c;
    k ^= 1;
  }
  cudaStreamSynchronize(ctx->stream);
  std::fclose(f);
  for (int i = 0; i < 2; ++i) { if (pin[i]) cudaFreeHost(pin[i]); cudaEventDestroy(ev[i]); }
  if (!ok) { dev_free(ctx, d, alloc); return s ? s : S615_E_OOM; }
  return finish_upload(ctx, t, d, alloc, lay, cell_bytes);
}

int s615_load_table(s615_ctx* ctx, const char* path, int expected_N, int layout, int* table_id) {
  NvtxRange nvtx("s615_load_table");
  if (!ctx || !path) return S615_E_ARG;
  if (serving_blocks(ctx)) return S615_E_BUSY;
  cudaSetDevice(ctx->device);
  DevTable t;
  int s = load_part(ctx, path, expected_N, layout, &t);
  if (s) return s;
  if (t.hdr.shard_count != 1) { free_table(ctx, t); return S615_E_FORMAT; }   // one shard of a set
  int id = 0;
  add_table(ctx, t, &id);
  if ((s = smoke_table(ctx, id))) { s615_free_table(ctx, id); return s; }
  if (table_id) *table_id = id;
  return S615_OK;
}

int s615_load_table_shards(s615_ctx* ctx, const char* const* paths, int n, int expected_N,
                           int layout, int* table_id) {
  if (!ctx || !paths || n < 1 || n > 64) return S615_E_ARG;
  if (serving_blocks(ctx)) return S615_E_BUSY;
  cudaSetDevice(ctx->device);
  std::vector<DevTable> parts;
  int s = S615_OK;
  for (int k = 0; k < n && !s; ++k) {
    DevTable t;
    if (!paths[k]) { s = S615_E_ARG; break; }
    s = load_part(ctx, paths[k], expected_N, layout, &t);
    if (s) break;
    // consecutive shards of one S (all of them, or the range a rank holds),
    // mode key % S, and one N and r for the whole set
    const s615_header& h = t.hdr;
    const bool first_ok = k || (h.shard_count >= 2 && h.shard_count <= 64 &&
                                (int)(h.shard_count - h.shard_index) >= n);
    if (!first_ok || h.shard_mode != 0 ||
        (k && (h.shard_count != parts[0].hdr.shard_count ||
               h.shard_index != parts[0].hdr.shard_index + (u32)k || h.N != parts[0].hdr.N ||
               h.r != parts[0].hdr.r))) {
      free_table(ctx, t);
      s = S615_E_FORMAT;
      break;
    }
    parts.push_back(std::move(t));
  }
  if (s) {
    for (DevTable& p : parts) free_table(ctx, p);
    return s;
  }
  const u32 S = parts[0].hdr.shard_count, lo = parts[0].hdr.shard_index;
  DevTable set;
  if ((s = make_set(ctx, std::move(parts), S, lo, &set))) return s;
  int id = 0;
  add_table(ctx, std::move(set), &id);
  if ((s = smoke_table(ctx, id))) { s615_free_table(ctx, id); return s; }
  if (table_id) *table_id = id;
  return S615_OK;
}

// The packed file bytes of a resident table into buf (len bytes).
static int export_packed(s615_ctx* ctx, const DevTable& t, u8* buf, u64 len) {
  if (!len) return S615_OK;
  if (t.layout == S615_LAYOUT_PACKED) {
    S615_CU(cudaMemcpy(buf, t.d_cells, len, cudaMemcpyDeviceToHost));
    return S615_OK;
  }
  void* pk = nullptr;
  const size_t pb = ((len + 7) / 8 + 1) * 8;
  int s = dev_alloc(ctx, &pk, pb);
  if (s) return s;
  s = launch_pack(ctx, t.d_cells, t.cell_bytes, t.hdr.m_cells, t.hdr.r, static_cast<u8*>(pk), len,
                  ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (!s && e == cudaSuccess) e = cudaMemcpy(buf, pk, len, cudaMemcpyDeviceToHost);
  dev_free(ctx, pk, pb);
  if (s) return s;
  return cuda_status(e);
}

int s615_export_table(s615_ctx* ctx, int id, s615_header* hdr, uint8_t* buf, size_t cap,
                      size_t* len) {
  if (!ctx) return S615_E_ARG;
  DevTable* t = find_table(ctx, id);
  if (!t) return S615_E_NOTABLE;
  if (!t->parts.empty()) return S615_E_ARG;   // a set: export or save its shards one by one
  cudaSetDevice(ctx->device);
  const u64 n = packed_bytes(t->hdr.m_cells, t->hdr.r);
  if (hdr) *hdr = t->hdr;
  if (len) *len = n;
  if (!buf) return S615_OK;
  if (cap < n) return S615_E_OVERFLOW;
  return export_packed(ctx, *t, buf, n);
}

static int save_part(s615_ctx* ctx, const DevTable* t, const char* path);

int s615_save_table(s615_ctx* ctx, int id, const char* path) {
  if (!ctx || !path) return S615_E_ARG;
  DevTable* t = find_table(ctx, id);
  if (!t) return S615_E_NOTABLE;
  if (!t->parts.empty()) return S615_E_ARG;
  cudaSetDevice(ctx->device);
  return save_part(ctx, t, path);
}

int s615_set_probe_groups(s615_ctx* ctx, int id, int groups) {
  if (!ctx) return S615_E_ARG;
  if (serving_blocks(ctx)) return S615_E_BUSY;
  DevTable* t = find_table(ctx, id);
  if (!t) return S615_E_NOTABLE;
  if (t->parts.empty() || groups < 0 || groups > (int)t->parts.size()) return S615_E_ARG;   // <= shards held
  t->groups = (u32)groups;
  return S615_OK;
}

int s615_save_table_shard(s615_ctx* ctx, int id, int shard, const char* path) {
  if (!ctx || !path) return S615_E_ARG;
  DevTable* t = find_table(ctx, id);
  if (!t) return S615_E_NOTABLE;
  const int i = shard - (int)t->shard_lo;   // shard numbers are the set's own
  if (t->parts.empty() || i < 0 || i >= (int)t->parts.size()) return S615_E_ARG;
  cudaSetDevice(ctx->device);
  return save_part(ctx, &t->parts[(size_t)i], path);
}

// One table's file: its header, then the packed cells.
static int save_part(s615_ctx* ctx, const DevTable* t, const char* path) {
  const u64 len = packed_bytes(t->hdr.m_cells, t->hdr.r);
  std::vector<u8> host(len);
  const int s = export_packed(ctx, *t, host.data(), len);
  if (s) return s;
  FILE* f = std::fopen(path, "wb");
  if (!f) return S615_E_IO;
  bool ok = std::fwrite(&t->hdr, sizeof t->hdr, 1, f) == 1;
  if (ok && len) ok = std::fwrite(host.data(), 1, len, f) == len;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? S615_OK : S615_E_IO;
}

int s615_build_table(s615_ctx* ctx, int N, int r, int layout, int* table_id) {
  NvtxRange nvtx("s615_build_table");
  if (!ctx || N < 1 || N > 4 * kNSoftMax || r < 8 || r > 64) return S615_E_ARG;
  if (serving_blocks(ctx)) return S615_E_BUSY;
  cudaSetDevice(ctx->device);
  // distinct values of i^6 mod 2^64 (many i collide 2-adically)
  std::vector<u64> vals((size_t)N);
  for (int i = 1; i <= N; ++i) { const u64 x2 = (u64)i * (u64)i; vals[i - 1] = x2 * x2 * x2; }
  std::sort(vals.begin(), vals.end());
  vals.erase(std::unique(vals.begin(), vals.end()), vals.end());
  void* dv = nullptr;
  int s = dev_alloc(ctx, &dv, vals.size() * 8);
  if (s) return s;
  S615_CU(cudaMemcpy(dv, vals.data(), vals.size() * 8, cudaMemcpyHostToDevice));
  u64 seeds[4];
  for (int o = 0; o < 4; ++o) seeds[o] = kSeedBase + (u64)o * kPhi;
  DevTable t;
  s = build_xor_device(ctx, static_cast<const u64*>(dv), vals.size(), nullptr, 0, r, seeds, 4, N,
                       layout == S615_LAYOUT_AUTO ? S615_LAYOUT_WIDE : layout, &t);
  dev_free(ctx, dv, vals.size() * 8);
  if (s) return s;
  int id = 0;
  add_table(ctx, t, &id);
  if ((s = smoke_table(ctx, id))) { s615_free_table(ctx, id); return s; }
  if (table_id) *table_id = id;
  return S615_OK;
}

int s615_build_table_sharded(s615_ctx* ctx, int N, int r, int shards, int layout, int* table_id) {
  return s615_build_table_shard_range(ctx, N, r, shards, 0, shards, layout, table_id);
}

int s615_build_table_shard_range(s615_ctx* ctx, int N, int r, int shards, int lo, int hi,
                                 int layout, int* table_id) {
  if (!ctx || N < 1 || N > 8 * kNSoftMax || r < 8 || r > 64 || shards < 2 || shards > 64 ||
      lo < 0 || hi > shards || lo >= hi)
    return S615_E_ARG;
  if (serving_blocks(ctx)) return S615_E_BUSY;
  cudaSetDevice(ctx->device);
  std::vector<u64> vals((size_t)N);
  for (int i = 1; i <= N; ++i) { const u64 x2 = (u64)i * (u64)i; vals[i - 1] = x2 * x2 * x2; }
  std::sort(vals.begin(), vals.end());
  vals.erase(std::unique(vals.begin(), vals.end()), vals.end());
  void* dv = nullptr;
  int s = dev_alloc(ctx, &dv, vals.size() * 8);
  if (s) return s;
  S615_CU(cudaMemcpy(dv, vals.data(), vals.size() * 8, cudaMemcpyHostToDevice));
  u64 seeds[4];
  for (int o = 0; o < 4; ++o) seeds[o] = kSeedBase + (u64)o * kPhi;
  std::vector<DevTable> parts;
  // one shard at a time: a build's scratch is sized for its shard's keys
  for (int k = lo; k < hi && !s; ++k) {
    DevTable t;
    s = build_xor_device(ctx, static_cast<const u64*>(dv), vals.size(), nullptr, 0, r, seeds, 4, N,
                         layout == S615_LAYOUT_AUTO ? S615_LAYOUT_WIDE : layout, &t, (u32)shards,
                         (u32)k);
    if (!s) parts.push_back(std::move(t));
  }
  dev_free(ctx, dv, vals.size() * 8);
  if (s) {
    for (DevTable& p : parts) free_table(ctx, p);
    return s;
  }
  DevTable set;
  if ((s = make_set(ctx, std::move(parts), (u32)shards, (u32)lo, &set))) return s;
  int id = 0;
  add_table(ctx, std::move(set), &id);
  if ((s = smoke_table(ctx, id))) { s615_free_table(ctx, id); return s; }
  if (table_id) *table_id = id;
  return S615_OK;
}

int s615_build_table_keys(s615_ctx* ctx, const uint64_t* keys, size_t n, int r, uint64_t base_seed,
                          int layout, int* table_id) {
  if (!ctx || (n && !keys) || r < 1 || r > 64) return S615_E_ARG;
  if (serving_blocks(ctx)) return S615_E_BUSY;
  cudaSetDevice(ctx->device);
  void* dk = nullptr;
  int s = dev_alloc(ctx, &dk, std::max<size_t>(n, 1) * 8);
  if (s) return s;
  if (n) S615_CU(cudaMemcpy(dk, keys, n * 8, cudaMemcpyHostToDevice));
  DevTable t;
  const u64 seed = base_seed;
  s = build_xor_device(ctx, nullptr, 0, static_cast<const u64*>(dk), n, r, &seed, 1, 0,
                       layout == S615_LAYOUT_AUTO ? S615_LAYOUT_WIDE : layout, &t);
  dev_free(ctx, dk, std::max<size_t>(n, 1) * 8);
  if (s) return s;
  return add_table(ctx, t, table_id);
}

int s615_mem_info(s615_ctx* ctx, size_t* free_b, size_t* total_b) {
  if (!ctx || !free_b || !total_b) return S615_E_ARG;
  cudaSetDevice(ctx->device);
  S615_CU(cudaMemGetInfo(free_b, total_b));
  return S615_OK;
}

int s615_unit_status(const s615_unit* unit) {
  if (!unit) return S615_E_ARG;
  DevUnit d;
  bool skip = false;
  const int s = make_dev_unit(*unit, 0, &d, &skip);
  if (s) return s;
  return skip ? 1 : S615_OK;
}

int s615_unit_candidates(uint64_t B, int cls, uint64_t* out, size_t cap, size_t* n) {
  if (!n || cls < 1 || cls > 5) return S615_E_ARG;
  const auto v = unit_candidates(B, cls);
  for (size_t i = 0; i < v.size() && i < cap; ++i) out[i] = v[i];
  *n = v.size();
  return v.size() > cap ? S615_E_OVERFLOW : S615_OK;
}

int s615_617_candidates(uint64_t B, s615_unit* out, size_t cap, size_t* n) {
  if (!n || B > 2353973ULL || (cap && !out)) return S615_E_ARG;
  const auto v = candidates617(B);
  for (size_t i = 0; i < v.size() && i < cap; ++i) {
    s615_unit x{};
    x.cls = S615_CLS_617;
    x.kind = 0;
    x.B = B;
    x.u = v[i].first;
    x.w = (uint32_t)v[i].second;
    out[i] = x;
  }
  *n = v.size();
  return v.size() > cap ? S615_E_OVERFLOW : S615_OK;
}

int s615_617_jobs(uint64_t B, int cls, s615_unit* out, size_t cap, size_t* n) {
  if (!n || B > 2353973ULL || cls < 1 || cls > 4 || (cap && !out)) return S615_E_ARG;
  const auto v = jobs617(B, cls);
  for (size_t i = 0; i < v.size() && i < cap; ++i) out[i] = v[i];
  *n = v.size();
  return v.size() > cap ? S615_E_OVERFLOW : S615_OK;
}

// ---------------------------------------------------------- peel batches
}  // extern "C"

namespace s615 {

int arena_get(s615_ctx* ctx, int k, size_t bytes, void** p) {
  if (bytes > ctx->arena_cap[k]) {
    // the outgrown buffer goes to the batch pool rather than to cudaFree,
    // whose device-wide sync (and occasional long stalls) would land on
    // whatever else is in flight, e.g. the serving loop's other slot
    pool_put(ctx, ctx->arena[k], ctx->arena_cap[k]);
    ctx->arena[k] = nullptr;
    ctx->arena_cap[k] = 0;
    void* q = nullptr;
    size_t got = 0;
    const int s = pool_get(ctx, std::max<size_t>(bytes + bytes / 4, 4096), &q, &got);
    if (s) return s;
    ctx->arena[k] = q;
    ctx->arena_cap[k] = got;
  }
  *p = ctx->arena[k];
  return S615_OK;
}

// Host threads for a pass over n units: one per 8,192 units, at most the
// CPUs the process may run on (and 32); one below 16,384 units.
static size_t host_threads(size_t n) {
  if (n < (1u << 14)) return 1;
  size_t hw = std::thread::hardware_concurrency();
  cpu_set_t set;   // the CPUs this process may run on, when fewer than the machine's
  if (sched_getaffinity(0, sizeof set, &set) == 0) hw = (size_t)CPU_COUNT(&set);
  return std::max<size_t>(1, std::min<size_t>({hw, 32, n / 8192}));
}

// Run work(t) for t in [0, nt) on nt threads (inline when nt == 1).  A range
// whose thread cannot be started (the process is out of threads) runs on the
// calling thread instead, so no exception leaves the C ABI.
template <class F>
static void run_threads(size_t nt, F&& work) {
  if (nt == 1) { work(0); return; }
  std::vector<std::thread> th;
  size_t t = 0;
  try {
    for (; t < nt; ++t) th.emplace_back(work, t);
  } catch (...) {
  }
  for (size_t k = t; k < nt; ++k) work(k);
  for (auto& x : th) x.join();
}

// make_dev_unit over every unit (on several host threads for large batches),
// the kept records compacted in unit order.  Returns the error of the
// lowest-index unit that has one, as a sequential pass would.
// One device record per input unit, in input order.  A unit the reference
// drops (u >= B, an empty residue class or window) stays in place as a class-0
// record that gets no work items, so no pass compacts the array.
static int pack_units(s615_ctx* ctx, const s615_unit* units, size_t n, DevUnit** out_p,
                      size_t* n_out) {
  DevUnit* out = static_cast<DevUnit*>(
      stage_get(ctx->unit_stage, std::max<size_t>(n, 1) * sizeof(DevUnit)));
  if (!out) return S615_E_OOM;
  *out_p = out;
  const size_t nt = host_threads(n);
  std::vector<int> err(nt, 0);
  auto work = [&](size_t t) {
    for (size_t i = n * t / nt, hi = n * (t + 1) / nt; i < hi; ++i) {
      bool skip = false;
      const int s = make_dev_unit(units[i], (u32)i, &out[i], &skip);
      if (s) { err[t] = s; return; }
      if (skip) out[i].cls = 0;
    }
  };
  run_threads(nt, work);
  for (size_t t = 0; t < nt; ++t)
    if (err[t]) return err[t];
  *n_out = n;
  return S615_OK;
}

int fill_batch(s615_ctx* ctx, const s615_unit* units, size_t n, s615_batch* b) {
  b->n_items = b->n_main = 0;
  DevUnit* du = nullptr;
  size_t nd = 0;
  {
    NvtxRange nvtx("pack units");
    if (const int s = pack_units(ctx, units, n, &du, &nd)) return s;
  }
  // Job rows per item: up to 64, fewer when the batch is small, so that its
  // items still fill the GPU (about 64 warps per SM).
  u32 job_rows = 8;
  while (job_rows < kJobRows && (u64)job_rows * ctx->num_sms * 64 < nd) job_rows *= 2;
  // Rows per class 2-5 item: 64, or 32 / 16 when a batch would otherwise
  // have fewer items than about 40 warps per SM (a small serving batch).
  const u64 want_items = (u64)ctx->num_sms * 40;
  u32 unit_rows = kItemRows;
  u32 bucket = 0;
  while (bucket < 39 && (2ull << bucket) <= n) ++bucket;
  const auto& tuned = ctx->tune[bucket];
  b->blocks_per_sm = ctx->force_bps ? ctx->force_bps : tuned.blocks_per_sm;
  if (ctx->force_rows || tuned.item_rows) {
    unit_rows = ctx->force_rows ? ctx->force_rows : tuned.item_rows;
  } else {
    while (unit_rows > 16) {
      u64 items = 0;
      for (size_t k = 0; k < nd && items < want_items; ++k) {
        const DevUnit& d = du[k];
        if (d.cls < 2 || d.cls > 5) continue;
        for (u32 ir = 0; ir < d.nres1; ++ir) {
          u32 jmin = 0, jend = 0;
          class_rows(d.res1[ir], d.mod1, d.fmax1, &jmin, &jend);
          if (jend > jmin) items += (jend - jmin + unit_rows - 1) / unit_rows;
        }
      }
      if (items >= want_items) break;
      unit_rows /= 2;
    }
  }
  b->item_rows = unit_rows;
  // a batch too small to fill the GPU even with 16-row items (a serving
  // request) also splits each class 2-4 row chunk four ways over its tiles
  b->parts3 = (!ctx->force_rows && !tuned.item_rows && unit_rows == 16) ? 4u : 1u;
  nvtxRangePushA("work items");
  // Work items unit by unit in input order, on several host threads for a
  // large batch: each thread counts its range's items, then writes them in
  // place.  Ranges are cut at multiples of job_rows, where a single pass
  // starts a new item too (consecutive job rows share items, but never across
  // such a multiple), so the items equal one sequential pass's.
  const size_t nt = host_threads(nd);
  std::vector<size_t> cut(nt + 1, nd);
  cut[0] = 0;
  for (size_t t = 1; t < nt; ++t)
    cut[t] = std::max(cut[t - 1], std::min(nd, nd * t / nt / job_rows * job_rows));
  // classes 1, 7 and 8 (c4 windows) run in the second kernel, after the others
  auto second = [](const DevUnit& d) {
    return d.cls == S615_CLS_617 || d.cls == 1 || d.cls == S615_CLS_617_FIND4;
  };
  std::vector<size_t> cnt_main(nt, 0), cnt_617(nt, 0);
  run_threads(nt, [&](size_t t) {
    ItemCount m, c;
    for (size_t k = cut[t]; k < cut[t + 1]; ++k) {
      const DevUnit& d = du[k];
      if (d.cls == 0) continue;   // dropped
      if (second(d)) unit_items(d, (u32)k, c, job_rows, unit_rows, b->parts3);
      else unit_items(d, (u32)k, m, job_rows, unit_rows, b->parts3);
    }
    cnt_main[t] = m.n;
    cnt_617[t] = c.n;
  });
  std::vector<size_t> at(nt + 1, 0), at617(nt + 1, 0);
  for (size_t t = 0; t < nt; ++t) at[t + 1] = at[t] + cnt_main[t];
  at617[0] = at[nt];
  for (size_t t = 0; t < nt; ++t) at617[t + 1] = at617[t] + cnt_617[t];
  const size_t total = at617[nt];
  if (total > b->host_items_cap) {
    b->host_items.reset();
    b->host_items_cap = 0;
    b->host_items.reset(new (std::nothrow) u64[std::max<size_t>(total, 1)]);
    if (!b->host_items) { nvtxRangePop(); return S615_E_OOM; }
    b->host_items_cap = std::max<size_t>(total, 1);
  }
  u64* items = b->host_items.get();
  run_threads(nt, [&](size_t t) {
    ItemWriter m, c;
    m.p = items + at[t];
    c.p = items + at617[t];
    for (size_t k = cut[t]; k < cut[t + 1]; ++k) {
      const DevUnit& d = du[k];
      if (d.cls == 0) continue;
      if (second(d)) unit_items(d, (u32)k, c, job_rows, unit_rows, b->parts3);
      else unit_items(d, (u32)k, m, job_rows, unit_rows, b->parts3);
    }
  });
  // heaviest first: a candidate's first rows (smallest d) have the largest T
  // and windows, so every candidate's chunk 0 goes out before any chunk 1
  std::stable_sort(items + at[nt], items + total,
                   [](u64 a, u64 c) { return item_chunk(a) < item_chunk(c); });
  nvtxRangePop();
  NvtxRange upload("upload batch");
  b->n_units = nd;
  b->n_main = at[nt];
  b->n_items = total;
  int s = 0;
  void* p = nullptr;
  size_t got = 0;
  if (!b->d_units || nd > b->cap_units) {
    pool_put(ctx, b->d_units, b->units_bytes);
    b->d_units = nullptr;
    b->cap_units = b->units_bytes = 0;
    if ((s = pool_get(ctx, std::max<size_t>(nd, 1) * sizeof(DevUnit), &p, &got))) return s;
    b->d_units = static_cast<DevUnit*>(p);
    b->units_bytes = got;
    b->cap_units = got / sizeof(DevUnit);
  }
  if (!b->d_items || b->n_items > b->cap_items) {
    pool_put(ctx, b->d_items, b->items_bytes);
    b->d_items = nullptr;
    b->cap_items = b->items_bytes = 0;
    if ((s = pool_get(ctx, std::max<size_t>(b->n_items, 1) * sizeof(u64), &p, &got))) return s;
    b->d_items = static_cast<u64*>(p);
    b->items_bytes = got;
    b->cap_items = got / sizeof(u64);
  }
  if (!b->d_ctr) {
    if ((s = pool_get(ctx, sizeof(Cls5Counters) + 64, &p, &got))) return s;
    b->d_ctr = static_cast<Cls5Counters*>(p);
    b->d_work = reinterpret_cast<u32*>(static_cast<char*>(p) + sizeof(Cls5Counters));
    b->ctr_bytes = got;
  }
  if (!b->d_hits) {
    if ((s = pool_get(ctx, (size_t)(1u << 20) * sizeof(s615_hit), &p, &got))) return s;
    b->d_hits = static_cast<s615_hit*>(p);
    b->hit_cap = 1u << 20;
    b->hits_bytes = got;
  }
  if (nd)
    S615_CU(cudaMemcpy(b->d_units, du, nd * sizeof(DevUnit), cudaMemcpyHostToDevice));
  if (b->n_items)
    S615_CU(cudaMemcpy(b->d_items, b->host_items.get(), b->n_items * sizeof(u64), cudaMemcpyHostToDevice));
  return S615_OK;
}

}  // namespace s615

extern "C" {

int s615_prepare(s615_ctx* ctx, const s615_unit* units, size_t n, s615_batch** out) {
  NvtxRange nvtx("s615_prepare");
  if (!ctx || !out || (n && !units) || n > kMaxBatchUnits) return S615_E_ARG;
  if (serving_blocks(ctx)) return S615_E_BUSY;
  cudaSetDevice(ctx->device);
  std::unique_ptr<s615_batch> b(new s615_batch());
  const int s = fill_batch(ctx, units, n, b.get());
  if (s) {
    s615_batch_free(ctx, b.release());
    return s;
  }
  *out = b.release();
  return S615_OK;
}

int s615_batch_size(const s615_batch* b, size_t* n_units, size_t* n_items, size_t* h2d_bytes) {
  if (!b) return S615_E_ARG;
  if (n_units) *n_units = b->n_units;
  if (n_items) *n_items = b->n_items;
  if (h2d_bytes) *h2d_bytes = b->n_units * sizeof(DevUnit) + b->n_items * sizeof(u64);
  return S615_OK;
}

int s615_batch_free(s615_ctx* ctx, s615_batch* b) {
  if (!ctx || !b) return S615_E_ARG;
  if (b->done) {   // its last launch has finished before another batch may reuse its buffers
    cudaEventSynchronize(b->done);
    cudaEventDestroy(b->done);
    b->done = nullptr;
  }
  // the device buffers go to the context's pool for the next batch
  pool_put(ctx, b->d_units, b->units_bytes);
  pool_put(ctx, b->d_items, b->items_bytes);
  pool_put(ctx, b->d_ctr, b->ctr_bytes);
  pool_put(ctx, b->d_hits, b->hits_bytes);
  delete b;
  return S615_OK;
}

int s615_run_batch(s615_ctx* ctx, int id, s615_batch* b, unsigned flags, void* stream) {
  NvtxRange nvtx("s615_run_batch");
  if (!ctx || !b) return S615_E_ARG;
  DevTable* t = find_table(ctx, id);
  if (!t) return S615_E_NOTABLE;
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  const TableView tv = view_of(*t);
  // after the launches: an event that s615_batch_free waits on before the
  // batch's buffers go to the pool (the caller may free without a sync)
  auto mark_done = [&]() {
    if (!b->done && cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      b->done = nullptr;
    }
    if (b->done) cudaEventRecord(b->done, st);
  };
  S615_CU(cudaMemsetAsync(b->d_ctr, 0, sizeof(Cls5Counters) + 64, st));
  if (!(flags & S615_F_PLAIN)) {
    const int s = launch_peel(ctx, tv, b, flags, st, 0);
    mark_done();
    return s;
  }
  // Plain form: one unit per launch and a sync after each, like the
  // reference's per-chunk loop.  (cls 7 items go out heaviest first, so a
  // cls 7 unit's items are not contiguous: each run of them is one launch.)
  s615_batch one;   // a view of one unit's items; its vectors stay empty
  one.d_units = b->d_units;
  one.n_units = b->n_units;
  one.d_hits = b->d_hits;
  one.hit_cap = b->hit_cap;
  one.d_ctr = b->d_ctr;
  one.d_work = b->d_work;
  one.item_rows = b->item_rows;
  one.parts3 = b->parts3;
  one.blocks_per_sm = b->blocks_per_sm;
  size_t i = 0;
  while (i < b->n_items) {
    size_t j = i;
    while (j < b->n_items && item_unit(b->host_items[j]) == item_unit(b->host_items[i])) ++j;
    one.d_items = b->d_items + i;
    one.n_items = j - i;
    one.n_main = i < b->n_main ? j - i : 0;   // a unit's items are all of one kernel
    S615_CU(cudaMemsetAsync(b->d_work, 0, 8, st));
    int s = launch_peel(ctx, tv, &one, flags, st, 0);
    if (s) { mark_done(); return s; }
    S615_CU(cudaStreamSynchronize(st));
    i = j;
  }
  mark_done();
  return S615_OK;
}

int s615_batch_results(s615_ctx* ctx, s615_batch* b, s615_hit* hits, size_t hit_cap,
                       size_t* n_hits, s615_counters* counters) {
  NvtxRange nvtx("s615_batch_results");
  if (!ctx || !b) return S615_E_ARG;
  Cls5Counters c{};
  S615_CU(cudaStreamSynchronize(ctx->stream));
  S615_CU(cudaMemcpy(&c, b->d_ctr, sizeof c, cudaMemcpyDeviceToHost));
  if (counters) {
    counters->calls = c.calls;
    counters->probes = c.probes;
    counters->pos = c.pos;
    counters->gated = c.pos - c.probes;
    counters->hits = c.hits;
    counters->tri_total = c.tri_total;
    counters->tri_skipped = c.tri_skipped;
  }
  const size_t nh = (size_t)c.hits;
  if (n_hits) *n_hits = nh;
  const size_t avail = std::min<size_t>(nh, b->hit_cap);
  const size_t take = std::min(avail, hit_cap);
  if (take && hits) S615_CU(cudaMemcpy(hits, b->d_hits, take * sizeof(s615_hit), cudaMemcpyDeviceToHost));
  if (nh > b->hit_cap || nh > hit_cap) return S615_E_OVERFLOW;
  return S615_OK;
}

// One call = s615_prepare + s615_run_batch + s615_batch_results on the
// context's kept batch: its device buffers are reused while they are large
// enough, so repeated calls allocate nothing.
int s615_run(s615_ctx* ctx, int id, const s615_unit* units, size_t n, unsigned flags,
             s615_hit* hits, size_t hit_cap, size_t* n_hits, s615_counters* counters) {
  NvtxRange nvtx("s615_run");
  if (!ctx || (n && !units) || n > kMaxBatchUnits) return S615_E_ARG;
  if (serving_blocks(ctx)) return S615_E_BUSY;
  if (!find_table(ctx, id)) return S615_E_NOTABLE;
  cudaSetDevice(ctx->device);
  if (!ctx->run_batch) ctx->run_batch = new s615_batch();
  s615_batch* b = ctx->run_batch;
  ctx->run_busy = true;
  int s = fill_batch(ctx, units, n, b);
  if (!s) s = s615_run_batch(ctx, id, b, flags, nullptr);
  if (!s) s = s615_batch_results(ctx, b, hits, hit_cap, n_hits, counters);
  ctx->run_busy = false;
  // an overflow still returns counters and the hits that fit; any other
  // failure keeps no device buffers
  if (s && s != S615_E_OVERFLOW) release_run_batch(ctx);
  return s;
}

int s615_autotune(s615_ctx* ctx, int id, const s615_unit* units, size_t n, unsigned flags,
                  s615_tune_entry* table, size_t cap, size_t* n_entries, s615_tune_entry* best) {
  if (!ctx || !units || n == 0 || (cap && !table)) return S615_E_ARG;
  if (serving_blocks(ctx)) return S615_E_BUSY;
  if (!find_table(ctx, id)) return S615_E_NOTABLE;
  cudaSetDevice(ctx->device);
  u32 bucket = 0;
  while (bucket < 39 && (2ull << bucket) <= n) ++bucket;
  std::vector<s615_tune_entry> got;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int s = S615_OK;
  const u32 max_bps = (flags & S615_F_SHARP) ? 3u : 5u;   // k_peel's launch bounds
  for (u32 rows : {16u, 32u, 64u}) {
    for (u32 bps = 1; bps <= max_bps && !s; ++bps) {
      ctx->force_rows = rows;
      ctx->force_bps = bps;
      s615_batch* b = nullptr;
      s = s615_prepare(ctx, units, n, &b);
      ctx->force_rows = ctx->force_bps = 0;
      if (s) break;
      float ms = 0;
      s = s615_run_batch(ctx, id, b, flags, nullptr);   // warm
      if (!s) cudaEventRecord(e0, ctx->stream);
      if (!s) s = s615_run_batch(ctx, id, b, flags, nullptr);
      if (!s) {
        cudaEventRecord(e1, ctx->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) s = S615_E_DEVICE;
        else cudaEventElapsedTime(&ms, e0, e1);
      }
      s615_batch_free(ctx, b);
      if (!s) got.push_back(s615_tune_entry{rows, bps, ms});
    }
    if (s) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (s) return s;
  size_t k = 0;
  for (size_t i = 1; i < got.size(); ++i)
    if (got[i].ms < got[k].ms) k = i;
  ctx->tune[bucket].item_rows = got[k].item_rows;
  ctx->tune[bucket].blocks_per_sm = got[k].blocks_per_sm;
  if (best) *best = got[k];
  if (n_entries) *n_entries = got.size();
  for (size_t i = 0; i < got.size() && i < cap; ++i) table[i] = got[i];
  return got.size() > cap && table ? S615_E_OVERFLOW : S615_OK;
}

int s615_tune_reset(s615_ctx* ctx) {
  if (!ctx) return S615_E_ARG;
  for (auto& t : ctx->tune) t = s615_ctx::Tune{};
  return S615_OK;
}

int s615_cls5_run(s615_ctx* ctx, int id, const s615_unit* units, size_t n, unsigned flags,
                  s615_hit* hits, size_t hit_cap, size_t* n_hits, s615_counters* counters) {
  for (size_t i = 0; i < n; ++i)
    if (units[i].cls != 5) return S615_E_FORMAT;
  return s615_run(ctx, id, units, n, flags, hits, hit_cap, n_hits, counters);
}

int s615_verify(s615_ctx* ctx, const s615_unit* units, size_t n_units, const s615_hit* hits,
                size_t n_hits, int N, s615_solution* out, size_t cap, size_t* n_out) {
  NvtxRange nvtx("s615_verify");
  if (!ctx || !n_out || N < 1) return S615_E_ARG;
  if (serving_blocks(ctx)) return S615_E_BUSY;
  cudaSetDevice(ctx->device);
  return verify_device(ctx, units, n_units, hits, n_hits, N, out, cap, n_out);
}

int s615_cls5_verify(s615_ctx* ctx, const s615_unit* units, size_t n_units, const s615_hit* hits,
                     size_t n_hits, int N, s615_solution* out, size_t cap, size_t* n_out) {
  for (size_t i = 0; i < n_units; ++i)
    if (units[i].cls != 5) return S615_E_FORMAT;
  return s615_verify(ctx, units, n_units, hits, n_hits, N, out, cap, n_out);
}

// Host self-test (no GPU): the reference's --selftest-host checks
// (fourcore_cls5_gpu_v4.cu:186-263) plus the engine's own invariants.
// Returns 0 on success, else the number of the failed check.
int s615_selftest_host(void) {
  // 1. pow6 in three limbs against repeated multiplication
  for (u64 x : {1ULL, 42ULL, 100003ULL, 2353975ULL, 2752470ULL}) {
    W3 a = pow6_w3(x), b{{1, 0, 0}};
    for (int i = 0; i < 6; ++i) b = mul_w3_u64(b, x);
    if (!eq_w3(a, b)) return 1;
  }
  // 2. gate = CRT product of the five factor sets; 27/504 and 50/247
  if (!gate_product_matches()) return 2;
  // 3. exact remainder against %
  std::mt19937_64 rng(615);
  for (int i = 0; i < 200000; ++i) {
    u64 block = (rng() >> (rng() % 62)) | 2;
    const u64 h = rng();
    if (fast_mod(h, block, mod_recip(block)) != h % block) return 3;
  }
  const u64 blocks[] = {2, 3, 1ULL << 32, (1ULL << 63) + 1, ~0ULL, 1190335832ULL};
  for (const u64 block : blocks) {
    const u64 hs[] = {0, ~0ULL, block - 1, block, 2 * block - 1, 12345678901234567ULL};
    for (const u64 h : hs)
      if (fast_mod(h, block, mod_recip(block)) != h % block) return 3;
  }
  // 4. the row formulation: T = (V - d^6)/64 equals the exact peel at the
  //    reference's sample (B=100003, u=17646, d=9, e=44)
  {
    const u64 B = 100003, u = 17646, d = 9, e = 44;
    W3 R = pow6_w3(B);
    sub_w3(R, pow6_w3(u));
    W3 V = R;
    if (sub_w3(V, pow6_w3(14 * e))) return 4;
    if (divmod_w3(V, kM21) != 0) return 4;
    W3 R2 = R;
    sub_w3(R2, pow6_w3(14 * e));
    sub_w3(R2, pow6_w3(21 * d));
    if (divmod_w3(R2, kM42) != 0) return 4;
    W3 T = V;
    if (sub_w3(T, pow6_w3(d))) return 4;
    if (divmod_w3(T, 64) != 0 || !eq_w3(T, R2)) return 4;
  }
  // 5. B^6 at B=2752470 needs at most 192 bits (134)
  {
    W3 b6 = pow6_w3(2752470ULL);
    if (b6.l[2] == 0 || (b6.l[2] >> 7) != 0) return 5;
  }
  // 6. capacity rule
  if (capacity_for(0) != 33 || capacity_for(45150) != 55569) return 6;
  return 0;
}

}  // extern "C"
