// table.cu -- xor-filter query and the packed <-> wide HBM layouts.
//
// k_xor_query is the device form of xor_might_contain
// (spike/ribbon/xor_filter.hpp:472-483, fourcore_cls5_gpu_v4.cu:322-334):
// identical hash, cell indices and fingerprint comparison.  Cell indices are
// 64-bit (the reference's u32 variant in fourcore_find_device.cuh:54-63
// wraps once 3*block > 2^32).
#include <cuda_runtime.h>

#include <algorithm>

#include "s615_device.cuh"

namespace s615 {

namespace {

__global__ void k_xor_query(TableView t, const u64* __restrict__ keys, u64 n,
                            u8* __restrict__ out) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n;
       i += (u64)gridDim.x * blockDim.x)
    out[i] = might_contain(t, keys[i]) ? 1 : 0;
}

// One thread per cell: gather r bits from the packed bytes (read as aligned
// 64-bit words) into a 4- or 8-byte wide cell.
__global__ void k_unpack(const unsigned long long* __restrict__ packed, u64 m, u32 r,
                         void* __restrict__ wide, int cell_bytes) {
  const u64 mask = fp_mask(r);
  for (u64 c = blockIdx.x * (u64)blockDim.x + threadIdx.x; c < m;
       c += (u64)gridDim.x * blockDim.x) {
    const u64 bit = c * (u64)r, w = bit >> 6;
    const u32 o = (u32)(bit & 63);
    u64 v = packed[w] >> o;
    if (o + r > 64) v |= packed[w + 1] << (64 - o);
    v &= mask;
    if (cell_bytes == 8) static_cast<u64*>(wide)[c] = v;
    else static_cast<u32*>(wide)[c] = (u32)v;
  }
}

// One thread per output 64-bit word: OR in every cell overlapping bits
// [64w, 64w+64).  No two threads write the same word, so no atomics.
template <typename Cell>
__global__ void k_pack(const Cell* __restrict__ wide, u64 m, u32 r,
                       unsigned long long* __restrict__ packed, u64 n_words) {
  const u64 mask = fp_mask(r);
  for (u64 w = blockIdx.x * (u64)blockDim.x + threadIdx.x; w < n_words;
       w += (u64)gridDim.x * blockDim.x) {
    const u64 lo = w * 64;
    u64 c = lo / r;
    u64 word = 0;
    for (; c < m; ++c) {
      const u64 p = c * (u64)r;
      if (p >= lo + 64) break;
      const u64 v = (u64)wide[c] & mask;
      if (p >= lo) word |= v << (p - lo);
      else word |= v >> (lo - p);
    }
    packed[w] = word;
  }
}

int grid_for(s615_ctx* ctx, u64 n, int threads) {
  const u64 want = (n + threads - 1) / threads;
  const u64 cap = (u64)ctx->num_sms * 16;
  return (int)(want < cap ? (want ? want : 1) : cap);
}

}  // namespace

TableView view_of(const DevTable& t) {
  TableView v{};
  v.shards = 1;
  if (!t.parts.empty()) {   // a shard set: the parts' views live in HBM
    v.shards = t.hdr.shard_count;
    v.block = v.shards;   // the shard index is fast_mod(mix, S, recip)
    v.recip = mod_recip(v.shards);
    v.parts = static_cast<const TableView*>(t.d_views);
    v.shard_seed = kShardSeed;
    size_t bytes = 0;
    for (const DevTable& p : t.parts) bytes += p.bytes;
    const u64 want = t.groups ? t.groups : (bytes + kProbeGroupBytes - 1) / kProbeGroupBytes;
    v.groups = (u32)std::min<u64>(std::max<u64>(want, 1), t.parts.size());
    v.grp_lo = t.shard_lo;   // the shards this set holds; other keys are not its to probe
    v.grp_hi = t.shard_lo + (u32)t.parts.size();
    v.r = t.hdr.r;
    v.fpmask = fp_mask(t.hdr.r);
    return v;
  }
  v.cells = t.d_cells;
  v.bytes = t.bytes;
  v.block = t.hdr.m_cells / 3;
  v.recip = mod_recip(v.block);
  v.fpmask = fp_mask(t.hdr.r);
  v.seed = t.hdr.mix_seed;
  v.r = t.hdr.r;
  v.layout = (u32)t.layout;
  v.cell_bytes = (u32)t.cell_bytes;
  if (t.hdr.n_keys == 0 || t.hdr.m_cells < 3) v.block = 0;
  return v;
}

int launch_xor_query(s615_ctx* ctx, const TableView& tv, const u64* d_keys, size_t n,
                     u8* d_out, cudaStream_t st) {
  if (n == 0) return S615_OK;
  k_xor_query<<<grid_for(ctx, n, 256), 256, 0, st>>>(tv, d_keys, n, d_out);
  ctx->launches++;
  S615_CU(cudaGetLastError());
  return S615_OK;
}

int launch_unpack(s615_ctx* ctx, const u8* d_packed, u64 m, u32 r, void* d_wide, int cell_bytes,
                  cudaStream_t st) {
  if (m == 0) return S615_OK;
  k_unpack<<<grid_for(ctx, m, 256), 256, 0, st>>>(
      reinterpret_cast<const unsigned long long*>(d_packed), m, r, d_wide, cell_bytes);
  ctx->launches++;
  S615_CU(cudaGetLastError());
  return S615_OK;
}

int launch_pack(s615_ctx* ctx, const void* d_wide, int cell_bytes, u64 m, u32 r, u8* d_packed,
                u64 packed_len, cudaStream_t st) {
  const u64 n_words = (packed_len + 7) / 8;
  if (n_words == 0) return S615_OK;
  auto* out = reinterpret_cast<unsigned long long*>(d_packed);
  if (cell_bytes == 8)
    k_pack<<<grid_for(ctx, n_words, 256), 256, 0, st>>>(static_cast<const u64*>(d_wide), m, r, out,
                                                        n_words);
  else
    k_pack<<<grid_for(ctx, n_words, 256), 256, 0, st>>>(static_cast<const u32*>(d_wide), m, r, out,
                                                        n_words);
  ctx->launches++;
  S615_CU(cudaGetLastError());
  return S615_OK;
}

S615_CHECK_TAKE_DEFINE(check_take_table)

}  // namespace s615
