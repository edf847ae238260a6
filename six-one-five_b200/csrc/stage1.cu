// stage1.cu -- Stage-1 class-5 units generated and packed on the device.
//
// The reference emits units on the host (fourcore_hunt_v3.cpp:371-381 over
// unit_candidates, fourcore_classes_v3.hpp:114-154), writes them as .buc text
// and the GPU program packs them again (pack_unit5, fourcore_cls5_gpu_v4.cu:
// 169-184).  Here one thread per B does both straight into a batch:
//   u = s + 7^6 k for the seeds s with s^6 = B^6 (mod 7^6), u <= B-1, 6 | u;
//   e residues: roots of B^6 14^-6 (mod 3^6); d residues: roots of
//   (B^6 - u^6) 21^-6 (mod 2^6); base = B^6 - u^6 mod 2^128 and the limits of
// make_dev_unit, in ascending u per B (the reference's order).  The units'
// work items follow, one thread per unit.  Only per-B and per-unit counts
// cross to the host (for the two prefix sums).
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <numeric>
#include <vector>

#include "engine.hpp"

namespace s615 {

namespace {

constexpr u32 kM2 = 64, kM3 = 729, kM7 = 117649;

struct Roots {                 // CSR root lists, offsets then roots, per modulus
  const u32 *off2, *r2, *off3, *r3, *off7, *r7;
  u32 inv14_3, inv21_2;        // (14^6)^-1 mod 3^6, (21^6)^-1 mod 2^6
};

__device__ __forceinline__ u32 pow6_mod(u64 x, u32 m) {
  x %= m;
  const u64 x2 = x * x % m, x3 = x2 * x % m;
  return (u32)(x3 * x3 % m);
}

__device__ __forceinline__ bool eligible(u64 B) { return B > 1 && (B & 1) && B % 3 && B % 7; }

// The seeds of B ascending (at most 6) and their count.
__device__ __forceinline__ u32 seeds_of(const Roots& R, u64 B, u32 s[8]) {
  const u32 b7 = pow6_mod(B, kM7);
  const u32 lo = R.off7[b7], hi = R.off7[b7 + 1];
  u32 n = 0;
  for (u32 i = lo; i < hi && n < 8; ++i) s[n++] = R.r7[i];
  return n;   // r7 lists are ascending
}

// Units of B, ascending: k outer (u in [k 7^6, (k+1) 7^6)), seeds inner.
template <class F>
__device__ __forceinline__ void each_unit(const Roots& R, u64 B, F f) {
  u32 s[8];
  const u32 ns = seeds_of(R, B, s);
  for (u64 k = 0; k * kM7 < B; ++k)
    for (u32 i = 0; i < ns; ++i) {
      const u64 u = (u64)s[i] + k * kM7;
      if (u <= B - 1 && u % 6 == 0) f(u);
    }
}

__global__ void k_s1_count(Roots R, u64 B_lo, u32 nB, u32* counts) {
  const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nB) return;
  const u64 B = B_lo + i;
  u32 c = 0;
  if (eligible(B)) each_unit(R, B, [&](u64) { ++c; });
  counts[i] = c;
}

__global__ void k_s1_units(Roots R, u64 B_lo, u32 nB, const u32* unit_off, DevUnit* units,
                           u32* items_per_unit) {
  const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nB) return;
  const u64 B = B_lo + i;
  if (!eligible(B)) return;
  u32 k = unit_off[i];
  // B^6 mod 2^128 and its residues
  const u128 B3 = (u128)(B * B) * B;
  const u128 B6 = B3 * B3;
  const u32 te = (u32)((u64)pow6_mod(B, kM3) * R.inv14_3 % kM3);
  const u32 e_lo = R.off3[te], e_n = min(R.off3[te + 1] - e_lo, 12u);
  const u32 fmax1 = (u32)((B - 1) / 14), fmax2 = (u32)((B - 1) / 21), lim = (u32)((B - 1) / 42);
  each_unit(R, B, [&](u64 u) {
    DevUnit d;
    memset(&d, 0, sizeof d);
    const u128 u3 = (u128)(u * u) * u;
    const u128 base = B6 - u3 * u3;
    d.base_lo = (u64)base;
    d.base_hi = (u64)(base >> 64);
    d.B = B; d.u = u;
    d.cls = 5; d.f = 0; d.mod1 = kModE;
    d.fmax1 = fmax1; d.fmax2 = fmax2; d.lim = lim;
    d.id = k;
    d.nres1 = e_n;
    for (u32 j = 0; j < e_n; ++j) d.res1[j] = R.r3[e_lo + j];
    const u32 td = (u32)(((u64)pow6_mod(B, kM2) + kM2 - pow6_mod(u, kM2)) % kM2 * R.inv21_2 % kM2);
    const u32 d_lo = R.off2[td], d_n = min(R.off2[td + 1] - d_lo, 12u);
    d.nres2 = d_n;
    for (u32 j = 0; j < d_n; ++j) d.res2[j] = R.r2[d_lo + j];
    u32 ni = 0;
    for (u32 j = 0; j < e_n; ++j) {
      u32 jmin, jend;
      class_rows(d.res1[j], kModE, fmax1, &jmin, &jend);
      const u32 rows = jend > jmin ? jend - jmin : 0;
      ni += (rows + kItemRows - 1) / kItemRows;
    }
    units[k] = d;
    items_per_unit[k] = ni;
    ++k;
  });
}

__global__ void k_s1_items(const DevUnit* units, u32 n_units, const u32* item_off, u64* items) {
  const u32 k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_units) return;
  const DevUnit& d = units[k];
  u32 o = item_off[k];
  for (u32 j = 0; j < d.nres1; ++j) {
    u32 jmin, jend;
    class_rows(d.res1[j], d.mod1, d.fmax1, &jmin, &jend);
    const u32 rows = jend > jmin ? jend - jmin : 0;
    for (u32 c = 0; c * kItemRows < rows; ++c) items[o++] = make_item(k, j, c);
  }
}

__global__ void k_s1_gather(const DevUnit* units, u32 n, u64* bu) {
  const u32 k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) { bu[2 * k] = units[k].B; bu[2 * k + 1] = units[k].u; }
}

int roots_on_device(s615_ctx* ctx, Roots* R) {
  std::vector<u32> o2, r2, o3, r3, o7, r7;
  root_csr(2, o2, r2);
  root_csr(3, o3, r3);
  root_csr(7, o7, r7);
  const size_t words = o2.size() + r2.size() + o3.size() + r3.size() + o7.size() + r7.size();
  if (!ctx->d_roots) {
    void* p = nullptr;
    const int s = dev_alloc(ctx, &p, words * sizeof(u32));
    if (s) return s;
    std::vector<u32> all;
    all.reserve(words);
    for (auto* v : {&o2, &r2, &o3, &r3, &o7, &r7}) all.insert(all.end(), v->begin(), v->end());
    S615_CU(cudaMemcpy(p, all.data(), words * sizeof(u32), cudaMemcpyHostToDevice));
    ctx->d_roots = static_cast<u32*>(p);
    ctx->roots_bytes = words * sizeof(u32);
  }
  const u32* q = ctx->d_roots;
  R->off2 = q; q += o2.size();
  R->r2 = q; q += r2.size();
  R->off3 = q; q += o3.size();
  R->r3 = q; q += r3.size();
  R->off7 = q; q += o7.size();
  R->r7 = q;
  R->inv14_3 = inv_pow6_mod(14, kM3);
  R->inv21_2 = inv_pow6_mod(21, kM2);
  return S615_OK;
}

}  // namespace

}  // namespace s615

using namespace s615;

extern "C" {

int s615_prepare_band(s615_ctx* ctx, uint64_t B_lo, uint64_t B_hi, s615_batch** out) {
  if (!ctx || !out || B_lo < 2 || B_hi < B_lo || B_hi > 40000000ULL || B_hi - B_lo >= (1u << 26))
    return S615_E_ARG;
  if (serving_blocks(ctx)) return S615_E_BUSY;
  cudaSetDevice(ctx->device);
  Roots R;
  int s = roots_on_device(ctx, &R);
  if (s) return s;
  const u32 nB = (u32)(B_hi - B_lo + 1);
  cudaStream_t st = ctx->stream;
  std::unique_ptr<s615_batch> b(new s615_batch());
  // 1. units per B -> offsets
  void* p = nullptr;
  if ((s = arena_get(ctx, 0, (size_t)nB * 4 * 2 + 16, &p))) return s;
  u32* d_counts = static_cast<u32*>(p);
  u32* d_off = d_counts + nB;
  k_s1_count<<<(nB + 255) / 256, 256, 0, st>>>(R, B_lo, nB, d_counts);
  ctx->launches++;
  S615_CU(cudaGetLastError());
  std::vector<u32> counts(nB), off(nB);
  S615_CU(cudaMemcpyAsync(counts.data(), d_counts, nB * 4, cudaMemcpyDeviceToHost, st));
  S615_CU(cudaStreamSynchronize(st));
  u64 n_units = 0;
  for (u32 i = 0; i < nB; ++i) { off[i] = (u32)n_units; n_units += counts[i]; }
  if (n_units > kMaxBatchUnits) return S615_E_ARG;
  S615_CU(cudaMemcpyAsync(d_off, off.data(), nB * 4, cudaMemcpyHostToDevice, st));
  // 2. the batch's unit records and item counts
  const size_t nu = std::max<size_t>(n_units, 1);
  if ((s = dev_alloc(ctx, &p, nu * sizeof(DevUnit)))) return s;
  b->d_units = static_cast<DevUnit*>(p);
  b->cap_units = nu;
  b->n_units = n_units;
  if ((s = arena_get(ctx, 1, nu * 4 * 2 + 16, &p))) { s615_batch_free(ctx, b.release()); return s; }
  u32* d_ni = static_cast<u32*>(p);
  u32* d_io = d_ni + nu;
  if (n_units) {
    k_s1_units<<<(nB + 127) / 128, 128, 0, st>>>(R, B_lo, nB, d_off, b->d_units, d_ni);
    ctx->launches++;
    S615_CU(cudaGetLastError());
  }
  std::vector<u32> ni(n_units), io(n_units);
  if (n_units) S615_CU(cudaMemcpyAsync(ni.data(), d_ni, n_units * 4, cudaMemcpyDeviceToHost, st));
  S615_CU(cudaStreamSynchronize(st));
  u64 n_items = 0;
  for (u64 k = 0; k < n_units; ++k) { io[k] = (u32)n_items; n_items += ni[k]; }
  if (n_items >> 32) { s615_batch_free(ctx, b.release()); return S615_E_ARG; }
  // 3. work items
  const size_t nit = std::max<size_t>(n_items, 1);
  if ((s = dev_alloc(ctx, &p, nit * sizeof(u64)))) { s615_batch_free(ctx, b.release()); return s; }
  b->d_items = static_cast<u64*>(p);
  b->cap_items = nit;
  b->n_items = n_items;
  b->n_main = n_items;
  if (n_units) {
    S615_CU(cudaMemcpyAsync(d_io, io.data(), n_units * 4, cudaMemcpyHostToDevice, st));
    k_s1_items<<<(u32)((n_units + 255) / 256), 256, 0, st>>>(b->d_units, (u32)n_units, d_io, b->d_items);
    ctx->launches++;
    S615_CU(cudaGetLastError());
  }
  // 4. counters, cursors, hits
  if ((s = dev_alloc(ctx, &p, sizeof(Cls5Counters) + 64))) { s615_batch_free(ctx, b.release()); return s; }
  b->d_ctr = static_cast<Cls5Counters*>(p);
  b->d_work = reinterpret_cast<u32*>(static_cast<char*>(p) + sizeof(Cls5Counters));
  if ((s = dev_alloc(ctx, &p, (size_t)(1u << 20) * sizeof(s615_hit)))) {
    s615_batch_free(ctx, b.release());
    return s;
  }
  b->d_hits = static_cast<s615_hit*>(p);
  b->hit_cap = 1u << 20;
  S615_CU(cudaStreamSynchronize(st));
  *out = b.release();
  return S615_OK;
}

int s615_batch_units(s615_ctx* ctx, const s615_batch* b, s615_unit* out, size_t cap, size_t* n) {
  if (!ctx || !b || !n || (cap && !out)) return S615_E_ARG;
  *n = b->n_units;
  if (!cap || !b->n_units) return b->n_units > cap ? S615_E_OVERFLOW : S615_OK;
  cudaSetDevice(ctx->device);
  const size_t take = std::min(cap, b->n_units);
  void* p = nullptr;
  int s = arena_get(ctx, 2, take * 16, &p);
  if (s) return s;
  cudaStream_t st = ctx->stream;
  k_s1_gather<<<(u32)((take + 255) / 256), 256, 0, st>>>(b->d_units, (u32)take, static_cast<u64*>(p));
  ctx->launches++;
  S615_CU(cudaGetLastError());
  std::vector<u64> bu(2 * take);
  S615_CU(cudaMemcpyAsync(bu.data(), p, take * 16, cudaMemcpyDeviceToHost, st));
  S615_CU(cudaStreamSynchronize(st));
  for (size_t k = 0; k < take; ++k) {
    s615_unit x{};
    x.cls = 5;
    x.kind = 0;
    x.B = bu[2 * k];
    x.u = bu[2 * k + 1];
    out[k] = x;
  }
  return b->n_units > cap ? S615_E_OVERFLOW : S615_OK;
}

}  // extern "C"
