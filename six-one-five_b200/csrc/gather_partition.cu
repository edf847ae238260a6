// gather_partition.cu -- measurement tool (make bench-tools): random cell
// gathers against gathers grouped by table slice (so a slice is read while
// L2-resident), the cost of the radix partition that groups them and of
// putting the gathered values back in lookup order, on a buffer of the
// table's footprint.
//   bin/gather_partition [table_GiB] [log2 lookups]
#include <cub/cub.cuh>
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
typedef unsigned long long u64;
typedef unsigned int u32;
#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { \
  printf("CUDA %s at %d\n", cudaGetErrorString(e_), __LINE__); return 1; } } while (0)
__device__ __forceinline__ u64 mix(u64 x) {
  x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
  return x;
}
__device__ __forceinline__ u64 ld64(const u64* p) {
  u64 v; asm volatile("ld.global.cg.L2::64B.u64 %0, [%1];" : "=l"(v) : "l"(p)); return v;
}
__global__ void k_gen(u32* idx, u32* id, u64 m, u64 n) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < m; i += (u64)gridDim.x * blockDim.x) {
    idx[i] = (u32)__umul64hi(mix(i * 0x9E3779B97F4A7C15ULL + 7), n);
    id[i] = (u32)i;
  }
}
__global__ void k_gather(const u64* __restrict__ T, const u32* __restrict__ idx, u64 m, u64* __restrict__ out) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < m; i += (u64)gridDim.x * blockDim.x)
    out[i] = ld64(T + idx[i]);
}
__global__ void k_gather4(const u64* __restrict__ T, const u32* __restrict__ idx, u64 m, u64* __restrict__ out) {
  const u64 nt = (u64)gridDim.x * blockDim.x;
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < m; i += 4 * nt) {
    u64 v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = (i + k * nt < m) ? ld64(T + idx[i + k * nt]) : 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) if (i + k * nt < m) out[i + k * nt] = v[k];
  }
}
__global__ void k_scatter(const u64* __restrict__ vals, const u32* __restrict__ id, u64 m, u64* __restrict__ res) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < m; i += (u64)gridDim.x * blockDim.x)
    res[id[i]] = vals[i];
}
int main(int argc, char** argv) {
  const double gib = argc > 1 ? atof(argv[1]) : 26.93;
  const int lg = argc > 2 ? atoi(argv[2]) : 28;
  const u64 n = (u64)(gib * (double)(1ull << 30)) / 8;
  const u64 m = 1ull << lg;
  if (n >= (1ull << 32) || lg > 30) { printf("sizes out of range\n"); return 1; }
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
  u64 *T = nullptr, *out = nullptr, *res = nullptr;
  u32 *idx = nullptr, *idx2 = nullptr, *id = nullptr, *id2 = nullptr;
  CK(cudaMalloc(&T, n * 8)); CK(cudaMemset(T, 1, n * 8));
  CK(cudaMalloc(&out, m * 8)); CK(cudaMalloc(&res, m * 8));
  CK(cudaMalloc(&idx, m * 4)); CK(cudaMalloc(&idx2, m * 4));
  CK(cudaMalloc(&id, m * 4)); CK(cudaMalloc(&id2, m * 4));
  k_gen<<<sms * 8, 256>>>(idx, id, m, n);
  CK(cudaGetLastError()); CK(cudaDeviceSynchronize());
  cudaEvent_t a, b; cudaEventCreate(&a); cudaEventCreate(&b);
  auto timeit = [&](auto&& fn) {
    fn(); cudaDeviceSynchronize();
    float best = 1e30f;
    for (int r = 0; r < 3; ++r) {
      cudaEventRecord(a); fn(); cudaEventRecord(b); cudaEventSynchronize(b);
      float t = 0; cudaEventElapsedTime(&t, a, b); if (t < best) best = t;
    }
    return best;
  };
  printf("table %.2f GiB (%llu cells), %llu lookups (%.2f per 64-B chunk)\n", gib, n, m, (double)m / (n / 8.0));
  float t = timeit([&] { k_gather<<<sms * 8, 256>>>(T, idx, m, out); });
  printf("random gather           %8.3f ms  %.3e lookups/s\n", t, m / (t * 1e-3));
  t = timeit([&] { k_gather4<<<sms * 4, 256>>>(T, idx, m, out); });
  printf("random gather x4        %8.3f ms  %.3e lookups/s\n", t, m / (t * 1e-3));
  for (int slice_bits : {22, 23, 24, 32}) {
    const int begin = slice_bits == 32 ? 0 : slice_bits;
    size_t tb = 0; void* tmp = nullptr;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, idx, idx2, id, id2, (int)m, begin, 32);
    CK(cudaMalloc(&tmp, tb));
    float ts = timeit([&] { cub::DeviceRadixSort::SortPairs(tmp, tb, idx, idx2, id, id2, (int)m, begin, 32); });
    float tg = timeit([&] { k_gather<<<sms * 8, 256>>>(T, idx2, m, out); });
    float tg4 = timeit([&] { k_gather4<<<sms * 4, 256>>>(T, idx2, m, out); });
    float tsc = timeit([&] { k_scatter<<<sms * 8, 256>>>(out, id2, m, res); });
    printf("slice 2^%d cells (%.0f MB): partition(pairs, bits %d..31) %.3f ms %.3e/s | grouped gather %.3f ms "
           "%.3e/s (x4 %.3f ms) | scatter back %.3f ms %.3e/s\n", slice_bits,
           slice_bits == 32 ? 0.0 : (double)(8ull << slice_bits) / 1e6, begin, ts, m / (ts * 1e-3), tg,
           m / (tg * 1e-3), tg4, tsc, m / (tsc * 1e-3));
    cudaFree(tmp);
  }
  CK(cudaGetLastError());
  printf("status ok\n");
  return 0;
}
