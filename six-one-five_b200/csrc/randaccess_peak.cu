// randaccess_peak.cu -- the B200's random 8-byte read rate, the ceiling of the
// xor probe (three random cells per probe).
//
// Reads `iters` 8-byte words at hashed (uniform, always in-bounds) positions of
// a buffer (2 GiB unless sizes are given) with four load forms and prints
// reads/s.  The result is the
// denominator for the probe kernel's random-access roofline.
//   bin/randaccess_peak            (run under ncu with dram__sectors_read.sum to
//                                   see the bytes each form moves per read)
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>

typedef unsigned long long u64;

__device__ __forceinline__ u64 mix(u64 x) {
  x ^= x >> 33; x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33;
  return x;
}

template <int V>
__global__ void k_random_reads(const u64* __restrict__ p, u64 n, u64 iters, u64* out) {
  u64 acc = 0;
  const u64 tid = blockIdx.x * (u64)blockDim.x + threadIdx.x, nt = (u64)gridDim.x * blockDim.x;
  for (u64 i = tid; i < iters; i += nt) {
    const u64 j = mix(i * 0x9E3779B97F4A7C15ULL + V) % n;
    u64 v;
    if (V == 0) v = __ldg(p + j);                                   // L1-allocating, read-only
    else if (V == 1) v = __ldcg(p + j);                             // L2 only
    else asm volatile("ld.global.cg.L2::64B.u64 %0, [%1];" : "=l"(v) : "l"(p + j));  // L2 only, 64 B fill
    acc ^= v;
  }
  if (acc == 0x123456789ULL) out[0] = acc;
}

// The same random 64-B-fill reads with the index taken as the high half of
// h * n (one multiply instead of a 64-bit remainder) and four independent loads
// per thread per iteration, so that neither the index arithmetic nor a lack of
// loads in flight limits the rate.
__global__ void k_random_reads_ilp(const u64* __restrict__ p, u64 n, u64 iters, u64* out) {
  u64 acc = 0;
  const u64 tid = blockIdx.x * (u64)blockDim.x + threadIdx.x, nt = (u64)gridDim.x * blockDim.x;
  for (u64 i = tid * 4; i < iters; i += nt * 4) {
    u64 v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const u64 j = __umul64hi(mix((i + k) * 0x9E3779B97F4A7C15ULL + 3), n);   // j < n
      asm volatile("ld.global.cg.L2::64B.u64 %0, [%1];" : "=l"(v[k]) : "l"(p + j));
    }
    acc ^= v[0] ^ v[1] ^ v[2] ^ v[3];
  }
  if (acc == 0x123456789ULL) out[0] = acc;
}

// Usage: randaccess_peak [GiB ...] -- one line per load form and buffer size
// (default 2 GiB); larger buffers show how the rate falls with the footprint.
int main(int argc, char** argv) {
  const u64 iters = 1ull << 27;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  u64* o = nullptr;
  if (cudaMalloc(&o, 8) != cudaSuccess) { std::printf("alloc failed\n"); return 1; }
  const char* names[4] = {"ld.global.nc (L1)", "ld.global.cg", "ld.global.cg.L2::64B",
                          "ld.global.cg.L2::64B x4"};
  const int nsizes = argc > 1 ? argc - 1 : 1;
  cudaError_t e = cudaSuccess;
  for (int si = 0; si < nsizes && e == cudaSuccess; ++si) {
    const double gib = argc > 1 ? std::atof(argv[1 + si]) : 2.0;
    const u64 n = (u64)(gib * (double)(1ull << 30)) / 8;
    u64* p = nullptr;
    if (n < 1024 || cudaMalloc(&p, n * 8) != cudaSuccess) {
      std::printf("%.1f GiB: alloc failed\n", gib);
      cudaGetLastError();
      continue;
    }
    cudaMemset(p, 1, n * 8);
    for (int v = 0; v < 4; ++v) {
      auto launch = [&]() {
        if (v == 0) k_random_reads<0><<<sms * 8, 256>>>(p, n, iters, o);
        else if (v == 1) k_random_reads<1><<<sms * 8, 256>>>(p, n, iters, o);
        else if (v == 2) k_random_reads<2><<<sms * 8, 256>>>(p, n, iters, o);
        else k_random_reads_ilp<<<sms * 8, 256>>>(p, n, iters, o);
      };
      launch();
      cudaEventRecord(a);
      launch();
      cudaEventRecord(b);
      cudaEventSynchronize(b);
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      std::printf("%7.1f GiB  %-24s %.3f ms  %.3e random reads/s\n", gib, names[v], ms,
                  iters / (ms * 1e-3));
    }
    // the x4 form with fewer resident blocks: fewer reads in flight per SM
    for (int bps : {1, 2, 4}) {
      k_random_reads_ilp<<<sms * bps, 256>>>(p, n, iters, o);
      cudaEventRecord(a);
      k_random_reads_ilp<<<sms * bps, 256>>>(p, n, iters, o);
      cudaEventRecord(b);
      cudaEventSynchronize(b);
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      std::printf("%7.1f GiB  %-17s bps=%d %.3f ms  %.3e random reads/s\n", gib,
                  "ld.global.cg.L2::64B x4", bps, ms, iters / (ms * 1e-3));
    }
    cudaFree(p);
    e = cudaGetLastError();
  }
  std::printf("status: %s\n", cudaGetErrorString(e));
  cudaFree(o);
  return e == cudaSuccess ? 0 : 1;
}
