// randaccess_peak.cu -- the B200's random 8-byte read rate, the ceiling of the
// xor probe (three random cells per probe).
//
// Reads `iters` 8-byte words at hashed (uniform, always in-bounds) positions of
// a buffer (2 GiB unless sizes are given) with five load forms and prints
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

// The xor probe's access shape: three reads per key, one in each third of the
// buffer (block, block + j1, 2 block + j2), 64-B fills.  `keys` keys, 3 reads each.
__global__ void k_random_reads_thirds(const u64* __restrict__ p, u64 n, u64 keys, u64* out) {
  u64 acc = 0;
  const u64 blk = n / 3;
  const u64 tid = blockIdx.x * (u64)blockDim.x + threadIdx.x, nt = (u64)gridDim.x * blockDim.x;
  for (u64 q = tid; q < keys; q += nt) {
    const u64 h = mix(q * 0x9E3779B97F4A7C15ULL + 5);
    const u64 j0 = __umul64hi(h, blk);                                         // < blk
    const u64 j1 = blk + __umul64hi(mix(h ^ 0x9E3779B97F4A7C15ULL), blk);      // < 2 blk
    const u64 j2 = 2 * blk + __umul64hi(mix(h ^ 0xBF58476D1CE4E5B9ULL), blk);  // < 3 blk <= n
    u64 a, b, c;
    asm volatile("ld.global.cg.L2::64B.u64 %0, [%1];" : "=l"(a) : "l"(p + j0));
    asm volatile("ld.global.cg.L2::64B.u64 %0, [%1];" : "=l"(b) : "l"(p + j1));
    asm volatile("ld.global.cg.L2::64B.u64 %0, [%1];" : "=l"(c) : "l"(p + j2));
    acc ^= a ^ b ^ c;
  }
  if (acc == 0x123456789ULL) out[0] = acc;
}

// Usage: randaccess_peak [GiB ...] -- one line per load form and buffer size
// (default 2 GiB); larger buffers show how the rate falls with the footprint.
int main(int argc, char** argv) {
  // 2^30 reads per launch (~25 ms at full rate); best of five launches after one
  // warm launch, so that a short launch's ramp does not set the ceiling
  const u64 iters = 1ull << 30;
  const int reps = 5;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  u64* o = nullptr;
  if (cudaMalloc(&o, 8) != cudaSuccess) { std::printf("alloc failed\n"); return 1; }
  const char* names[5] = {"ld.global.nc (L1)", "ld.global.cg", "ld.global.cg.L2::64B",
                          "ld.global.cg.L2::64B x4", "ld.global.cg.L2::64B thirds"};
  const u64 keys = iters / 3;
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
    for (int v = 0; v < 5; ++v) {
      auto launch = [&]() {
        if (v == 0) k_random_reads<0><<<sms * 8, 256>>>(p, n, iters, o);
        else if (v == 1) k_random_reads<1><<<sms * 8, 256>>>(p, n, iters, o);
        else if (v == 2) k_random_reads<2><<<sms * 8, 256>>>(p, n, iters, o);
        else if (v == 3) k_random_reads_ilp<<<sms * 8, 256>>>(p, n, iters, o);
        else k_random_reads_thirds<<<sms * 8, 256>>>(p, n, keys, o);
      };
      const u64 reads = v == 4 ? 3 * keys : iters;
      launch();
      float ms = 1e30f;
      for (int k = 0; k < reps; ++k) {
        cudaEventRecord(a);
        launch();
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float t = 0;
        cudaEventElapsedTime(&t, a, b);
        if (t < ms) ms = t;
      }
      std::printf("%7.1f GiB  %-24s %.3f ms  %.3e random reads/s\n", gib, names[v], ms,
                  reads / (ms * 1e-3));
    }
    // one read in flight per thread, from 32 to 2048 threads per SM: the rate as a
    // function of the reads in flight
    for (int tps : {32, 64, 128, 256, 512, 1024}) {
      const int th = tps < 256 ? tps : 256, bl = tps < 256 ? 1 : tps / 256;
      k_random_reads<2><<<sms * bl, th>>>(p, n, iters / 8, o);
      float ms = 1e30f;
      for (int k = 0; k < reps; ++k) {
        cudaEventRecord(a);
        k_random_reads<2><<<sms * bl, th>>>(p, n, iters / 8, o);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float t = 0;
        cudaEventElapsedTime(&t, a, b);
        if (t < ms) ms = t;
      }
      std::printf("%7.1f GiB  %-17s tps=%d %.3f ms  %.3e random reads/s\n", gib,
                  "ld.global.cg.L2::64B", tps, ms, (iters / 8) / (ms * 1e-3));
    }
    // the x4 form with fewer resident blocks: fewer reads in flight per SM
    for (int bps : {1, 2, 4}) {
      k_random_reads_ilp<<<sms * bps, 256>>>(p, n, iters, o);
      float ms = 1e30f;
      for (int k = 0; k < reps; ++k) {
        cudaEventRecord(a);
        k_random_reads_ilp<<<sms * bps, 256>>>(p, n, iters, o);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float t = 0;
        cudaEventElapsedTime(&t, a, b);
        if (t < ms) ms = t;
      }
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
