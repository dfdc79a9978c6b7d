// Integer-pipe peak probes (include/epik2_probe.h): independent chains of POPC, LOP3
// and IADD on every SM.  Each thread writes one result word, so the work cannot be
// removed by the compiler and every store stays inside the output buffer.
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/epik2_probe.h"

namespace {

__global__ void k_popc(uint32_t* out, int iters, uint32_t seed) {
  uint32_t b[8], a[8];
#pragma unroll
  for (int r = 0; r < 8; r++) {
    b[r] = seed * (threadIdx.x + 1) + r * 0x9e3779b9u;
    a[r] = 0;
  }
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int r = 0; r < 8; r++) {
      uint32_t p;
      asm volatile("popc.b32 %0, %1;" : "=r"(p) : "r"(b[r] ^ (uint32_t)it));
      a[r] += p;
    }
  }
  uint32_t s = 0;
#pragma unroll
  for (int r = 0; r < 8; r++) s += a[r];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void k_lop3(uint32_t* out, int iters, uint32_t seed) {
  uint32_t x[8];
  uint32_t y = seed * 7u + threadIdx.x, z = seed ^ 0x12345678u;
#pragma unroll
  for (int r = 0; r < 8; r++) x[r] = seed * (threadIdx.x + 1) + r;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int r = 0; r < 8; r++) asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(x[r]) : "r"(y), "r"(z));
    y += 1;
  }
  uint32_t s = 0;
#pragma unroll
  for (int r = 0; r < 8; r++) s ^= x[r];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void k_iadd(uint32_t* out, int iters, uint32_t seed) {
  uint32_t x[8];
  const uint32_t y = seed * 7u + threadIdx.x;
#pragma unroll
  for (int r = 0; r < 8; r++) x[r] = seed * (threadIdx.x + 1) + r;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int r = 0; r < 8; r++) asm volatile("add.u32 %0, %0, %1;" : "+r"(x[r]) : "r"(y));
  }
  uint32_t s = 0;
#pragma unroll
  for (int r = 0; r < 8; r++) s ^= x[r];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

typedef void (*probe_fn)(uint32_t*, int, uint32_t);

int time_probe(probe_fn f, int blocks, int threads, int iters, uint32_t* d_out, double* ops_per_s) {
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return -2;
  for (int w = 0; w < 3; w++) f<<<blocks, threads>>>(d_out, iters / 10, 1u);
  if (cudaDeviceSynchronize() != cudaSuccess) return -2;
  float best = 1e30f;
  for (int rep = 0; rep < 5; rep++) {
    cudaEventRecord(e0);
    f<<<blocks, threads>>>(d_out, iters, 2u + rep);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess) return -2;
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ops_per_s = (double)blocks * threads * iters * 8.0 / (best * 1e-3);
  return 0;
}

}  // namespace

extern "C" int epik2_probe_int_peaks(int device, double* popc_per_s, double* lop3_per_s, double* iadd_per_s) {
  if (!popc_per_s || !lop3_per_s || !iadd_per_s) return -1;
  if (cudaSetDevice(device) != cudaSuccess) return -7;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return -7;
  const int blocks = sms * 8, threads = 256;
  uint32_t* d_out = nullptr;
  if (cudaMalloc(&d_out, (size_t)blocks * threads * sizeof(uint32_t)) != cudaSuccess) return -3;
  int r = time_probe(k_popc, blocks, threads, 20000, d_out, popc_per_s);
  if (!r) r = time_probe(k_lop3, blocks, threads, 40000, d_out, lop3_per_s);
  if (!r) r = time_probe(k_iadd, blocks, threads, 60000, d_out, iadd_per_s);
  cudaFree(d_out);
  return r;
}
