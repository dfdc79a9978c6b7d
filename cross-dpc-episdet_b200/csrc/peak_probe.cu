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

// Back-to-back tcgen05.mma from zeroed shared memory (no-swizzle K-major descriptors, LBO
// 128 B, SBO 1024 B), 512 tensor-memory columns per CTA: kind::i8 M128 N256 K32, or the
// search kernel's block-scaled FP4 shape kind::mxf4 M128 N224 K64 with its scale factors
// (every byte 2^1) in columns [224, 256).  Accumulators alternate between columns 0 and 256.
constexpr uint32_t kIdescProbe = (2u << 4) | (1u << 7) | (1u << 10) | ((256u >> 3) << 17) | ((128u >> 4) << 24);
constexpr uint32_t kIdescProbeFp4 = (1u << 7) | (1u << 10) | ((224u >> 3) << 17) | (1u << 23) | ((128u >> 4) << 24);
constexpr int kProbeSmem = 153600;  // > half an SM's shared memory: one CTA per SM

__device__ __forceinline__ uint64_t probe_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46);
}

template <bool kFp4>
__global__ void __launch_bounds__(128, 1) k_tc_probe(int n_mma, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint32_t s_tmem;
  __shared__ __align__(8) uint64_t bar;
  const int tid = threadIdx.x;
  for (int t = tid; t < 49152 / 4; t += blockDim.x) reinterpret_cast<uint32_t*>(smem)[t] = 0;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
  const uint32_t sbar = (uint32_t)__cvta_generic_to_shared(&bar);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sbar), "r"(1u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(&s_tmem)),
                 "r"(512u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  if (kFp4) {  // scale factors: columns [224, 256) of the warp's 32 lanes
    const uint32_t ta = tmem + ((uint32_t)(32 * (tid >> 5)) << 16) + 224u, v = 0x80808080u;
#pragma unroll
    for (int c = 0; c < 32; c += 16)
      asm volatile(
          "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, "
          "%1, %1};" ::"r"(ta + c),
          "r"(v)
          : "memory");
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (tid == 0) {
    for (int q = 0; q < n_mma; q++) {
      const int kk = q & 3;
      const uint32_t d = tmem + ((q >> 2) & 1) * 256;
      const uint64_t a = probe_desc(sbase + kk * 256), b = probe_desc(sbase + 16384 + kk * 256);
      if (kFp4)
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::mxf4.block_scale.scale_vec::2X [%0], %1, %2, %3, [%5], [%6], p;\n\t}\n" ::"r"(d),
            "l"(a), "l"(b), "r"(kIdescProbeFp4), "r"(q > 1 ? 1u : 0u), "r"(tmem + 224u), "r"(tmem + 240u));
      else
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
            "l"(a), "l"(b), "r"(kIdescProbe), "r"(q > 1 ? 1u : 0u), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(sbar) : "memory");
    uint32_t ok = 0;
    const long long t0 = clock64();
    while (!ok) {
      asm volatile(
          "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, "
          "p;\n\t}\n"
          : "=r"(ok)
          : "r"(sbar), "r"(0u)
          : "memory");
      if (clock64() - t0 > 4000000000LL) {
        atomicExch(err, 1);
        break;
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (tid < 32) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
  }
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

namespace {

template <bool kFp4>
int probe_tc(int device, double* mac_per_s) {
  if (!mac_per_s) return -1;
  if (cudaSetDevice(device) != cudaSuccess) return -7;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return -7;
  int* d_err = nullptr;
  if (cudaMalloc(&d_err, sizeof(int)) != cudaSuccess) return -3;
  cudaMemset(d_err, 0, sizeof(int));
  if (cudaFuncSetAttribute(k_tc_probe<kFp4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kProbeSmem) !=
      cudaSuccess) {
    cudaFree(d_err);
    return -2;
  }
  const int n_mma = 16384;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_tc_probe<kFp4><<<sms, 128, kProbeSmem>>>(1024, d_err);
  cudaEventRecord(e0);
  k_tc_probe<kFp4><<<sms, 128, kProbeSmem>>>(n_mma, d_err);
  cudaEventRecord(e1);
  int r = cudaEventSynchronize(e1) == cudaSuccess ? 0 : -2;
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  int herr = 0;
  cudaMemcpy(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_err);
  if (r) return r;
  if (herr) return -6;
  const double macs_per_mma = kFp4 ? 128.0 * 224.0 * 64.0 : 128.0 * 256.0 * 32.0;
  *mac_per_s = (double)n_mma * macs_per_mma * sms / (ms * 1e-3);
  return 0;
}

}  // namespace

extern "C" int epik2_probe_tc_i8(int device, double* mac_per_s) { return probe_tc<false>(device, mac_per_s); }

extern "C" int epik2_probe_tc_fp4(int device, double* mac_per_s) { return probe_tc<true>(device, mac_per_s); }
