// PTX building blocks of the tensor-core kernels (sm_100a): tcgen05 matrix products with
// accumulators in tensor memory, their commits, tensor-memory loads and stores, mbarriers
// (bounded waits), cluster addressing for CTA pairs, and the expansion of 32-sample bit-plane
// words into int8 and E2M1 operand bytes.  Shared by scan_tc.cu and scan_pipe.cu.
#pragma once
#include <cstdint>

namespace epik2 {

constexpr long long kWaitLimit = 4000000000LL;  // default SM clocks (~2 s) before a wait gives up
// instruction descriptor: D s32, A/B signed 8-bit, both K-major, N = 256, M = 128
constexpr uint32_t kIdescI8 = (2u << 4) | (1u << 7) | (1u << 10) | ((256u >> 3) << 17) | ((128u >> 4) << 24);
// block-scaled instruction descriptor (kind::mxf4): A/B E2M1, scale factors UE8M0, both
// K-major, N = 224, M = 128, K = 64, scale-factor byte selectors 0.  D is FP32.
constexpr uint32_t kIdescFp4 = (1u << 7) | (1u << 10) | ((224u >> 3) << 17) | (1u << 23) | ((128u >> 4) << 24);
// the same for a CTA pair (cta_group::2): M = 256, each CTA holding 128 rows of A, 112 of B
constexpr uint32_t kIdescFp4Pair = (1u << 7) | (1u << 10) | ((224u >> 3) << 17) | (1u << 23) | ((256u >> 4) << 24);
// FP4 format: TMEM columns [224, 256) hold the scale factors (all 2^1), A's from 224 (4
// columns), B's from 240 (8 columns); class 0 accumulates into [0, 224), class 1 into
// [256, 480).
constexpr uint32_t kSfaCol = 224, kSfbCol = 240;

__device__ __forceinline__ uint32_t smem_u32(const void* ptr) {
  return (uint32_t)__cvta_generic_to_shared(ptr);
}

// Shared-memory matrix descriptor, no swizzle, K-major: LBO = 128 B (next 16-byte K
// group), SBO = bytes between groups of 8 rows, descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) |
         ((uint64_t)1 << 46);
}

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdescI8), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// One block-scaled FP4 MMA: operands 0 or 0.5 (E2M1 0b0001), every scale factor 2, so each
// product is 0 or 1 and the FP32 sums are exact counts (below 2^24 per class).
__device__ __forceinline__ void mma_fp4(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate,
                                        uint32_t sfa_tmem, uint32_t sfb_tmem) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::mxf4.block_scale.scale_vec::2X [%0], %1, %2, %3, [%5], [%6], p;\n\t}\n" ::"r"(
          d_tmem),
      "l"(a), "l"(b), "r"(kIdescFp4), "r"(accumulate), "r"(sfa_tmem), "r"(sfb_tmem));
}

__device__ __forceinline__ void tmem_st16_fill(uint32_t addr, uint32_t v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, "
      "%1};" ::"r"(addr),
      "r"(v)
      : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// CTA-pair forms.  The MMA is issued by the even CTA of a cluster of two; each CTA's shared
// memory holds its half of A and of B at the same offsets, and each CTA's tensor memory
// receives its 128 rows of D.
__device__ __forceinline__ void mma_fp4_pair(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate,
                                             uint32_t sfa_tmem, uint32_t sfb_tmem) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::mxf4.block_scale.scale_vec::2X [%0], %1, %2, %3, [%5], [%6], p;\n\t}\n" ::"r"(
          d_tmem),
      "l"(a), "l"(b), "r"(kIdescFp4Pair), "r"(accumulate), "r"(sfa_tmem), "r"(sfb_tmem));
}
// arrive on the mbarrier at this offset in both CTAs of the pair once the MMAs complete
__device__ __forceinline__ void mma_commit_pair(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(bar),
      "h"((uint16_t)3)
      : "memory");
}
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// address of the same shared-memory offset in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t map_cta(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
__device__ __forceinline__ void bar_arrive_cluster(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
__device__ __forceinline__ void st_cluster_s64(uint32_t cluster_addr, long long v) {
  asm volatile("st.shared::cluster.b64 [%0], %1;" ::"r"(cluster_addr), "l"(v) : "memory");
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void bar_arrive(uint32_t bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void bar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool bar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait with cluster-scope acquire (arrivals come from the other CTA of a pair).
__device__ __forceinline__ bool bar_wait_cluster(uint32_t bar, uint32_t parity, long long limit) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > limit) return false;
  }
}

// Bounded wait for the completion of the mbarrier phase with the given parity.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity, long long limit) {
  const long long t0 = clock64();
  while (!bar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) return false;
  }
  return true;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
  return d;
}

// 16 sample bits (low half of h) -> 16 int8 operand bytes, 0 (absent) or -1 (present);
// both operands use -1, so every product is 0 or (-1)*(-1) = +1 and the int32 sums are
// the exact counts.  One PRMT per 4 bytes: the selector is h itself, whose nibble b holds
// sample bits 4b..4b+3; the 8-byte pools alternate 0x00/0xFF so that the byte picked by
// the nibble's low 3 bits is 0xFF exactly when the tested bit (bit 0, 1 or 2 of the
// nibble) is set, and the nibble's sign-replicate bit cannot change a 0x00/0xFF byte.
// Byte 4t+b of the group therefore holds sample t+4b: the same sample order is used for
// A and B, so the products still pair each sample with itself.
__device__ __forceinline__ uint4 expand16(uint32_t h) {
  uint4 r;
  r.x = prmt(0xFF00FF00u, 0xFF00FF00u, h);        // nibble bit 0: samples 0, 4, 8, 12
  r.y = prmt(0xFFFF0000u, 0xFFFF0000u, h);        // nibble bit 1: samples 1, 5, 9, 13
  r.z = prmt(0x00000000u, 0xFFFFFFFFu, h);        // nibble bit 2: samples 2, 6, 10, 14
  r.w = prmt(0xFF00FF00u, 0xFF00FF00u, h >> 3);   // nibble bit 3 via shift: 3, 7, 11, 15
  return r;
}

// 32 sample bits -> 16 bytes of E2M1 operands, 0 (absent) or 0.5 (present, nibble 0b0001):
// 32-bit word q of the group holds samples q, q+4, ..., q+28 in its eight nibbles.  The same
// order is used for A and B.
__device__ __forceinline__ uint4 expand32_fp4(uint32_t w) {
  return make_uint4(w & 0x11111111u, (w >> 1) & 0x11111111u, (w >> 2) & 0x11111111u, (w >> 3) & 0x11111111u);
}

__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void sts128(uint32_t saddr, uint4 v) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(saddr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
               : "memory");
}

}  // namespace epik2
