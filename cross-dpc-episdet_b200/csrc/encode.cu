// Genotype encoding and the per-SNP / per-pair count tables.
//
// encode : uint8 genotypes [n_samples][n_snps] (the reference's sample-major layout,
//          GPU/v4.cpp:94) -> per-class {g0, g1} bit planes, word-major.  Replaces the
//          host loops data_to_binary + binary_to_tiled (GPU/v4.cpp:112-196).  As there,
//          genotype 2 (and any value other than 0/1) sets neither plane, so g2 is the
//          complement of g0|g1 inside the class and padding bits stay zero.
// counts : single-SNP counts n_c(g) and pair counts n_c(g_x, g_y) for g in {0,1}, the
//          lower-order margins from which the search derives every cell that involves
//          genotype 2 (inclusion-exclusion; no reference counterpart -- the reference
//          counts all 27 cells directly, GPU/v4.cpp:331-385).
#include "epik2_internal.h"

namespace epik2 {

// One thread per (class word, SNP).  Threads of a block cover consecutive SNPs so the
// reads of one sample row are coalesced; the sample index comes from the class-sorted
// permutation (broadcast).
__global__ void k_encode(const uint8_t* __restrict__ geno, const int32_t* __restrict__ perm, uint2* __restrict__ planes,
                         int64_t n_snps, int64_t m_pad, int64_t w0, int64_t w1, int64_t n0, int64_t n1) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= m_pad) return;
  const int64_t wt = w0 + w1;
  for (int64_t w = blockIdx.y; w < wt; w += gridDim.y) {
    const bool cases = w >= w0;
    const int64_t base = 32 * (cases ? w - w0 : w);
    const int64_t n_class = cases ? n1 : n0;
    const int32_t* pc = perm + (cases ? n0 : 0);
    uint32_t g0 = 0, g1 = 0;
    if (m < n_snps) {
      const int64_t lim = n_class - base < 32 ? n_class - base : 32;
      for (int64_t b = 0; b < lim; b++) {
        const int64_t s = pc[base + b];
        const uint32_t g = geno[s * n_snps + m];
        g0 |= (uint32_t)(g == 0) << b;
        g1 |= (uint32_t)(g == 1) << b;
      }
    }
    planes[w * m_pad + m] = make_uint2(g0, g1);
  }
}

// The same encoding, 16 SNPs per thread, for matrices whose rows are whole 16-byte pieces
// (n_snps a multiple of 16): one 128-bit load per sample gives the thread all 16 genotypes,
// so a warp reads 512 consecutive bytes of a sample row per load.  Per 32-bit piece,
// __vcmpeq4 marks the bytes equal to 0 and to 1; bit b of a plane word is sample b of the
// class word, as in k_encode.  Groups past n_snps (up to m_pad) write zero planes.
__global__ void k_encode16(const uint8_t* __restrict__ geno, const int32_t* __restrict__ perm,
                           uint2* __restrict__ planes, int64_t n_snps, int64_t m_pad, int64_t w0, int64_t w1,
                           int64_t n0, int64_t n1) {
  const int64_t m0 = 16 * ((int64_t)blockIdx.x * blockDim.x + threadIdx.x);
  if (m0 >= m_pad) return;
  const int64_t wt = w0 + w1;
  for (int64_t w = blockIdx.y; w < wt; w += gridDim.y) {
    const bool cases = w >= w0;
    const int64_t base = 32 * (cases ? w - w0 : w);
    const int64_t n_class = cases ? n1 : n0;
    const int32_t* pc = perm + (cases ? n0 : 0);
    uint32_t g0[16], g1[16];
#pragma unroll
    for (int q = 0; q < 16; q++) g0[q] = g1[q] = 0;
    if (m0 < n_snps) {
      const int64_t lim = n_class - base < 32 ? n_class - base : 32;
      for (int64_t b = 0; b < lim; b++) {
        const int64_t s = pc[base + b];
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(geno + s * n_snps + m0));
        const uint32_t x[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int h = 0; h < 4; h++) {
          const uint32_t z = __vcmpeq4(x[h], 0u), o = __vcmpeq4(x[h], 0x01010101u);
#pragma unroll
          for (int t = 0; t < 4; t++) {
            g0[4 * h + t] |= ((z >> (8 * t)) & 1u) << b;
            g1[4 * h + t] |= ((o >> (8 * t)) & 1u) << b;
          }
        }
      }
    }
    uint4* dst = reinterpret_cast<uint4*>(planes + w * m_pad + m0);
#pragma unroll
    for (int q = 0; q < 8; q++) dst[q] = make_uint4(g0[2 * q], g1[2 * q], g0[2 * q + 1], g1[2 * q + 1]);
  }
}

// singles[c][m][g] = popcount over class c's words of plane g of SNP m.
__global__ void k_singles(const uint2* __restrict__ planes, uint32_t* __restrict__ singles, int64_t m_pad, int64_t w0,
                          int64_t w1) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= m_pad) return;
  uint32_t c0g0 = 0, c0g1 = 0, c1g0 = 0, c1g1 = 0;
  for (int64_t w = 0; w < w0; w++) {
    const uint2 v = planes[w * m_pad + m];
    c0g0 += __popc(v.x);
    c0g1 += __popc(v.y);
  }
  for (int64_t w = w0; w < w0 + w1; w++) {
    const uint2 v = planes[w * m_pad + m];
    c1g0 += __popc(v.x);
    c1g1 += __popc(v.y);
  }
  singles[(0 * m_pad + m) * 2 + 0] = c0g0;
  singles[(0 * m_pad + m) * 2 + 1] = c0g1;
  singles[(1 * m_pad + m) * 2 + 0] = c1g0;
  singles[(1 * m_pad + m) * 2 + 1] = c1g1;
}

// pairs[c][tri(x,y)] = (n(0,0), n(0,1), n(1,0), n(1,1)) of SNPs x < y in class c.
// Block (x, y-strip of 256); the x word is a broadcast load, y words are coalesced.
__global__ void k_pairs(const uint2* __restrict__ planes, uint4* __restrict__ pairs, int64_t m_pad, int64_t w0,
                        int64_t w1) {
  const int64_t x = blockIdx.x;
  const int64_t y = (int64_t)blockIdx.y * blockDim.x + threadIdx.x;
  if ((int64_t)blockIdx.y * blockDim.x + blockDim.x <= x + 1) return;  // whole strip at or below the diagonal
  if (y <= x || y >= m_pad) return;
  const int64_t tri = tri_size(m_pad);
  const int64_t off = tri_offset(m_pad, x, y);
  for (int c = 0; c < 2; c++) {
    const int64_t wb = c ? w0 : 0, we = c ? w0 + w1 : w0;
    uint32_t n00 = 0, n01 = 0, n10 = 0, n11 = 0;
    for (int64_t w = wb; w < we; w++) {
      const uint2 a = planes[w * m_pad + x];
      const uint2 b = planes[w * m_pad + y];
      n00 += __popc(a.x & b.x);
      n01 += __popc(a.x & b.y);
      n10 += __popc(a.y & b.x);
      n11 += __popc(a.y & b.y);
    }
    pairs[c * tri + off] = make_uint4(n00, n01, n10, n11);
  }
}

cudaError_t launch_encode(const DevDataset& d, cudaStream_t stream) {
  const int64_t wt = d.w0 + d.w1;
  if (wt == 0 || d.m_pad == 0) return cudaSuccess;
  const bool vec = d.n_snps % 16 == 0 && ((uintptr_t)d.geno % 16) == 0 && ((uintptr_t)d.planes % 16) == 0;
  if (vec) {  // 16 SNPs per thread
    const int64_t groups = d.m_pad / 16;
    dim3 grid((unsigned)((groups + 127) / 128), (unsigned)(wt < 65535 ? wt : 65535));
    k_encode16<<<grid, 128, 0, stream>>>(d.geno, d.perm, d.planes, d.n_snps, d.m_pad, d.w0, d.w1, d.n_controls,
                                         d.n_cases);
  } else {
    dim3 grid((unsigned)((d.m_pad + 255) / 256), (unsigned)(wt < 65535 ? wt : 65535));
    k_encode<<<grid, 256, 0, stream>>>(d.geno, d.perm, d.planes, d.n_snps, d.m_pad, d.w0, d.w1, d.n_controls,
                                      d.n_cases);
  }
  return cudaGetLastError();
}

cudaError_t launch_counts(const DevDataset& d, cudaStream_t stream, bool pairs) {
  if (d.m_pad == 0) return cudaSuccess;
  k_singles<<<(unsigned)((d.m_pad + 255) / 256), 256, 0, stream>>>(d.planes, d.singles, d.m_pad, d.w0, d.w1);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (d.m_pad < 2 || !pairs) return cudaSuccess;
  dim3 grid((unsigned)d.m_pad, (unsigned)((d.m_pad + 255) / 256));
  k_pairs<<<grid, 256, 0, stream>>>(d.planes, d.pairs, d.m_pad, d.w0, d.w1);
  return cudaGetLastError();
}

}  // namespace epik2
