// Exhaustive triplet search on the integer pipe (LOP3 + POPC), K2 score and argmin.
//
// Replaces kernel_epi (GPU/v4.cpp:295-594; same arithmetic as GPU/v2.cpp:260-553) and
// the host argmin (GPU/v4.cpp:599-608).  Differences in method, none in result:
//   * Work unit = one warp, one pair group (i, j0..j0+3) and a strip of 32 SNPs k (one
//     per lane).  The warp walks every class word once per strip; the i and j words are
//     warp-uniform loads, the k words one coalesced 256-byte load.
//   * Only the 8 cells with g_i, g_j, g_k in {0,1} are popcounted (one LOP3 + POPC +
//     IADD each per word).  The other 19 cells per class follow exactly from the pair
//     counts (i,j), (i,k), (j,k), the single-SNP counts and the class size by
//     inclusion-exclusion, in unsigned 32-bit arithmetic.  The reference popcounts all
//     27 cells (GPU/v4.cpp:359-385); the resulting tables are identical.
//   * Persistent warps take pair groups from an atomic counter, heaviest first.
//   * K2 uses a lookup table of ln n! for every n up to n_samples+1, built on the host in
//     the reference CPU arithmetic, and the reference's float accumulation order
//     (CPU/v2.cpp:514-517): score += (lut[n0+n1+1] - lut[n0]) - lut[n1], then fabs.
//   * Argmin: (score, i, j, k) lexicographic, warp shuffle -> one slot per warp -> a
//     single-block reduction.  This is the lowest-index tie-break of GPU/v2.cpp:556-565.
#include <cfloat>

#include "epik2_internal.h"
#include "scan_common.cuh"

namespace epik2 {

// Accumulate the 8 popcounted cells (4*g_i + 2*g_j + g_k, genotypes 0/1) of the four
// pairs (i, jl[q]) against SNP k over class words [wb, we).
__device__ __forceinline__ void count_words(const uint2* __restrict__ planes, int64_t m_pad, int64_t wb, int64_t we,
                                            int i, const int (&jl)[kPairsPerWarp], int k,
                                            uint32_t (&acc)[kPairsPerWarp][8]) {
  const uint2* pw = planes + wb * m_pad;
#pragma unroll 2
  for (int64_t w = wb; w < we; ++w, pw += m_pad) {
    const uint2 a = __ldg(pw + i);
    uint2 b[kPairsPerWarp];
#pragma unroll
    for (int q = 0; q < kPairsPerWarp; q++) b[q] = __ldg(pw + jl[q]);
    const uint2 c = __ldg(pw + k);
#pragma unroll
    for (int q = 0; q < kPairsPerWarp; q++) {
      acc[q][0] += __popc(a.x & b[q].x & c.x);
      acc[q][1] += __popc(a.x & b[q].x & c.y);
      acc[q][2] += __popc(a.x & b[q].y & c.x);
      acc[q][3] += __popc(a.x & b[q].y & c.y);
      acc[q][4] += __popc(a.y & b[q].x & c.x);
      acc[q][5] += __popc(a.y & b[q].x & c.y);
      acc[q][6] += __popc(a.y & b[q].y & c.x);
      acc[q][7] += __popc(a.y & b[q].y & c.y);
    }
  }
}

template <bool kDump, bool kTopK>
__global__ void __launch_bounds__(kScanThreads, 2) k_scan_int(const ScanParams p) {
  const int lane = threadIdx.x & 31;
  const int64_t gwarp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t m_pad = p.m_pad;
  const int m = p.m;
  const int64_t tri = p.tri;
  float best_s = FLT_MAX;
  unsigned long long best_k = ~0ull;
  // top-k list (kTopK): lane r holds the r-th best of this warp
  float list_s = FLT_MAX;
  unsigned long long list_k = ~0ull;

  for (;;) {
    unsigned long long g = 0;
    if (lane == 0) g = atomicAdd(p.counter, 1ull);
    g = __shfl_sync(kFull, g, 0);
    if (g >= (unsigned long long)p.n_groups) break;
    int lo = 0, hi = p.n_first;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (p.pg_off[mid] <= (int64_t)g) lo = mid;
      else hi = mid;
    }
    const int i = p.i_begin + lo;
    const int j0 = i + 1 + kPairsPerWarp * (int)((int64_t)g - p.pg_off[lo]);
    const int nj = min(kPairsPerWarp, m - j0);
    int jl[kPairsPerWarp];
#pragma unroll
    for (int q = 0; q < kPairsPerWarp; q++) jl[q] = min(j0 + q, (int)m_pad - 1);
    const int s_begin = (j0 + 1) >> 5, s_end = (int)(m_pad >> 5);
    const uint2 si0 = *reinterpret_cast<const uint2*>(p.singles + ((int64_t)i) * 2);
    const uint2 si1 = *reinterpret_cast<const uint2*>(p.singles + (m_pad + i) * 2);

    for (int s = s_begin; s < s_end; ++s) {
      const int k = (s << 5) + lane;
      uint32_t acc0[kPairsPerWarp][8], acc1[kPairsPerWarp][8];
#pragma unroll
      for (int q = 0; q < kPairsPerWarp; q++)
#pragma unroll
        for (int c = 0; c < 8; c++) {
          acc0[q][c] = 0;
          acc1[q][c] = 0;
        }
      count_words(p.planes, m_pad, 0, p.w0, i, jl, k, acc0);
      count_words(p.planes, m_pad, p.w0, p.w0 + p.w1, i, jl, k, acc1);

      const bool k_ok = k < m;
      uint2 sk0 = make_uint2(0, 0), sk1 = make_uint2(0, 0);
      uint4 pik0 = make_uint4(0, 0, 0, 0), pik1 = pik0;
      if (k_ok && k > i) {
        sk0 = *reinterpret_cast<const uint2*>(p.singles + ((int64_t)k) * 2);
        sk1 = *reinterpret_cast<const uint2*>(p.singles + (m_pad + k) * 2);
        const int64_t oik = tri_offset(m_pad, i, k);
        pik0 = __ldg(p.pairs + oik);
        pik1 = __ldg(p.pairs + tri + oik);
      }
#pragma unroll
      for (int q = 0; q < kPairsPerWarp; q++) {
        const int j = j0 + q;
        const bool valid = (q < nj) && k_ok && (k > j);
        float sc = FLT_MAX;
        unsigned long long key = ~0ull;
        if (valid) {
          const uint2 sj0 = *reinterpret_cast<const uint2*>(p.singles + ((int64_t)j) * 2);
          const uint2 sj1 = *reinterpret_cast<const uint2*>(p.singles + (m_pad + j) * 2);
          const int64_t oij = tri_offset(m_pad, i, j), ojk = tri_offset(m_pad, j, k);
          const uint4 pij0 = __ldg(p.pairs + oij), pij1 = __ldg(p.pairs + tri + oij);
          const uint4 pjk0 = __ldg(p.pairs + ojk), pjk1 = __ldg(p.pairs + tri + ojk);
          uint32_t T0[27], T1[27];
          complete_table(acc0[q], (uint32_t)p.n0, si0, sj0, sk0, pij0, pik0, pjk0, T0);
          complete_table(acc1[q], (uint32_t)p.n1, si1, sj1, sk1, pij1, pik1, pjk1, T1);
          sc = k2_score(T0, T1, p.lut);
          key = pack_key((uint64_t)i, (uint64_t)j, (uint64_t)k);
          if (kDump) {
            const int64_t t = triplet_index(m, i, j, k);
            uint32_t* dt = p.dump_tables + t * 54;
#pragma unroll
            for (int c = 0; c < 27; c++) {
              dt[c] = T0[c];
              dt[27 + c] = T1[c];
            }
            p.dump_scores[t] = sc;
          }
          if (better(sc, key, best_s, best_k)) {
            best_s = sc;
            best_k = key;
          }
        }
        if (kTopK) {
          // threshold = the warp list's last entry (lane 31)
          const float ts = __shfl_sync(kFull, list_s, 31);
          const unsigned long long tk = __shfl_sync(kFull, list_k, 31);
          unsigned want = __ballot_sync(kFull, valid && better(sc, key, ts, tk));
          while (want) {
            const int src = __ffs(want) - 1;
            want &= want - 1;
            const float cs = __shfl_sync(kFull, sc, src);
            const unsigned long long ck = __shfl_sync(kFull, key, src);
            const float ts2 = __shfl_sync(kFull, list_s, 31);
            const unsigned long long tk2 = __shfl_sync(kFull, list_k, 31);
            if (better(cs, ck, ts2, tk2)) warp_list_insert(list_s, list_k, cs, ck, lane);
          }
        }
      }
    }
  }
  // warp argmin
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const float os = __shfl_xor_sync(kFull, best_s, off);
    const unsigned long long ok = __shfl_xor_sync(kFull, best_k, off);
    if (better(os, ok, best_s, best_k)) {
      best_s = os;
      best_k = ok;
    }
  }
  if (lane == 0) {
    p.slots[gwarp].score = best_s;
    p.slots[gwarp].key = best_k;
  }
  if (kTopK) {
    p.cand[gwarp * 32 + lane].score = list_s;
    p.cand[gwarp * 32 + lane].key = list_k;
  }
}

// Single-block reduction of per-warp slots.
__global__ void k_reduce_best(const BestSlot* __restrict__ slots, int n, BestSlot* __restrict__ out) {
  __shared__ float ss[32];
  __shared__ unsigned long long sk[32];
  float bs = FLT_MAX;
  unsigned long long bk = ~0ull;
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    if (better(slots[t].score, slots[t].key, bs, bk)) {
      bs = slots[t].score;
      bk = slots[t].key;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const float os = __shfl_xor_sync(kFull, bs, off);
    const unsigned long long ok = __shfl_xor_sync(kFull, bk, off);
    if (better(os, ok, bs, bk)) {
      bs = os;
      bk = ok;
    }
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    ss[w] = bs;
    sk[w] = bk;
  }
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    bs = lane < nw ? ss[lane] : FLT_MAX;
    bk = lane < nw ? sk[lane] : ~0ull;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const float os = __shfl_xor_sync(kFull, bs, off);
      const unsigned long long ok = __shfl_xor_sync(kFull, bk, off);
      if (better(os, ok, bs, bk)) {
        bs = os;
        bk = ok;
      }
    }
    if (lane == 0) {
      out->score = bs;
      out->key = bk;
    }
  }
}

// 54-cell table of (i,j,k) by one warp, all 27 cells per class popcounted directly as in
// the reference (GPU/v2.cpp:288-540) -- an independent check of the inclusion-exclusion
// path.  g2 = ~(g0|g1) restricted to the valid bits of the class's last word.  Every lane
// returns the full counts.
__device__ __forceinline__ void warp_direct_table(const uint2* __restrict__ planes, int64_t m_pad, int64_t w0,
                                                  int64_t w1, int64_t n0, int64_t n1, int64_t i, int64_t j, int64_t k,
                                                  int lane, uint32_t (&cnt)[54]) {
#pragma unroll
  for (int c = 0; c < 54; c++) cnt[c] = 0;
#pragma unroll
  for (int cl = 0; cl < 2; cl++) {
    const int64_t wb = cl ? w0 : 0, we = cl ? w0 + w1 : w0;
    const int64_t ncls = cl ? n1 : n0;
    for (int64_t w = wb + lane; w < we; w += 32) {
      const int64_t bits_left = ncls - 32 * (w - wb);
      const uint32_t valid = bits_left >= 32 ? 0xffffffffu : ((1u << bits_left) - 1u);
      const uint2 a = planes[w * m_pad + i], b = planes[w * m_pad + j], c = planes[w * m_pad + k];
      const uint32_t ga[3] = {a.x, a.y, ~(a.x | a.y) & valid};
      const uint32_t gb[3] = {b.x, b.y, ~(b.x | b.y) & valid};
      const uint32_t gc[3] = {c.x, c.y, ~(c.x | c.y) & valid};
#pragma unroll
      for (int x = 0; x < 3; x++)
#pragma unroll
        for (int y = 0; y < 3; y++)
#pragma unroll
          for (int z = 0; z < 3; z++) cnt[27 * cl + 9 * x + 3 * y + z] += __popc(ga[x] & gb[y] & gc[z]);
    }
  }
#pragma unroll
  for (int c = 0; c < 54; c++) {
    uint32_t v = cnt[c];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFull, v, off);
    cnt[c] = v;
  }
}

__global__ void k_tables_direct(const uint2* __restrict__ planes, int64_t m_pad, int64_t w0, int64_t w1, int64_t n0,
                                int64_t n1, const uint32_t* __restrict__ trip, int64_t n, uint32_t* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (t >= n) return;
  uint32_t cnt[54];
  warp_direct_table(planes, m_pad, w0, w1, n0, n1, trip[3 * t], trip[3 * t + 1], trip[3 * t + 2], lane, cnt);
  if (lane == 0)
#pragma unroll
    for (int c = 0; c < 54; c++) out[t * 54 + c] = cnt[c];
}

// Precision form: rescore candidates in FP64.  One warp per candidate recounts its
// table directly, then lane 0 evaluates K2 twice: FP32 in the reference order (must
// equal the search's score) and FP64 from a double ln n! table -- the only FP64 step.
__global__ void k_rescore(const uint2* __restrict__ planes, int64_t m_pad, int64_t w0, int64_t w1, int64_t n0,
                          int64_t n1, const BestSlot* __restrict__ cand, int64_t n, const float* __restrict__ lut32,
                          const double* __restrict__ lut64, Rescored* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (t >= n) return;
  const unsigned long long key = cand[t].key;
  if (key == ~0ull) {
    if (lane == 0) {
      out[t].s64 = 0.0;
      out[t].s32 = FLT_MAX;
      out[t].key = key;
    }
    return;
  }
  const int64_t i = (int64_t)(key >> 42), j = (int64_t)((key >> 21) & 0x1fffff), k = (int64_t)(key & 0x1fffff);
  uint32_t cnt[54];
  warp_direct_table(planes, m_pad, w0, w1, n0, n1, i, j, k, lane, cnt);
  if (lane == 0) {
    float s32 = 0.0f;
    double s64 = 0.0;
#pragma unroll
    for (int c = 0; c < 27; c++) {
      const uint32_t a = cnt[c], b = cnt[27 + c];
      s32 = __fadd_rn(s32, __fsub_rn(__fsub_rn(lut32[a + b + 1], lut32[a]), lut32[b]));
      s64 = __dadd_rn(s64, __dsub_rn(__dsub_rn(lut64[a + b + 1], lut64[a]), lut64[b]));
    }
    out[t].s64 = fabs(s64);
    out[t].s32 = fabsf(s32);
    out[t].key = key;
  }
}

int scan_blocks_per_sm() {
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_scan_int<false, false>, kScanThreads, 0);
  return nb > 0 ? nb : 1;
}

cudaError_t launch_scan_int(const ScanParams& p, int blocks, bool dump, cudaStream_t stream) {
  const bool topk = p.top_k > 1;
  if (dump) k_scan_int<true, false><<<blocks, kScanThreads, 0, stream>>>(p);
  else if (topk) k_scan_int<false, true><<<blocks, kScanThreads, 0, stream>>>(p);
  else k_scan_int<false, false><<<blocks, kScanThreads, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_reduce_best(const BestSlot* slots, int n, BestSlot* out, cudaStream_t stream) {
  k_reduce_best<<<1, 1024, 0, stream>>>(slots, n, out);
  return cudaGetLastError();
}

// FP64 rescore of each batched dataset's best triplet (one warp per dataset).
__global__ void k_rescore_jobs(const TcJob* __restrict__ jobs, const BestSlot* __restrict__ best, int n,
                               Rescored* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int b = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (b >= n) return;
  const unsigned long long key = best[b].key;
  if (key == ~0ull) {
    if (lane == 0) {
      out[b].s64 = 0.0;
      out[b].s32 = FLT_MAX;
      out[b].key = key;
    }
    return;
  }
  const TcJob& J = jobs[b];
  const int64_t i = (int64_t)(key >> 42), j = (int64_t)((key >> 21) & 0x1fffff), k = (int64_t)(key & 0x1fffff);
  uint32_t cnt[54];
  warp_direct_table(J.planes, J.m_pad, J.w0, J.w1, J.n0, J.n1, i, j, k, lane, cnt);
  if (lane == 0) {
    float s32 = 0.0f;
    double s64 = 0.0;
#pragma unroll
    for (int c = 0; c < 27; c++) {
      const uint32_t x = cnt[c], y = cnt[27 + c];
      s32 = __fadd_rn(s32, __fsub_rn(__fsub_rn(J.lut[x + y + 1], J.lut[x]), J.lut[y]));
      s64 = __dadd_rn(s64, __dsub_rn(__dsub_rn(J.lut64[x + y + 1], J.lut64[x]), J.lut64[y]));
    }
    out[b].s64 = fabs(s64);
    out[b].s32 = fabsf(s32);
    out[b].key = key;
  }
}

cudaError_t launch_rescore_jobs(const TcJob* jobs, const BestSlot* best, int n, Rescored* out, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  const int64_t threads = (int64_t)n * 32;
  k_rescore_jobs<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(jobs, best, n, out);
  return cudaGetLastError();
}

cudaError_t launch_rescore(const DevDataset& d, const BestSlot* cand, int64_t n, Rescored* out,
                           cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  const int64_t threads = n * 32;
  k_rescore<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(d.planes, d.m_pad, d.w0, d.w1, d.n_controls,
                                                                  d.n_cases, cand, n, d.lut, d.lut64, out);
  return cudaGetLastError();
}

cudaError_t launch_tables(const DevDataset& d, const uint32_t* triplets, int64_t n, uint32_t* out,
                          cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  const int64_t threads = n * 32;
  k_tables_direct<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(d.planes, d.m_pad, d.w0, d.w1,
                                                                        d.n_controls, d.n_cases, triplets, n, out);
  return cudaGetLastError();
}

}  // namespace epik2
