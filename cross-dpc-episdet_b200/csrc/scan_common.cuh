// Device helpers shared by the search kernels (integer and tensor-core engines): the
// selection order, the lexicographic triplet index, the inclusion-exclusion completion
// of a table from its 8 counted cells, the FP32 K2 score and the warp top-32 list.
#pragma once
#include <cfloat>
#include <cstdint>

#include "epik2_internal.h"

namespace epik2 {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ bool better(float s, unsigned long long k, float bs, unsigned long long bk) {
  return s < bs || (s == bs && k < bk);
}

// Lexicographic index of (i<j<k) among the C(m,3) triplets.
__device__ __forceinline__ int64_t triplet_index(int64_t m, int64_t i, int64_t j, int64_t k) {
  const int64_t mi = m - i;
  const int64_t before_i = m * (m - 1) * (m - 2) / 6 - mi * (mi - 1) * (mi - 2) / 6;
  const int64_t nb = j - i - 1;
  const int64_t before_j = nb * (m - 1) - (nb * (i + 1) + nb * (nb - 1) / 2);
  return before_i + before_j + (k - j - 1);
}

// Full 27-cell table of one class from the 8 measured cells and the margins.
__device__ __forceinline__ void complete_table(const uint32_t (&t8)[8], uint32_t n, uint2 si, uint2 sj, uint2 sk,
                                               uint4 pij, uint4 pik, uint4 pjk, uint32_t (&T)[27]) {
  const uint32_t Si[3] = {si.x, si.y, n - si.x - si.y};
  const uint32_t Sj[3] = {sj.x, sj.y, n - sj.x - sj.y};
  const uint32_t Sk[3] = {sk.x, sk.y, n - sk.x - sk.y};
  uint32_t PIJ[3][3], PIK[3][3], PJK[3][3];
  PIJ[0][0] = pij.x; PIJ[0][1] = pij.y; PIJ[1][0] = pij.z; PIJ[1][1] = pij.w;
  PIK[0][0] = pik.x; PIK[0][1] = pik.y; PIK[1][0] = pik.z; PIK[1][1] = pik.w;
  PJK[0][0] = pjk.x; PJK[0][1] = pjk.y; PJK[1][0] = pjk.z; PJK[1][1] = pjk.w;
#pragma unroll
  for (int a = 0; a < 2; a++) {
    PIJ[a][2] = Si[a] - PIJ[a][0] - PIJ[a][1];
    PIK[a][2] = Si[a] - PIK[a][0] - PIK[a][1];
    PJK[a][2] = Sj[a] - PJK[a][0] - PJK[a][1];
  }
#pragma unroll
  for (int b = 0; b < 3; b++) {
    PIJ[2][b] = Sj[b] - PIJ[0][b] - PIJ[1][b];
    PIK[2][b] = Sk[b] - PIK[0][b] - PIK[1][b];
    PJK[2][b] = Sk[b] - PJK[0][b] - PJK[1][b];
  }
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < 2; b++) {
      T[9 * a + 3 * b + 0] = t8[4 * a + 2 * b + 0];
      T[9 * a + 3 * b + 1] = t8[4 * a + 2 * b + 1];
      T[9 * a + 3 * b + 2] = PIJ[a][b] - t8[4 * a + 2 * b + 0] - t8[4 * a + 2 * b + 1];
    }
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int c = 0; c < 3; c++) T[9 * a + 6 + c] = PIK[a][c] - T[9 * a + c] - T[9 * a + 3 + c];
#pragma unroll
  for (int b = 0; b < 3; b++)
#pragma unroll
    for (int c = 0; c < 3; c++) T[18 + 3 * b + c] = PJK[b][c] - T[3 * b + c] - T[9 + 3 * b + c];
}

__device__ __forceinline__ float k2_score(const uint32_t (&T0)[27], const uint32_t (&T1)[27],
                                          const float* __restrict__ lut) {
  float score = 0.0f;
#pragma unroll
  for (int c = 0; c < 27; c++) {
    const float d = __fsub_rn(__ldg(lut + T0[c] + T1[c] + 1), __ldg(lut + T0[c]));
    score = __fadd_rn(score, __fsub_rn(d, __ldg(lut + T1[c])));
  }
  return fabsf(score);
}

// The same sum with the table in shared memory (lut points into the kernel's dynamic
// shared memory, so the lookups compile to shared-memory loads).
__device__ __forceinline__ float k2_score_shared(const uint32_t (&T0)[27], const uint32_t (&T1)[27],
                                                 const float* lut) {
  float score = 0.0f;
#pragma unroll
  for (int c = 0; c < 27; c++) {
    const float d = __fsub_rn(lut[T0[c] + T1[c] + 1], lut[T0[c]]);
    score = __fadd_rn(score, __fsub_rn(d, lut[T1[c]]));
  }
  return fabsf(score);
}

// Insert (s, key) into a warp-distributed sorted list (lane r holds the r-th best).
__device__ __forceinline__ void warp_list_insert(float& ls, unsigned long long& lk, float s, unsigned long long key,
                                                 int lane) {
  const unsigned before = __ballot_sync(kFull, better(ls, lk, s, key));
  const int pos = __popc(before);  // entries strictly better than the candidate
  const float us = __shfl_up_sync(kFull, ls, 1);
  const unsigned long long uk = __shfl_up_sync(kFull, lk, 1);
  if (lane > pos) {
    ls = us;
    lk = uk;
  } else if (lane == pos) {
    ls = s;
    lk = key;
  }
}

}  // namespace epik2
