// ref_tap_tables.cpp -- records every triplet's contingency table and K2 score as
// computed by the reference's own unblocked CPU search (CPU/v2.cpp).
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile from the unmodified reference
// source (included by path through -I).  CPU/v2.cpp built with NUM_THREADS=1 visits
// the triplets i<j<k in lexicographic order (CPU/v2.cpp:240-256) and, for each, fills
// its 54-entry frequency table `ft` (allocated once with _mm_malloc, CPU/v2.cpp:233)
// and then calls fabs(score) exactly once (CPU/v2.cpp:520).  Two taps observe this
// without changing the computation:
//   * _mm_malloc is routed through tap_mm_malloc, which remembers the 216-byte `ft`
//     allocation;
//   * fabs is routed through tap_fabs, which appends the current `ft` and the signed
//     score to the output before returning the absolute value.
//
// Usage:
//   ref_tap_tables file <geno.bin> <n_samples> <n_snps> <out.bin>
//   ref_tap_tables gen <n_samples> <n_snps> <out.bin>
// out.bin: int64 N, int64 M, int64 T, then N*M genotype bytes, N phenotype bytes,
//          T*54 uint32 tables, T float32 scores (fabs applied), in lexicographic order.

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <immintrin.h>
#include <omp.h>
#include <float.h>
#include <limits.h>
#include <math.h>

static uint32_t* g_ft = nullptr;
static std::vector<uint32_t> g_tables;
static std::vector<float> g_scores;

static inline void* tap_mm_malloc(size_t size, size_t align) {
  void* p = _mm_malloc(size, align);
  if (size == 2 * 27 * sizeof(uint32_t)) g_ft = (uint32_t*)p;
  return p;
}

static inline float tap_fabs(float x) {
  float r = std::fabs(x);
  if (g_ft) {
    g_tables.insert(g_tables.end(), g_ft, g_ft + 54);
    g_scores.push_back(r);
  }
  return r;
}

#define _mm_malloc tap_mm_malloc
#define fabs tap_fabs
#define main ref_main
#include REF_SOURCE
#undef main
#undef fabs
#undef _mm_malloc

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  std::string mode = argv[1];
  long long N, M;
  uint8_t *A, *B;
  const char* out;
  if (mode == "file" && argc >= 6) {
    N = atoll(argv[3]);
    M = atoll(argv[4]);
    out = argv[5];
    A = (uint8_t*)_mm_malloc(N * M, 64);
    B = (uint8_t*)_mm_malloc(N + 64, 64);
    FILE* f = fopen(argv[2], "rb");
    if (!f) return 3;
    if (fread(A, 1, N * M, f) != (size_t)(N * M) || fread(B, 1, N, f) != (size_t)N) return 3;
    fclose(f);
  } else if (mode == "gen" && argc >= 5) {
    N = atoll(argv[2]);
    M = atoll(argv[3]);
    out = argv[4];
    generate_data(N, M, &A, &B);
  } else {
    return 2;
  }
  std::vector<uint8_t> Acopy(A, A + N * M), Bcopy(B, B + N);

  addlogtable = new float[TABLE_MAX_SIZE];
  for (int i = 0; i < TABLE_MAX_SIZE; i++) addlogtable[i] = my_factorial(i);
  uint32_t *z, *o;
  long long phen_ones;
  A = transpose_data(N, M, A);
  transposed_to_binary(A, B, &z, &o, &phen_ones, M, N);
  process_epi_bin_no_phen_nor(z, o, phen_ones, 3, M, N, 27);

  long long T = (long long)g_scores.size();
  FILE* f = fopen(out, "wb");
  if (!f) return 3;
  fwrite(&N, 8, 1, f);
  fwrite(&M, 8, 1, f);
  fwrite(&T, 8, 1, f);
  fwrite(Acopy.data(), 1, N * M, f);
  fwrite(Bcopy.data(), 1, N, f);
  fwrite(g_tables.data(), 4, g_tables.size(), f);
  fwrite(g_scores.data(), 4, g_scores.size(), f);
  fclose(f);
  return 0;
}
