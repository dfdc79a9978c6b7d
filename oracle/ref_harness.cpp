// ref_harness.cpp -- drives the reference's own CPU search on data read from a file.
//
// TEST / BASELINE INFRASTRUCTURE ONLY.  Built by oracle/Makefile from the unmodified
// reference sources (the source file is included by path through -I; nothing of it
// is copied here).  The harness replaces only the reference's main():
//   * the genotype matrix and phenotype come from a file (or from the reference's own
//     generate_data, mode "gen"), instead of always from generate_data;
//   * omp_set_num_threads is routed through ref_threads() so one binary built with a
//     large NUM_THREADS can run with the thread count given in REF_THREADS;
//   * printf is routed through tap_printf, which also prints the best score's exact
//     float bits (the reference prints it with %f only).
// The search itself runs the reference's functions in the order of its main
// (CPU/v4_popc_avx512.cpp:4583-4630, CPU/v2.cpp:559-600).
//
// Usage:
//   ref_harness file <geno.bin> <n_samples> <n_snps> [block_pac block_snp]
//       geno.bin = n_samples*n_snps genotype bytes (sample-major) + n_samples phenotype bytes
//   ref_harness gen <n_samples> <n_snps> [block_pac block_snp]
//   ref_harness addlog <n_max> <out.bin>        (raw float32 addlog(0..n_max))

// All standard headers first: the reference defines a min(a,b) macro that breaks them.
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <cstdarg>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <immintrin.h>
#include <omp.h>
#include <float.h>
#include <limits.h>
#include <math.h>

static int ref_threads(int compiled) {
  const char* e = getenv("REF_THREADS");
  int t = e ? atoi(e) : omp_get_num_procs();
  if (t < 1) t = 1;
  if (t > compiled) t = compiled;
  omp_set_num_threads(t);
  return t;
}

static int tap_printf(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  int r = vprintf(fmt, ap);
  va_end(ap);
  if (strncmp(fmt, "Best SNPs", 9) == 0) {
    va_list aq;
    va_start(aq, fmt);
    int a = va_arg(aq, int), b = va_arg(aq, int), c = va_arg(aq, int);
    double s = va_arg(aq, double);
    va_end(aq);
    float f = (float)s;
    uint32_t bits;
    memcpy(&bits, &f, 4);
    printf("EXACT %d %d %d %a 0x%08x\n", a, b, c, s, bits);
  }
  return r;
}

#define omp_set_num_threads(n) ref_threads(n)
#define printf tap_printf
#define main ref_main
#include REF_SOURCE
#undef main
#undef printf
#undef omp_set_num_threads

static double now_s() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: %s file|gen|addlog ...\n", argv[0]);
    return 2;
  }
  std::string mode = argv[1];
  addlogtable = new float[TABLE_MAX_SIZE];
  for (int i = 0; i < TABLE_MAX_SIZE; i++) addlogtable[i] = my_factorial(i);

  if (mode == "addlog") {
    if (argc < 4) return 2;
    long n_max = atol(argv[2]);
    FILE* f = fopen(argv[3], "wb");
    if (!f) return 3;
    for (long n = 0; n <= n_max; n++) {
      float v = addlog((int)n);
      fwrite(&v, 4, 1, f);
    }
    fclose(f);
    return 0;
  }

  long long N, M;
  uint8_t *A, *B;
  int argi;
  if (mode == "file") {
    if (argc < 5) return 2;
    N = atoll(argv[3]);
    M = atoll(argv[4]);
    A = (uint8_t*)_mm_malloc(N * M, 64);
    B = (uint8_t*)_mm_malloc(N + 64, 64);
    FILE* f = fopen(argv[2], "rb");
    if (!f) { fprintf(stderr, "cannot open %s\n", argv[2]); return 3; }
    if (fread(A, 1, N * M, f) != (size_t)(N * M) || fread(B, 1, N, f) != (size_t)N) {
      fprintf(stderr, "short read\n");
      return 3;
    }
    fclose(f);
    argi = 5;
  } else if (mode == "gen") {
    if (argc < 4) return 2;
    N = atoll(argv[2]);
    M = atoll(argv[3]);
    generate_data(N, M, &A, &B);
    argi = 4;
  } else {
    return 2;
  }

#if REF_BLOCKED
  int block_pac = argc > argi ? atoi(argv[argi]) : 64;
  int block_snp = argc > argi + 1 ? atoi(argv[argi + 1]) : 16;
#endif
  uint32_t *z, *o;
  long long phen_ones;
  double t0 = now_s();
  A = transpose_data(N, M, A);
  transposed_to_binary(A, B, &z, &o, &phen_ones, M, N);
#if REF_BLOCKED
  z = transform_data_2_block(N - phen_ones, M, z, block_pac, block_snp);
  o = transform_data_2_block(phen_ones, M, o, block_pac, block_snp);
#endif
  double t1 = now_s();
#if REF_BLOCKED
  process_epi_bin_no_phen_nor_block(z, o, phen_ones, 3, M, N, 27, block_snp, block_pac);
#else
  process_epi_bin_no_phen_nor(z, o, phen_ones, 3, M, N, 27);
#endif
  double t2 = now_s();
  const char* e = getenv("REF_THREADS");
  int threads = e ? atoi(e) : omp_get_num_procs();
  if (threads > NUM_THREADS) threads = NUM_THREADS;
  fprintf(stdout, "WALL_ENCODE_S %.6f\nWALL_SEARCH_S %.6f\nTHREADS %d\n", t1 - t0, t2 - t1, threads);
  return 0;
}
