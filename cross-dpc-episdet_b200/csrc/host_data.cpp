// Host-side data sources and the K2 log-factorial table.
//
// Compiled with -ffp-contract=off so that every double expression below rounds
// exactly as written (the table must match the reference CPU path bit for bit).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <random>
#include <vector>

#include "epik2_internal.h"

namespace epik2 {

// ln n! as the reference CPU path computes it (CPU/v4_popc_avx512.cpp:213-241):
//   n < 748 : t[0] = t[1] = 0, t[n] = (float)((double)t[n-1] + log(n))      (my_factorial)
//   n >= 748: (float)((n + 0.5) * log(n) - (n - 1) * log(exp(1)) + TABLE_ERROR) in double
// The reference's GPU kernels evaluate the Stirling tail in float with the SYCL device
// log/exp (GPU/v4.cpp:52-61); that arithmetic is not reproducible here, so the search
// follows the CPU path, which the reference's CPU programs all share.
void build_k2_lut_range(int64_t n_begin, int64_t n_end, float* out) {
  const double table_error = -0.0810;  // TABLE_ERROR, GPU/v4.cpp:16
  float t[kTableMaxSize];
  t[0] = 0.0f;
  t[1] = 0.0f;
  for (int n = 2; n < kTableMaxSize; n++) t[n] = (float)((double)t[n - 1] + std::log((double)n));
  const double log_e = std::log(std::exp(1.0));
  for (int64_t n = n_begin; n < n_end; n++) {
    if (n < kTableMaxSize) {
      out[n - n_begin] = t[n];
    } else {
      double a = ((double)n + 0.5) * std::log((double)n);
      double b = (double)(n - 1) * log_e;
      out[n - n_begin] = (float)(a - b + table_error);
    }
  }
}

void build_k2_lut(int64_t n_max, float* lut) { build_k2_lut_range(0, n_max + 1, lut); }

// The same ln n! evaluated entirely in double (precision form's FP64 rescore): the table
// part accumulated in double, the Stirling tail in double and not rounded to float.
void build_k2_lut64(int64_t n_max, double* lut) {
  const double table_error = -0.0810;
  const double log_e = std::log(std::exp(1.0));
  double acc = 0.0;
  for (int64_t n = 0; n <= n_max; n++) {
    if (n < kTableMaxSize) {
      if (n >= 2) acc += std::log((double)n);
      lut[n] = acc;
    } else {
      lut[n] = ((double)n + 0.5) * std::log((double)n) - (double)(n - 1) * log_e + table_error;
    }
  }
}

// The reference's synthetic input (GPU/v4.cpp:81-110): srand(100); rand()%3 per
// genotype in sample-major order; exactly n/2 cases by rejection sampling.  An index
// equal to n (rand()==RAND_MAX) is dropped, which is where the reference's write lands
// outside its phenotype vector.
void generate_reference(int64_t n, int64_t m, uint8_t* geno, uint8_t* pheno) {
  srand(100);
  for (int64_t i = 0; i < n; i++)
    for (int64_t j = 0; j < m; j++) geno[i * m + j] = (uint8_t)(rand() % 3);
  std::vector<uint8_t> b((size_t)n + 1, 0);
  for (int64_t i = 0; i < n / 2; i++) {
    int index = (int)(n * ((double)rand() / (RAND_MAX)));
    while (b[(size_t)index] == 1) index = (int)(n * ((double)rand() / (RAND_MAX)));
    b[(size_t)index] = 1;
  }
  for (int64_t i = 0; i < n; i++) pheno[i] = b[(size_t)i];
}

// Seeded Hardy-Weinberg matrix with planted triplets (benchmark workloads).
//   p_m = lo + (hi-lo)*u, then per sample, per SNP: g = 0 if u < q^2, 1 if u < q^2+2pq,
//   else 2 (q = 1-p).  u = (x >> 11) * 2^-53 from std::mt19937_64(seed).
//   Exactly n_cases cases: risk r_s = the largest effect among planted triplets whose
//   three SNPs all carry >= 1 minor allele, else r0 so that the risks sum to n_cases;
//   cases are the n_cases largest Efraimidis-Spirakis keys log(u')/w, w = r/(1-r),
//   u' = ((x >> 11) + 1) * 2^-53, ties to the lower sample index.
void generate_hwe(uint64_t seed, int64_t n, int64_t m, int64_t n_cases, double maf_lo, double maf_hi,
                  int n_planted, const int64_t* planted, const double* effects, uint8_t* geno, uint8_t* pheno) {
  std::mt19937_64 rng(seed);
  const double inv53 = 1.0 / 9007199254740992.0;
  auto u01 = [&]() { return (double)(rng() >> 11) * inv53; };
  std::vector<double> p((size_t)std::max<int64_t>(m, 1));
  for (int64_t j = 0; j < m; j++) p[(size_t)j] = maf_lo + (maf_hi - maf_lo) * u01();
  for (int64_t s = 0; s < n; s++) {
    uint8_t* row = geno + s * m;
    for (int64_t j = 0; j < m; j++) {
      double u = u01();
      double q = 1.0 - p[(size_t)j];
      double t0 = q * q;
      double t1 = t0 + 2.0 * p[(size_t)j] * q;
      row[j] = (uint8_t)(u < t0 ? 0 : (u < t1 ? 1 : 2));
    }
  }
  std::vector<double> risk((size_t)std::max<int64_t>(n, 1), -1.0);
  int64_t n_car = 0;
  double car_sum = 0.0;
  for (int64_t s = 0; s < n; s++) {
    double best = -1.0;
    for (int t = 0; t < n_planted; t++) {
      const int64_t* tr = planted + 3 * t;
      const uint8_t* row = geno + s * m;
      if (row[tr[0]] >= 1 && row[tr[1]] >= 1 && row[tr[2]] >= 1 && effects[t] > best) best = effects[t];
    }
    risk[(size_t)s] = best;
    if (best >= 0.0) {
      n_car++;
      car_sum += best;
    }
  }
  double r0 = (n > n_car) ? ((double)n_cases - car_sum) / (double)(n - n_car) : 0.5;
  r0 = std::min(std::max(r0, 1e-9), 1.0 - 1e-9);
  std::vector<std::pair<double, int64_t>> keys((size_t)n);
  for (int64_t s = 0; s < n; s++) {
    double rs = risk[(size_t)s] >= 0.0 ? risk[(size_t)s] : r0;
    double w = rs / (1.0 - rs);
    double u = ((double)(rng() >> 11) + 1.0) * inv53;
    keys[(size_t)s] = {std::log(u) / w, s};
  }
  std::sort(keys.begin(), keys.end(), [](const std::pair<double, int64_t>& a, const std::pair<double, int64_t>& b) {
    if (a.first != b.first) return a.first > b.first;
    return a.second < b.second;
  });
  for (int64_t s = 0; s < n; s++) pheno[s] = 0;
  for (int64_t s = 0; s < n_cases && s < n; s++) pheno[keys[(size_t)s].second] = 1;
}

}  // namespace epik2
