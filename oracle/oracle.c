/*
 * oracle.c -- CPU restatement of the reference's third-order K2 epistasis search.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: only the
 * test suite, the smoke check and the CPU-baseline leg of the benchmark load it.
 * The product library never links it and has no CPU fallback.
 *
 * Every function restates one step of hiperbio/cross-dpc-episdet (paths relative
 * to that project):
 *   oracle_gen_reference   GPU/v4.cpp:81-110, CPU/v2.cpp:56-80   (srand(100)/rand() data)
 *   oracle_encode          GPU/v2.cpp:124-184, CPU/v2.cpp:95-150 (per-class {g0,g1} planes)
 *   oracle_masks           GPU/v2.cpp:215-221, CPU/v2.cpp:224-231
 *   oracle_table           GPU/v2.cpp:288-540 (NOR-derived g2, 27 AND3 + popcount per class)
 *   oracle_lut             CPU/v2.cpp:177-200 (my_factorial table, addlog Stirling tail, CPU
 *                          double arithmetic stored to float)
 *   oracle_k2              CPU/v2.cpp:514-517 (float accumulation in cell order, then fabs)
 *   oracle_scan            CPU/v2.cpp:240-525 (lexicographic i<j<k visit, strict '<' keeps the
 *                          lowest index on ties)
 * plus the seeded Hardy-Weinberg/planted generator of the benchmark workloads
 * (oracle_gen_hwe, restated independently of the product's C++ copy) and an FP64
 * K2 oracle (oracle_k2_fp64: table and Stirling tail in double).
 *
 * Cell order: c = 9*g_i + 3*g_j + g_k; controls (phenotype 0) fill ft[0..26],
 * cases (phenotype 1) fill ft[27..53]  (GPU/v4.cpp:317-319).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_TABLE_MAX_SIZE 748   /* CPU/v2.cpp:12 */
#define ORACLE_TABLE_ERROR (-0.0810) /* CPU/v2.cpp:13 */

/* ------------------------------------------------------------------ */
/* glibc rand() generator, as the reference's generate_data           */
/* ------------------------------------------------------------------ */

/* A is [N][M] sample-major, B is [N].  B must hold N+1 bytes: the reference's
 * rejection sampler can draw index N when rand()==RAND_MAX (GPU/v4.cpp:104);
 * that write lands outside the phenotype vector, which B[N] absorbs here. */
void oracle_gen_reference(int64_t N, int64_t M, uint8_t *A, uint8_t *B) {
  srand(100);
  for (int64_t i = 0; i < N; i++)
    for (int64_t j = 0; j < M; j++) A[i * M + j] = (uint8_t)(rand() % 3);
  for (int64_t i = 0; i <= N; i++) B[i] = 0;
  for (int64_t i = 0; i < N / 2; i++) {
    int index = (int)(N * ((double)rand() / (RAND_MAX)));
    while (B[index] == 1) index = (int)(N * ((double)rand() / (RAND_MAX)));
    B[index] = 1;
  }
}

/* ------------------------------------------------------------------ */
/* MT19937-64 (Matsumoto & Nishimura 2004), restated from the paper    */
/* ------------------------------------------------------------------ */
typedef struct { uint64_t mt[312]; int idx; } oracle_mt64;

static void mt64_seed(oracle_mt64 *r, uint64_t seed) {
  r->mt[0] = seed;
  for (int i = 1; i < 312; i++)
    r->mt[i] = 6364136223846793005ULL * (r->mt[i - 1] ^ (r->mt[i - 1] >> 62)) + (uint64_t)i;
  r->idx = 312;
}

static uint64_t mt64_next(oracle_mt64 *r) {
  if (r->idx >= 312) {
    for (int i = 0; i < 312; i++) {
      uint64_t x = (r->mt[i] & 0xFFFFFFFF80000000ULL) | (r->mt[(i + 1) % 312] & 0x7FFFFFFFULL);
      uint64_t xa = x >> 1;
      if (x & 1ULL) xa ^= 0xB5026F5AA96619E9ULL;
      r->mt[i] = r->mt[(i + 156) % 312] ^ xa;
    }
    r->idx = 0;
  }
  uint64_t y = r->mt[r->idx++];
  y ^= (y >> 29) & 0x5555555555555555ULL;
  y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
  y ^= (y << 37) & 0xFFF7EEE000000000ULL;
  y ^= y >> 43;
  return y;
}

/* n-th output (1-based) of a generator seeded with `seed`; used by the tests to
 * pin the generator to the published check value. */
uint64_t oracle_mt64_nth(uint64_t seed, int64_t n) {
  oracle_mt64 r;
  mt64_seed(&r, seed);
  uint64_t v = 0;
  for (int64_t i = 0; i < n; i++) v = mt64_next(&r);
  return v;
}

static double u01(oracle_mt64 *r) { return (double)(mt64_next(r) >> 11) * (1.0 / 9007199254740992.0); }
static double u01_open0(oracle_mt64 *r) {
  return ((double)(mt64_next(r) >> 11) + 1.0) * (1.0 / 9007199254740992.0);
}

typedef struct { double key; int64_t idx; } oracle_keyed;
static int keyed_cmp(const void *a, const void *b) {
  const oracle_keyed *x = (const oracle_keyed *)a, *y = (const oracle_keyed *)b;
  if (x->key > y->key) return -1;
  if (x->key < y->key) return 1;
  return (x->idx < y->idx) ? -1 : (x->idx > y->idx);
}

/*
 * Seeded Hardy-Weinberg genotype matrix with planted triplets (benchmark data).
 *   p_m ~ U[maf_lo, maf_hi] (M draws), then for each sample s, each SNP m:
 *   u ~ U[0,1): g = 0 if u < q^2, 1 if u < q^2 + 2pq, else 2   (q = 1 - p).
 *   Exactly n_cases cases: sample s has risk r_s = max effect over planted
 *   triplets whose three SNPs all carry >= 1 minor allele, else r0 chosen so the
 *   risks sum to n_cases; cases are drawn by weighted sampling without
 *   replacement with Efraimidis-Spirakis keys log(u)/w, w = r/(1-r).
 * A is [N][M] sample-major like the reference's generate_data (GPU/v4.cpp:94).
 */
void oracle_gen_hwe(uint64_t seed, int64_t N, int64_t M, int64_t n_cases, double maf_lo, double maf_hi,
                    int n_planted, const int64_t *planted /* [n_planted][3] */, const double *effects,
                    uint8_t *A, uint8_t *B) {
  oracle_mt64 r;
  mt64_seed(&r, seed);
  double *p = (double *)malloc(sizeof(double) * (size_t)(M > 0 ? M : 1));
  for (int64_t m = 0; m < M; m++) p[m] = maf_lo + (maf_hi - maf_lo) * u01(&r);
  for (int64_t s = 0; s < N; s++) {
    for (int64_t m = 0; m < M; m++) {
      double u = u01(&r);
      double q = 1.0 - p[m];
      double t0 = q * q;
      double t1 = t0 + 2.0 * p[m] * q;
      A[s * M + m] = (uint8_t)(u < t0 ? 0 : (u < t1 ? 1 : 2));
    }
  }
  double *risk = (double *)malloc(sizeof(double) * (size_t)(N > 0 ? N : 1));
  int64_t n_car = 0;
  double car_sum = 0.0;
  for (int64_t s = 0; s < N; s++) {
    double best = -1.0;
    for (int t = 0; t < n_planted; t++) {
      const int64_t *tr = planted + 3 * t;
      if (A[s * M + tr[0]] >= 1 && A[s * M + tr[1]] >= 1 && A[s * M + tr[2]] >= 1 && effects[t] > best)
        best = effects[t];
    }
    risk[s] = best;
    if (best >= 0.0) { n_car++; car_sum += best; }
  }
  double r0 = (N > n_car) ? ((double)n_cases - car_sum) / (double)(N - n_car) : 0.5;
  if (r0 < 1e-9) r0 = 1e-9;
  if (r0 > 1.0 - 1e-9) r0 = 1.0 - 1e-9;
  oracle_keyed *keys = (oracle_keyed *)malloc(sizeof(oracle_keyed) * (size_t)(N > 0 ? N : 1));
  for (int64_t s = 0; s < N; s++) {
    double rs = risk[s] >= 0.0 ? risk[s] : r0;
    double w = rs / (1.0 - rs);
    keys[s].key = log(u01_open0(&r)) / w;
    keys[s].idx = s;
  }
  qsort(keys, (size_t)N, sizeof(oracle_keyed), keyed_cmp);
  for (int64_t s = 0; s < N; s++) B[s] = 0;
  for (int64_t s = 0; s < n_cases && s < N; s++) B[keys[s].idx] = 1;
  free(keys);
  free(risk);
  free(p);
}

/* ------------------------------------------------------------------ */
/* Encoding                                                            */
/* ------------------------------------------------------------------ */

/* Planes in the reference's CPU layout [snp][word][2] per class (CPU/v2.cpp:122-150):
 * a sample shifts every word of its class left by one and sets bit 0 of plane g when
 * its genotype is g in {0,1}; genotype 2 (and any other value) sets neither.
 * z holds controls (phenotype != 1), o holds cases (phenotype == 1). */
void oracle_encode(const uint8_t *A, const uint8_t *B, int64_t N, int64_t M, uint32_t *z, uint32_t *o,
                   int64_t *n_cases_out) {
  int64_t n1 = 0;
  for (int64_t s = 0; s < N; s++) n1 += (B[s] == 1);
  int64_t n0 = N - n1;
  int64_t W0 = (n0 + 31) / 32, W1 = (n1 + 31) / 32;
  memset(z, 0, sizeof(uint32_t) * (size_t)(M * W0 * 2));
  memset(o, 0, sizeof(uint32_t) * (size_t)(M * W1 * 2));
  for (int64_t m = 0; m < M; m++) {
    int64_t c0 = 0, c1 = 0;
    for (int64_t s = 0; s < N; s++) {
      uint32_t g = A[s * M + m];
      uint32_t *w;
      if (B[s] == 1) { w = &o[(m * W1 + c1 / 32) * 2]; c1++; }
      else { w = &z[(m * W0 + c0 / 32) * 2]; c0++; }
      w[0] <<= 1;
      w[1] <<= 1;
      if (g == 0 || g == 1) w[g] |= 1u;
    }
  }
  *n_cases_out = n1;
}

/* Last-word masks for the derived genotype-2 plane: 0xFFFFFFFF >> (32*W - n). */
void oracle_masks(int64_t n0, int64_t n1, uint32_t *mask0, uint32_t *mask1) {
  int64_t W0 = (n0 + 31) / 32, W1 = (n1 + 31) / 32;
  *mask0 = 0xFFFFFFFFu >> (uint32_t)(W0 * 32 - n0);
  *mask1 = 0xFFFFFFFFu >> (uint32_t)(W1 * 32 - n1);
}

/* ------------------------------------------------------------------ */
/* Contingency tables                                                  */
/* ------------------------------------------------------------------ */

/* 27 counts of one class for SNPs (i,j,k): g2 = ~(g0|g1), masked on the last word. */
static void table_class(const uint32_t *P, int64_t W, uint32_t mask, int64_t i, int64_t j, int64_t k,
                        uint32_t *ft) {
  for (int c = 0; c < 27; c++) ft[c] = 0;
  if (W == 0) return;
  const uint32_t *a = P + i * W * 2, *b = P + j * W * 2, *t = P + k * W * 2;
  for (int64_t w = 0; w < W; w++) {
    uint32_t m = (w == W - 1) ? mask : 0xFFFFFFFFu;
    uint32_t ga[3] = {a[2 * w], a[2 * w + 1], ~(a[2 * w] | a[2 * w + 1]) & m};
    uint32_t gb[3] = {b[2 * w], b[2 * w + 1], ~(b[2 * w] | b[2 * w + 1]) & m};
    uint32_t gt[3] = {t[2 * w], t[2 * w + 1], ~(t[2 * w] | t[2 * w + 1]) & m};
    for (int x = 0; x < 3; x++)
      for (int y = 0; y < 3; y++) {
        uint32_t ab = ga[x] & gb[y];
        for (int q = 0; q < 3; q++) ft[9 * x + 3 * y + q] += (uint32_t)__builtin_popcount(ab & gt[q]);
      }
  }
}

void oracle_table(const uint32_t *z, const uint32_t *o, int64_t n0, int64_t n1, int64_t i, int64_t j,
                  int64_t k, uint32_t *ft54) {
  uint32_t m0, m1;
  oracle_masks(n0, n1, &m0, &m1);
  table_class(z, (n0 + 31) / 32, m0, i, j, k, ft54);
  table_class(o, (n1 + 31) / 32, m1, i, j, k, ft54 + 27);
}

/* ------------------------------------------------------------------ */
/* K2 score                                                            */
/* ------------------------------------------------------------------ */

/* lut[n] = addlog(n) of the CPU reference for n in [0, n_max]:
 *   n < 748: t[0]=t[1]=0, t[n] = (float)((double)t[n-1] + log(n))   (my_factorial)
 *   n >= 748: (float)((n + 0.5)*log(n) - (n - 1)*log(exp(1)) + TABLE_ERROR)  in double. */
void oracle_lut(int64_t n_max, float *lut) {
  float t[ORACLE_TABLE_MAX_SIZE];
  t[0] = 0.0f;
  t[1] = 0.0f;
  for (int n = 2; n < ORACLE_TABLE_MAX_SIZE; n++) {
    volatile double acc = (double)t[n - 1] + log((double)n);
    t[n] = (float)acc;
  }
  for (int64_t n = 0; n <= n_max; n++) {
    if (n < ORACLE_TABLE_MAX_SIZE) {
      lut[n] = t[n];
    } else {
      volatile double a = ((double)n + 0.5) * log((double)n);
      volatile double b = (double)(n - 1) * log(exp(1.0));
      volatile double x = a - b + ORACLE_TABLE_ERROR;
      lut[n] = (float)x;
    }
  }
}

/* score = |sum_c (lut[n0+n1+1] - lut[n0]) - lut[n1]| in float, cells in order. */
float oracle_k2(const uint32_t *ft54, const float *lut) {
  float score = 0.0f;
  for (int c = 0; c < 27; c++) {
    volatile float d = lut[ft54[c] + ft54[27 + c] + 1] - lut[ft54[c]];
    volatile float e = d - lut[ft54[27 + c]];
    score = score + e;
  }
  return fabsf(score);
}

/* FP64 oracle: ln n! accumulated in double below 748, Stirling tail in double above. */
double oracle_lnfact_fp64(int64_t n) {
  static double t[ORACLE_TABLE_MAX_SIZE];
  static int init = 0;
  if (!init) {
    t[0] = 0.0;
    t[1] = 0.0;
    for (int q = 2; q < ORACLE_TABLE_MAX_SIZE; q++) t[q] = t[q - 1] + log((double)q);
    init = 1;
  }
  if (n < ORACLE_TABLE_MAX_SIZE) return t[n];
  return ((double)n + 0.5) * log((double)n) - (double)(n - 1) * log(exp(1.0)) + ORACLE_TABLE_ERROR;
}

double oracle_k2_fp64(const uint32_t *ft54) {
  double s = 0.0;
  for (int c = 0; c < 27; c++)
    s += oracle_lnfact_fp64(ft54[c] + ft54[27 + c] + 1) - oracle_lnfact_fp64(ft54[c]) -
         oracle_lnfact_fp64(ft54[27 + c]);
  return fabs(s);
}

/* Same formula with exact ln n! = lgamma(n+1) (secondary reference figure). */
double oracle_k2_lgamma(const uint32_t *ft54) {
  double s = 0.0;
  for (int c = 0; c < 27; c++) {
    double a = ft54[c], b = ft54[27 + c];
    s += lgamma(a + b + 2.0) - lgamma(a + 1.0) - lgamma(b + 1.0);
  }
  return fabs(s);
}

/* ------------------------------------------------------------------ */
/* Exhaustive scan                                                     */
/* ------------------------------------------------------------------ */

typedef struct { float score; int64_t i, j, k; } oracle_best;

static int better(float s, int64_t i, int64_t j, int64_t k, const oracle_best *b) {
  if (s < b->score) return 1;
  if (s > b->score) return 0;
  if (i != b->i) return i < b->i;
  if (j != b->j) return j < b->j;
  return k < b->k;
}

/* Lexicographic index of triplet (i<j<k) among all C(M,3). */
int64_t oracle_triplet_index(int64_t M, int64_t i, int64_t j, int64_t k) {
  /* triplets with first index < i */
  int64_t before_i = 0;
  /* sum_{a<i} C(M-1-a, 2) = C(M,3) - C(M-i,3) */
  int64_t Mi = M - i;
  int64_t cM3 = M * (M - 1) * (M - 2) / 6, cMi3 = Mi * (Mi - 1) * (Mi - 2) / 6;
  before_i = cM3 - cMi3;
  /* pairs (j', k') with i < j' < j: sum_{b=i+1}^{j-1} (M-1-b) */
  int64_t nb = j - i - 1;
  int64_t before_j = nb * (M - 1) - (nb * (i + 1) + nb * (nb - 1) / 2);
  return before_i + before_j + (k - j - 1);
}

/*
 * Full scan over all i<j<k of SNPs [0, M).  Writes the best (lowest score, ties to
 * the lowest (i,j,k)) and, when tables/scores are non-NULL, every triplet's 54
 * counts and score at its lexicographic index.  Returns the number of triplets.
 */
int64_t oracle_scan(const uint32_t *z, const uint32_t *o, int64_t n0, int64_t n1, int64_t M, const float *lut,
                    float *best_score, int64_t *best_ijk, uint32_t *tables, float *scores, int n_threads) {
  oracle_best g = {FLT_MAX, -1, -1, -1};
  int64_t T = (M >= 3) ? M * (M - 1) * (M - 2) / 6 : 0;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel
#endif
  {
    oracle_best b = {FLT_MAX, -1, -1, -1};
    uint32_t ft[54];
#ifdef _OPENMP
#pragma omp for schedule(dynamic)
#endif
    for (int64_t i = 0; i < M - 2; i++) {
      for (int64_t j = i + 1; j < M - 1; j++) {
        for (int64_t k = j + 1; k < M; k++) {
          oracle_table(z, o, n0, n1, i, j, k, ft);
          float s = oracle_k2(ft, lut);
          if (tables || scores) {
            int64_t t = oracle_triplet_index(M, i, j, k);
            if (tables) memcpy(tables + 54 * t, ft, sizeof(ft));
            if (scores) scores[t] = s;
          }
          if (better(s, i, j, k, &b)) { b.score = s; b.i = i; b.j = j; b.k = k; }
        }
      }
    }
#ifdef _OPENMP
#pragma omp critical
#endif
    {
      if (b.i >= 0 && better(b.score, b.i, b.j, b.k, &g)) g = b;
    }
  }
  *best_score = g.score;
  best_ijk[0] = g.i;
  best_ijk[1] = g.j;
  best_ijk[2] = g.k;
  return T;
}

/* Convenience: genotype matrix in, best triplet out (encode + LUT + scan). */
int64_t oracle_scan_u8(const uint8_t *A, const uint8_t *B, int64_t N, int64_t M, float *best_score,
                       int64_t *best_ijk, uint32_t *tables, float *scores, int n_threads) {
  int64_t n1 = 0;
  for (int64_t s = 0; s < N; s++) n1 += (B[s] == 1);
  int64_t n0 = N - n1;
  int64_t W0 = (n0 + 31) / 32, W1 = (n1 + 31) / 32;
  uint32_t *z = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(M * W0 * 2 + 1));
  uint32_t *o = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(M * W1 * 2 + 1));
  float *lut = (float *)malloc(sizeof(float) * (size_t)(N + 2));
  oracle_encode(A, B, N, M, z, o, &n1);
  oracle_lut(N + 1, lut);
  int64_t T = oracle_scan(z, o, n0, n1, M, lut, best_score, best_ijk, tables, scores, n_threads);
  free(lut);
  free(o);
  free(z);
  return T;
}

/* FP64 K2 of every triplet at its lexicographic index (precision-form oracle). */
int64_t oracle_scan_fp64_u8(const uint8_t *A, const uint8_t *B, int64_t N, int64_t M, double *scores64,
                            int n_threads) {
  int64_t n1 = 0;
  for (int64_t s = 0; s < N; s++) n1 += (B[s] == 1);
  int64_t n0 = N - n1;
  int64_t W0 = (n0 + 31) / 32, W1 = (n1 + 31) / 32;
  uint32_t *z = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(M * W0 * 2 + 1));
  uint32_t *o = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(M * W1 * 2 + 1));
  oracle_encode(A, B, N, M, z, o, &n1);
  (void)oracle_lnfact_fp64(0); /* initialise the table before the parallel region */
  int64_t T = (M >= 3) ? M * (M - 1) * (M - 2) / 6 : 0;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic)
#endif
  for (int64_t i = 0; i < M - 2; i++) {
    uint32_t ft[54];
    for (int64_t j = i + 1; j < M - 1; j++)
      for (int64_t k = j + 1; k < M; k++) {
        oracle_table(z, o, n0, n1, i, j, k, ft);
        scores64[oracle_triplet_index(M, i, j, k)] = oracle_k2_fp64(ft);
      }
  }
  free(o);
  free(z);
  return T;
}

/* ------------------------------------------------------------------ */
/* FP64 top-k over all triplets (precision-form oracle at full size)   */
/* ------------------------------------------------------------------ */

typedef struct { double s; int64_t t; } oracle_cand;

/* (s, t) orders before (s2, t2): lower FP64 score, ties to the lower lexicographic index. */
static int cand_before(double s, int64_t t, double s2, int64_t t2) { return s < s2 || (s == s2 && t < t2); }

/* Max-heap of the k best candidates (root = the worst kept). */
static void heap_offer(oracle_cand *h, int *n, int k, double s, int64_t t) {
  if (*n < k) {
    int c = (*n)++;
    h[c].s = s;
    h[c].t = t;
    while (c > 0) {
      int p = (c - 1) / 2;
      if (!cand_before(h[p].s, h[p].t, h[c].s, h[c].t)) break;
      oracle_cand x = h[p]; h[p] = h[c]; h[c] = x;
      c = p;
    }
    return;
  }
  if (!cand_before(s, t, h[0].s, h[0].t)) return;
  h[0].s = s;
  h[0].t = t;
  int c = 0;
  for (;;) {
    int l = 2 * c + 1, r = l + 1, w = c;
    if (l < *n && cand_before(h[w].s, h[w].t, h[l].s, h[l].t)) w = l;
    if (r < *n && cand_before(h[w].s, h[w].t, h[r].s, h[r].t)) w = r;
    if (w == c) break;
    oracle_cand x = h[w]; h[w] = h[c]; h[c] = x;
    c = w;
  }
}

static int cand_cmp(const void *a, const void *b) {
  const oracle_cand *x = (const oracle_cand *)a, *y = (const oracle_cand *)b;
  if (cand_before(x->s, x->t, y->s, y->t)) return -1;
  if (cand_before(y->s, y->t, x->s, x->t)) return 1;
  return 0;
}

/* The k lowest FP64 K2 scores of all C(M,3) triplets (ties to the lowest index), in order:
 * out_t[r] = lexicographic triplet index, out_s64[r] = FP64 score, out_ft[r*54..] = table.
 * Counting is the definitional 27-cell AND3 + popcount of oracle_table (GPU/v2.cpp:288-540)
 * on the same per-class planes, two 32-bit words at a time; the nine (g_i, g_j) planes of a
 * pair are formed once and reused for every k.  Returns the number written (min(k, T)). */
int64_t oracle_topk_fp64_u8(const uint8_t *A, const uint8_t *B, int64_t N, int64_t M, int k, int64_t *out_t,
                            double *out_s64, uint32_t *out_ft, int n_threads) {
  int64_t n1 = 0;
  for (int64_t s = 0; s < N; s++) n1 += (B[s] == 1);
  int64_t n0 = N - n1;
  int64_t W[2] = {(n0 + 31) / 32, (n1 + 31) / 32};
  uint32_t *planes[2];
  planes[0] = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(M * W[0] * 2 + 1));
  planes[1] = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(M * W[1] * 2 + 1));
  oracle_encode(A, B, N, M, planes[0], planes[1], &n1);
  uint32_t mask[2];
  oracle_masks(n0, n1, &mask[0], &mask[1]);
  /* 64-bit words per class: {g0, g1, g2} of 64 samples, g2 masked on the last 32-bit word
   * and zero past the class */
  int64_t V[2] = {(W[0] + 1) / 2, (W[1] + 1) / 2};
  uint64_t *g64[2];
  for (int c = 0; c < 2; c++) {
    g64[c] = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(M * V[c] * 3 + 1));
    for (int64_t m = 0; m < M; m++)
      for (int64_t v = 0; v < V[c]; v++) {
        uint64_t g[3] = {0, 0, 0};
        for (int h = 0; h < 2; h++) {
          int64_t w = 2 * v + h;
          if (w >= W[c]) continue;
          uint32_t a0 = planes[c][(m * W[c] + w) * 2], a1 = planes[c][(m * W[c] + w) * 2 + 1];
          uint32_t mk = (w == W[c] - 1) ? mask[c] : 0xFFFFFFFFu;
          g[0] |= (uint64_t)a0 << (32 * h);
          g[1] |= (uint64_t)a1 << (32 * h);
          g[2] |= (uint64_t)(~(a0 | a1) & mk) << (32 * h);
        }
        for (int q = 0; q < 3; q++) g64[c][(m * V[c] + v) * 3 + q] = g[q];
      }
  }
  (void)oracle_lnfact_fp64(0); /* initialise the table before the parallel region */
  int64_t T = (M >= 3) ? M * (M - 1) * (M - 2) / 6 : 0;
  if (k < 1) k = 1;
  int n_thr = 1;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
  n_thr = omp_get_max_threads();
#endif
  oracle_cand *heaps = (oracle_cand *)malloc(sizeof(oracle_cand) * (size_t)k * (size_t)n_thr);
  int *heap_n = (int *)calloc((size_t)n_thr, sizeof(int));
  const int64_t VT = V[0] + V[1];
#ifdef _OPENMP
#pragma omp parallel
#endif
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    oracle_cand *h = heaps + (size_t)k * (size_t)tid;
    uint64_t *pij = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(9 * VT + 1));
    uint32_t ft[54];
#ifdef _OPENMP
#pragma omp for schedule(dynamic)
#endif
    for (int64_t i = 0; i < M - 2; i++) {
      for (int64_t j = i + 1; j < M - 1; j++) {
        for (int c = 0; c < 2; c++) {
          const uint64_t *a = g64[c] + i * V[c] * 3, *b = g64[c] + j * V[c] * 3;
          uint64_t *dst = pij + (c ? 9 * V[0] : 0);
          for (int64_t v = 0; v < V[c]; v++)
            for (int x = 0; x < 3; x++)
              for (int y = 0; y < 3; y++) dst[v * 9 + 3 * x + y] = a[v * 3 + x] & b[v * 3 + y];
        }
        for (int64_t kk = j + 1; kk < M; kk++) {
          for (int c = 0; c < 2; c++) {
            const uint64_t *t3 = g64[c] + kk * V[c] * 3;
            const uint64_t *src = pij + (c ? 9 * V[0] : 0);
            uint32_t cnt[27];
            for (int q = 0; q < 27; q++) cnt[q] = 0;
            for (int64_t v = 0; v < V[c]; v++) {
              const uint64_t k0 = t3[v * 3], k1 = t3[v * 3 + 1], k2 = t3[v * 3 + 2];
              for (int xy = 0; xy < 9; xy++) {
                const uint64_t ab = src[v * 9 + xy];
                cnt[3 * xy + 0] += (uint32_t)__builtin_popcountll(ab & k0);
                cnt[3 * xy + 1] += (uint32_t)__builtin_popcountll(ab & k1);
                cnt[3 * xy + 2] += (uint32_t)__builtin_popcountll(ab & k2);
              }
            }
            memcpy(ft + 27 * c, cnt, sizeof(cnt));
          }
          heap_offer(h, &heap_n[tid], k, oracle_k2_fp64(ft), oracle_triplet_index(M, i, j, kk));
        }
      }
    }
    free(pij);
  }
  /* merge the per-thread heaps */
  oracle_cand *all = (oracle_cand *)malloc(sizeof(oracle_cand) * (size_t)k * (size_t)n_thr + 1);
  int64_t n_all = 0;
  for (int t = 0; t < n_thr; t++)
    for (int q = 0; q < heap_n[t]; q++) all[n_all++] = heaps[(size_t)k * (size_t)t + (size_t)q];
  qsort(all, (size_t)n_all, sizeof(oracle_cand), cand_cmp);
  int64_t n_out = n_all < k ? n_all : k;
  if (n_out > T) n_out = T;
  for (int64_t r = 0; r < n_out; r++) {
    out_t[r] = all[r].t;
    out_s64[r] = all[r].s;
  }
  /* tables of the kept triplets, by the per-triplet oracle */
  if (out_ft) {
    for (int64_t r = 0; r < n_out; r++) {
      int64_t t = out_t[r], i = 0, j, kk;
      /* invert the lexicographic index */
      while (oracle_triplet_index(M, i + 1, i + 2, i + 3) <= t && i + 1 < M - 2) i++;
      j = i + 1;
      while (j + 1 < M - 1 && oracle_triplet_index(M, i, j + 1, j + 2) <= t) j++;
      kk = j + 1 + (t - oracle_triplet_index(M, i, j, j + 1));
      oracle_table(planes[0], planes[1], n0, n1, i, j, kk, out_ft + 54 * r);
    }
  }
  free(all);
  free(heap_n);
  free(heaps);
  free(g64[0]);
  free(g64[1]);
  free(planes[0]);
  free(planes[1]);
  return n_out;
}
