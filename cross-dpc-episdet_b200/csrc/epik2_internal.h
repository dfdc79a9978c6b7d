// Internal declarations shared by the host API and the CUDA kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace epik2 {

constexpr int kWarp = 32;
constexpr int kPairsPerWarp = 4;      // (i, j0..j0+3) pair group handled by one warp
constexpr int kScanThreads = 256;     // 8 warps per CTA
constexpr int kTableMaxSize = 748;    // reference TABLE_MAX_SIZE (GPU/v4.cpp:15)

// Device-resident dataset.  Planes are word-major: for each 32-sample class word w
// (controls' words first, then cases'), one uint2 {g0 bits, g1 bits} per SNP, rows of
// m_pad SNPs.  Bit b of class word w is the sample of rank 32*w' + b in its class
// (w' = word index inside the class); padding bits and padding SNPs are zero.
struct DevDataset {
  int64_t n_samples = 0, n_snps = 0, n_cases = 0, n_controls = 0;
  int64_t m_pad = 0;      // n_snps rounded up to 32
  int64_t w0 = 0, w1 = 0; // words per class
  uint8_t* geno = nullptr;      // [n_samples][n_snps], kept for phenotype re-encoding
  int32_t* perm = nullptr;      // class-sorted sample order: controls then cases
  uint2* planes = nullptr;      // [w0+w1][m_pad]
  uint32_t* singles = nullptr;  // [2][m_pad][2] counts of g0, g1 per class
  uint4* pairs = nullptr;       // [2][tri(m_pad)] counts (00,01,10,11) for x<y
  float* lut = nullptr;         // ln n! in the reference CPU arithmetic, [0, n_samples+1]
  double* lut64 = nullptr;      // ln n! in double (precision form), [0, n_samples+1]
  int64_t tri = 0;              // entries per class in `pairs`
  void* block = nullptr;        // single allocation holding all of the above
  size_t bytes = 0;             // bytes the layout needs
  size_t block_bytes = 0;       // size of `block` (at least `bytes`)
  int32_t base_id = -1;         // replicate: dataset whose genotype matrix this one shares
  int32_t n_replicates = 0;     // live replicates sharing this dataset's genotypes
};

// Offset of pair (x, y), x < y, in a row-major strict upper triangle of an m x m matrix.
__host__ __device__ inline int64_t tri_offset(int64_t m, int64_t x, int64_t y) {
  return x * (m - 1) - (x * (x - 1)) / 2 + (y - x - 1);
}
__host__ __device__ inline int64_t tri_size(int64_t m) { return m * (m - 1) / 2; }

// Best-candidate record: score (positive float) + packed lexicographic key.
struct BestSlot {
  float score;
  uint32_t pad;
  unsigned long long key;  // (i << 42) | (j << 21) | k
};

__host__ __device__ inline unsigned long long pack_key(uint64_t i, uint64_t j, uint64_t k) {
  return (i << 42) | (j << 21) | k;
}

// FP64 rescore of one candidate.
struct Rescored {
  double s64;
  float s32;
  uint32_t pad;
  unsigned long long key;
};

struct ScanParams {
  const uint2* planes;
  const uint32_t* singles;
  const uint4* pairs;
  const float* lut;
  const int64_t* pg_off;   // prefix sums of pair groups per first index, [n_first + 1]
  int64_t n_groups;
  int64_t tri;
  int32_t n_first;         // number of first indices covered
  int32_t i_begin;
  int32_t m, m_pad, w0, w1, n0, n1;
  unsigned long long* counter;
  BestSlot* slots;         // one per warp in the grid
  int32_t top_k;           // >1: per-warp candidate lists of this many entries
  BestSlot* cand;          // [warps][top_k] when top_k > 1
  uint32_t* dump_tables;   // [C(m,3)][54] or null
  float* dump_scores;      // [C(m,3)] or null
};

// One dataset of a batched tensor-core search (device-resident job table).
struct TcJob {
  const uint2* planes;
  const uint32_t* singles;
  const uint4* pairs;
  const float* lut;
  const double* lut64;
  int64_t tri;
  int32_t m, m_pad, w0, w1, n0, n1;
};

// Tensor-core tile descriptor: first index i (bits 0-19), first SNP j0 of the pair block
// (bits 20-39), k block t of the pair block (bits 40-53: k in [k0, k0 + kK) with
// k0 = j0 + 1 + kK*t, so the blocks of a pair block start at its first valid k), batched job
// (bits 54-62).
__host__ __device__ inline uint64_t pack_tile(uint32_t i, uint32_t j0, uint32_t kb, uint32_t job) {
  return (uint64_t)i | ((uint64_t)j0 << 20) | ((uint64_t)kb << 40) | ((uint64_t)job << 54);
}
__host__ __device__ inline int tile_i(uint64_t d) { return (int)(d & 0xFFFFF); }
__host__ __device__ inline int tile_j0(uint64_t d) { return (int)((d >> 20) & 0xFFFFF); }
__host__ __device__ inline int tile_kb(uint64_t d) { return (int)((d >> 40) & 0x3FFF); }
__host__ __device__ inline int tile_job(uint64_t d) { return (int)((d >> 54) & 0x1FF); }
constexpr int kMaxBatchJobs = 512;  // datasets per batched launch (9 descriptor bits)
// First SNP k of tile descriptor d (kK SNPs k per tile).
__host__ __device__ inline int tile_k0(uint64_t d, int kK) { return tile_j0(d) + 1 + kK * tile_kb(d); }
// Tiles of the pair block starting at SNP j0 whose k run over [j0 + 1, k_end).
__host__ __device__ inline int64_t tiles_of_pair_block(int64_t j0, int64_t k_end, int64_t kK) {
  return k_end > j0 + 1 ? (k_end - j0 - 1 + kK - 1) / kK : 0;
}

// Tensor-core engine parameters (scan_tc.cu).  Tiles: for each pair block (i, j0..j0+31,
// or j0..j0+63 on CTA pairs) the k blocks [j0+1+kK*t, j0+1+kK*(t+1)) covering k < m (kK =
// 128 int8, 112 FP4), one descriptor (pack_tile) per tile, taken in order from a shared
// counter.
struct TcParams {
  const uint2* planes;
  const uint32_t* singles;
  const uint4* pairs;
  const float* lut;
  const uint64_t* tiles;   // [n_tiles] descriptors
  int64_t n_tiles;
  int64_t tri;
  int32_t m, m_pad, w0, w1, n0, n1;
  unsigned long long* counter;
  BestSlot* slots;         // one per warp in the grid
  int32_t top_k;
  BestSlot* cand;          // [warps][32] when top_k > 1
  uint32_t* dump_tables;
  float* dump_scores;
  int* err;                // set to 1 if a bounded wait expired
  // batched form (jobs != null): each tile's descriptor names its job
  const TcJob* jobs;
  int32_t n_jobs;
  BestSlot* job_slots;     // [n_jobs][grid]
  // pair-margin form (pairs_out != null): tiles (0, j0, k block) write the (j, k) pair
  // counts of both classes instead of scoring triplets
  uint4* pairs_out;
  // SM clocks a bounded mbarrier wait lasts before the kernel gives up (0 = about 2 s)
  long long wait_limit;
  // test hook: CTA 0 withholds one arrival so that its first wait expires (single CTAs)
  int32_t test_withhold;
  // replicate form (launch_scan_reps): jobs = the n_reps replicates of the base dataset
  // (p.planes ... p.n1), job_slots = [n_reps][grid] per-replicate results
  int32_t n_reps;
};

// Kernel launchers (scan_int.cu / scan_tc.cu / encode.cu); all asynchronous on `stream`.
cudaError_t launch_encode(const DevDataset& d, cudaStream_t stream);
cudaError_t launch_counts(const DevDataset& d, cudaStream_t stream, bool pairs = true);
// pair margins on tensor cores (the CTA-pair FP4 kernel; exact for classes below 2^24)
cudaError_t launch_pairs_tc(const TcParams& p, int blocks, cudaStream_t stream);
// replicate form of the CTA-pair FP4 search (16 words per stage): see TcParams::n_reps
cudaError_t launch_scan_reps(const TcParams& p, int blocks, cudaStream_t stream);
cudaError_t launch_scan_int(const ScanParams& p, int blocks, bool dump, cudaStream_t stream);
cudaError_t launch_reduce_best(const BestSlot* slots, int n, BestSlot* out, cudaStream_t stream);
cudaError_t launch_tables(const DevDataset& d, const uint32_t* triplets, int64_t n, uint32_t* out,
                          cudaStream_t stream);
cudaError_t launch_rescore(const DevDataset& d, const BestSlot* cand, int64_t n, Rescored* out, cudaStream_t stream);
int scan_blocks_per_sm();
// pair: FP4 on CTA pairs (clusters of two CTAs, tiles of 64 SNPs j); else one CTA per tile
// of 32 SNPs j
cudaError_t launch_scan_tc(const TcParams& p, int blocks, int words_per_stage, bool fp4, bool pair, bool dump,
                           cudaStream_t stream);
int tc_k_per_tile(bool fp4);  // SNPs k per tensor-core tile: 128 (int8) or 112 (FP4)
// The overlapped FP4 CTA-pair kernel (scan_pipe.cu): scoring of a tile runs while the next
// tile counts; 4 or 8 words per stage; classes of at most 65535 samples (16-bit staging).
cudaError_t launch_scan_pipe(const TcParams& p, int blocks, int words_per_stage, bool dump, cudaStream_t stream);
bool pipe_fits(int64_t n_controls, int64_t n_cases);
cudaError_t pipe_configure();  // dynamic shared-memory limits of the overlapped kernels (once)
int tc_pair_blocks(int sms);  // resident CTAs of the CTA-pair kernel (even)
// Tile descriptors of one pair-block list (prefix sums pb_off[0..n_pb], (i, j0) pairs) into
// out[pb_off[b] ...], tagged with `job`.
cudaError_t launch_expand_tiles(const int64_t* pb_off, const uint32_t* pb_ij, int64_t n_pb, bool fp4, int job,
                                uint64_t* out, cudaStream_t stream);
cudaError_t launch_reduce_jobs(const BestSlot* slots, int n_jobs, int per_job, BestSlot* out, cudaStream_t stream);
cudaError_t launch_fill_slots(BestSlot* slots, int64_t n, cudaStream_t stream);
cudaError_t tc_configure();
cudaError_t launch_rescore_jobs(const TcJob* jobs, const BestSlot* best, int n, Rescored* out, cudaStream_t stream);  // dynamic shared memory limits of the tensor-core kernels (once)
int tc_warps_per_block();

// Host helpers (host_data.cpp).
void build_k2_lut(int64_t n_max, float* lut);
void build_k2_lut_range(int64_t n_begin, int64_t n_end, float* out);  // out[n - n_begin], n in [begin, end)
void build_k2_lut64(int64_t n_max, double* lut);
void generate_reference(int64_t n, int64_t m, uint8_t* geno, uint8_t* pheno);
void generate_hwe(uint64_t seed, int64_t n, int64_t m, int64_t n_cases, double maf_lo, double maf_hi,
                  int n_planted, const int64_t* planted, const double* effects, uint8_t* geno, uint8_t* pheno);

}  // namespace epik2
