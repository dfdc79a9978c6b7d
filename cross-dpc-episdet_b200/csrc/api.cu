// C ABI (include/epik2.h): contexts, resident datasets, the plain search and the
// parity/inspection entry points.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/epik2.h"
#include "epik2_internal.h"

using namespace epik2;

struct epik2_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;      // current stream (own or caller's)
  cudaStream_t own_stream = nullptr;
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  cudaEvent_t ev_load[3] = {nullptr, nullptr, nullptr};  // load: before upload, after upload, prepared
  // host ln n! tables of the last sample count loaded (a matrix of the same shape reuses them)
  int64_t lut_samples = -1;
  std::vector<float> lut_host;
  std::vector<double> lut64_host;
  epik2_stats stats{};
  cudaDeviceProp prop{};
  std::string last_error;
  std::map<int32_t, std::unique_ptr<DevDataset>> datasets;
  int32_t next_id = 1;
  // one dataset allocation kept by the one-call entry point (epik2_scan_u8) for its next
  // call: allocating and freeing a few hundred MiB per call costs tens to hundreds of ms
  void* spare_block = nullptr;
  size_t spare_bytes = 0;
  // search scratch
  int engine = 0;               // default engine: 0 = auto, 1 = integer, 2 = tensor cores int8, 3 = tensor cores FP4
  int stage_words = 0;          // default tensor-core stage depth: 0 = autotuned
  int pair_tile = 0;            // default tensor-core pair tile: 0 = autotuned, 32 or 64
  int overlap = 0;              // default overlapped-kernel choice: 0 = tuned, 1 = off, 2 = on
  int scan_blocks = 0;          // integer engine grid
  int tc_blocks = 0;            // tensor-core engine grid (one CTA per SM)
  int n_slots = 0;              // per-warp slots, enough for either grid
  int* d_err = nullptr;
  int64_t wait_limit = 0;       // SM clocks of a bounded device-side wait (0 = kernel default)
  int test_withhold = 0;        // one-shot test hook of the bounded-wait error path
  int64_t* d_pb_off = nullptr;
  uint32_t* d_pb_ij = nullptr;
  int64_t pb_cap = 0;
  uint64_t* d_tiles = nullptr;  // tensor-core tile descriptors
  int64_t tiles_cap = 0;
  unsigned long long* d_counter = nullptr;
  BestSlot* d_slots = nullptr;  // one per warp of the scan grid
  BestSlot* d_best = nullptr;
  BestSlot* d_cand = nullptr;   // 32 per warp (top-k form)
  Rescored* d_resc = nullptr;   // FP64 rescore of every candidate
  int64_t* d_pgoff = nullptr;
  int64_t pgoff_cap = 0;
  BestSlot* h_best = nullptr;   // pinned
  // last top-k result
  std::vector<epik2_best> last_topk;
  // autotuner choices per (log2 samples, log2 SNPs)
  std::map<std::pair<int, int>, epik2_tune> tune_cache;
  // batched-form plans, keyed by the SNP count of every job (a plan holds no dataset
  // pointer: the job table is rewritten before every replay), least recently used first
  std::map<std::vector<int64_t>, std::unique_ptr<struct BatchPlan>> plans;
  std::vector<std::vector<int64_t>> plan_lru;
  // replicate form scratch: job table, per-CTA slots, results (grown, never shrunk)
  TcJob* d_rep_jobs = nullptr;
  BestSlot* d_rep_slots = nullptr;
  BestSlot* d_rep_res = nullptr;
  Rescored* d_rep_resc = nullptr;
  int64_t rep_cap = 0, rep_slot_cap = 0;
};

constexpr size_t kMaxPlans = 32;  // cached batched plans per context

struct BatchPlan {
  int64_t n_tiles = 0;
  std::vector<int> group_code;           // tc_code() of each launch group
  std::vector<int64_t> group_off;        // tiles of group g: [group_off[g], group_off[g+1])
  unsigned long long* d_counters = nullptr;  // one tile counter per group
  int32_t n_jobs = 0;
  epik2::TcJob* d_jobs = nullptr;
  uint64_t* d_tiles = nullptr;           // descriptors of every job's tiles, job after job
  int64_t* d_pb_off = nullptr;
  uint32_t* d_pb_ij = nullptr;
  epik2::BestSlot* d_job_slots = nullptr;
  epik2::BestSlot* d_results = nullptr;
  epik2::BestSlot* h_results = nullptr;  // pinned
  epik2::Rescored* d_resc = nullptr;     // FP64 rescore of each dataset's best
  epik2::Rescored* h_resc = nullptr;     // pinned
  int* h_err = nullptr;                  // pinned
  std::vector<epik2::TcJob> h_jobs;
  bool rescore = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~BatchPlan() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaFree(d_jobs);
    cudaFree(d_tiles);
    cudaFree(d_counters);
    cudaFree(d_pb_off);
    cudaFree(d_pb_ij);
    cudaFree(d_job_slots);
    cudaFree(d_results);
    cudaFreeHost(h_results);
    cudaFreeHost(h_err);
    cudaFree(d_resc);
    cudaFreeHost(h_resc);
  }
};

namespace {

int fail(epik2_ctx* ctx, int status, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return status;
}

int cuda_fail(epik2_ctx* ctx, cudaError_t e, const char* what) {
  std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return fail(ctx, EPIK2_E_NOMEM, msg);
  return fail(ctx, EPIK2_E_CUDA, msg);
}

#define CK(ctx, call, what)                                  \
  do {                                                       \
    cudaError_t _e = (call);                                 \
    if (_e != cudaSuccess) return cuda_fail(ctx, _e, what);  \
  } while (0)

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

void drop_spare(epik2_ctx* ctx) {
  if (ctx->spare_block) cudaFree(ctx->spare_block);
  ctx->spare_block = nullptr;
  ctx->spare_bytes = 0;
}

// A dataset allocation of at least `bytes`: the context's spare block when it fits without
// more than doubling the footprint, else a new one (the spare is released first).
cudaError_t take_block(epik2_ctx* ctx, size_t bytes, void** out, size_t* got) {
  if (ctx->spare_block && ctx->spare_bytes >= bytes && ctx->spare_bytes <= 2 * bytes) {
    *out = ctx->spare_block;
    *got = ctx->spare_bytes;
    ctx->spare_block = nullptr;
    ctx->spare_bytes = 0;
    return cudaSuccess;
  }
  drop_spare(ctx);
  *got = bytes;
  return cudaMalloc(out, bytes);
}

struct Layout {
  size_t geno, perm, planes, singles, pairs, lut, lut64, total;
};

Layout dataset_layout(int64_t s, int64_t m, bool with_geno = true) {
  const int64_t m_pad = (m + 31) / 32 * 32;
  const int64_t words = (s + 31) / 32 + 1;  // enough for any class split
  Layout L{};
  size_t off = 0;
  L.geno = off;
  off = align_up(off + (with_geno ? (size_t)(s * m) : 0), 256);
  L.perm = off;
  off = align_up(off + (size_t)s * 4, 256);
  L.planes = off;
  off = align_up(off + (size_t)(words * m_pad) * 8, 256);
  L.singles = off;
  off = align_up(off + (size_t)m_pad * 16, 256);
  L.pairs = off;
  off = align_up(off + (size_t)(2 * tri_size(m_pad)) * 16, 256);
  L.lut = off;
  off = align_up(off + (size_t)(s + 2) * 4, 256);
  L.lut64 = off;
  off = align_up(off + (size_t)(s + 2) * 8, 256);
  L.total = off;
  return L;
}

// Class-sorted sample order (controls, then cases) and the case count.
int64_t make_perm(const uint8_t* pheno, int64_t s, std::vector<int32_t>& perm) {
  perm.resize((size_t)s);
  int64_t n1 = 0;
  for (int64_t t = 0; t < s; t++) n1 += (pheno[t] == 1);
  int64_t c0 = 0, c1 = s - n1;
  for (int64_t t = 0; t < s; t++) {
    if (pheno[t] == 1) perm[(size_t)c1++] = (int32_t)t;
    else perm[(size_t)c0++] = (int32_t)t;
  }
  return n1;
}

int run_pairs_tc(epik2_ctx* ctx, DevDataset& d);
bool fp4_exact(const DevDataset& d);

int encode_with(epik2_ctx* ctx, DevDataset& d, const uint8_t* pheno) {
  std::vector<int32_t> perm;
  d.n_cases = make_perm(pheno, d.n_samples, perm);
  d.n_controls = d.n_samples - d.n_cases;
  d.w0 = (d.n_controls + 31) / 32;
  d.w1 = (d.n_cases + 31) / 32;
  CK(ctx, cudaMemcpyAsync(d.perm, perm.data(), perm.size() * 4, cudaMemcpyHostToDevice, ctx->stream), "upload perm");
  ctx->stats.h2d_bytes += perm.size() * 4;
  CK(ctx, launch_encode(d, ctx->stream), "encode kernel");
  // pair margins on tensor cores when FP4 counts are exact (classes below 2^24 samples),
  // else on the integer pipe
  const bool tc_pairs = fp4_exact(d) && d.m_pad >= 2;
  CK(ctx, launch_counts(d, ctx->stream, !tc_pairs), "count kernels");
  ctx->stats.kernel_launches += tc_pairs ? 2 : 3;
  if (tc_pairs) return run_pairs_tc(ctx, d);
  CK(ctx, cudaStreamSynchronize(ctx->stream), "encode");
  return EPIK2_OK;
}

DevDataset* find(epik2_ctx* ctx, int32_t id) {
  auto it = ctx->datasets.find(id);
  return it == ctx->datasets.end() ? nullptr : it->second.get();
}

void decode_key(unsigned long long key, uint32_t& i, uint32_t& j, uint32_t& k) {
  i = (uint32_t)(key >> 42);
  j = (uint32_t)((key >> 21) & ((1ull << 21) - 1));
  k = (uint32_t)(key & ((1ull << 21) - 1));
}

// Scratch buffers grow geometrically: a reallocation (which synchronises the device) happens
// O(log n) times, not whenever a slightly larger search comes.
int ensure_pb(epik2_ctx* ctx, int64_t n) {
  if (n <= ctx->pb_cap) return EPIK2_OK;
  n = std::max(n, 2 * ctx->pb_cap);
  cudaFree(ctx->d_pb_off);
  cudaFree(ctx->d_pb_ij);
  ctx->d_pb_off = nullptr;
  ctx->d_pb_ij = nullptr;
  ctx->pb_cap = 0;
  CK(ctx, cudaMalloc(&ctx->d_pb_off, (size_t)(n + 1) * 8), "alloc tile list");
  CK(ctx, cudaMalloc(&ctx->d_pb_ij, (size_t)n * 8), "alloc tile list");
  ctx->pb_cap = n;
  return EPIK2_OK;
}

int ensure_tiles(epik2_ctx* ctx, int64_t n) {
  if (n <= ctx->tiles_cap) return EPIK2_OK;
  n = std::max(n, 2 * ctx->tiles_cap);
  cudaFree(ctx->d_tiles);
  ctx->d_tiles = nullptr;
  ctx->tiles_cap = 0;
  CK(ctx, cudaMalloc(&ctx->d_tiles, (size_t)n * 8), "alloc tile descriptors");
  ctx->tiles_cap = n;
  return EPIK2_OK;
}

int ensure_pgoff(epik2_ctx* ctx, int64_t n) {
  if (n <= ctx->pgoff_cap) return EPIK2_OK;
  n = std::max(n, 2 * ctx->pgoff_cap);
  if (ctx->d_pgoff) cudaFree(ctx->d_pgoff);
  ctx->d_pgoff = nullptr;
  ctx->pgoff_cap = 0;
  CK(ctx, cudaMalloc(&ctx->d_pgoff, (size_t)n * 8), "alloc pair-group offsets");
  ctx->pgoff_cap = n;
  return EPIK2_OK;
}

int collect_topk(epik2_ctx* ctx, DevDataset& d, const epik2_opts* opts, int top_k, int n_warps);
int run_scan_tc(epik2_ctx* ctx, DevDataset& d, int64_t ib, int64_t ie, int top_k, uint32_t* dump_tables,
                float* dump_scores, BestSlot* best_out, const epik2_opts* opts, int kw, bool fp4, bool pair,
                bool overlap);

// FP4 accumulators are FP32: counts are exact below 2^24 per class.
bool fp4_exact(const DevDataset& d) { return d.n_controls < (1 << 24) && d.n_cases < (1 << 24); }
int tuned(epik2_ctx* ctx, DevDataset& d, epik2_tune* out);

// The tensor-core configurations the autotuner times: format, words per stage, pair tile,
// overlapped kernel.
struct TcConfig {
  int engine, kw;
  bool pair, overlap;
};
constexpr int kNumTcConfigs = 8;
constexpr TcConfig kTcConfigs[kNumTcConfigs] = {
    {EPIK2_ENGINE_TC, 4, false, false},     {EPIK2_ENGINE_TC, 8, false, false},
    {EPIK2_ENGINE_TC_FP4, 8, false, false}, {EPIK2_ENGINE_TC_FP4, 8, true, false},
    {EPIK2_ENGINE_TC_FP4, 16, false, false}, {EPIK2_ENGINE_TC_FP4, 16, true, false},
    {EPIK2_ENGINE_TC_FP4, 4, true, true},   {EPIK2_ENGINE_TC_FP4, 8, true, true}};

// Measured rate of a configuration in a tuner record (0 = not measured).
double tune_rate(const epik2_tune& t, int engine, int kw, bool pair, bool overlap) {
  if (engine == EPIK2_ENGINE_INT) return t.rate_int;
  if (engine == EPIK2_ENGINE_TC) return (pair || overlap) ? 0.0 : (kw == 4 ? t.rate_tc4 : t.rate_tc8);
  if (overlap) return !pair ? 0.0 : (kw == 4 ? t.rate_fp4_4_overlap : kw == 8 ? t.rate_fp4_8_overlap : 0.0);
  if (kw == 8) return pair ? t.rate_fp4_8_pair : t.rate_fp4_8;
  if (kw == 16) return pair ? t.rate_fp4_16 : t.rate_fp4_16_single;
  return 0.0;
}

// A configuration the kernels implement.
bool config_valid(int engine, int kw, bool pair, bool overlap) {
  if (engine == EPIK2_ENGINE_TC) return (kw == 4 || kw == 8) && !pair && !overlap;
  if (engine != EPIK2_ENGINE_TC_FP4) return false;
  if (overlap) return pair && (kw == 4 || kw == 8);
  return kw == 8 || kw == 16;
}

// Whether a dataset can take a configuration.
bool config_fits(const TcConfig& c, bool can_fp4, bool can_overlap) {
  if (c.engine == EPIK2_ENGINE_TC_FP4 && !can_fp4) return false;
  return !c.overlap || can_overlap;
}

// Batched-plan code of a configuration.
int tc_code(int kw, bool fp4, bool pair, bool overlap) {
  return kw * 8 + (overlap ? 4 : 0) + (pair ? 2 : 0) + (fp4 ? 1 : 0);
}

// Fill in the unset parts (0) of a requested configuration: the tuner's choice when it
// matches what was asked, else the fastest measured configuration that does.  ov: 0 =
// either kernel, 1 = sequential, 2 = overlapped.
void complete_config(const epik2_tune& t, bool can_fp4, bool can_overlap, int& engine, int& kw, int& pt, int& ov) {
  if (engine == 0 && kw == 0 && pt == 0 && ov == 0 && (t.engine != EPIK2_ENGINE_TC_FP4 || can_fp4)) {
    engine = t.engine;
    kw = t.stage_words;
    pt = t.pair_tile;
    ov = t.overlap ? 2 : 1;
    return;
  }
  double best = -1.0;
  TcConfig pick{engine ? engine : t.engine, kw, pt == 64, ov == 2};
  for (const TcConfig& c : kTcConfigs) {
    if (engine && c.engine != engine) continue;
    if (kw && c.kw != kw) continue;
    if (pt && c.pair != (pt == 64)) continue;
    if (ov && c.overlap != (ov == 2)) continue;
    if (!config_fits(c, can_fp4, can_overlap)) continue;
    const double r = tune_rate(t, c.engine, c.kw, c.pair, c.overlap);
    if (r > best) {
      best = r;
      pick = c;
    }
  }
  engine = pick.engine;
  kw = pick.kw;
  pt = pick.pair ? 64 : 32;
  ov = pick.overlap ? 2 : 1;
}

int run_scan(epik2_ctx* ctx, DevDataset& d, const epik2_opts* opts, uint32_t* dump_tables, float* dump_scores,
             BestSlot* best_out);

// Pair groups of first index i: j0 = i+1, i+5, ... while j0 <= m-2.
int64_t groups_of(int64_t m, int64_t i) { return (i <= m - 3) ? (m - 2 - i + kPairsPerWarp) / kPairsPerWarp : 0; }

int run_scan(epik2_ctx* ctx, DevDataset& d, const epik2_opts* opts, uint32_t* dump_tables, float* dump_scores,
             BestSlot* best_out) {
  const int64_t m = d.n_snps;
  int64_t ib = 0, ie = m;
  int top_k = 0;
  if (opts) {
    if (opts->snp_begin != 0 || opts->snp_end != 0) {
      ib = std::max<int64_t>(0, opts->snp_begin);
      ie = std::min<int64_t>(m, opts->snp_end);
    }
    if (opts->top_k < 0 || opts->top_k > 32) return fail(ctx, EPIK2_E_INVALID, "top_k must be in [0, 32]");
    top_k = opts->top_k;
    if (opts->engine < 0 || opts->engine > EPIK2_ENGINE_TC_FP4) return fail(ctx, EPIK2_E_INVALID, "unknown engine");
  }
  if (ie < ib) ie = ib;
  int engine = ctx->engine;
  if (opts && opts->engine != 0) engine = opts->engine;
  int kw = (opts && opts->stage_words) ? opts->stage_words : ctx->stage_words;
  int pt = (opts && opts->pair_tile) ? opts->pair_tile : ctx->pair_tile;
  int ov = (opts && opts->overlap) ? opts->overlap : ctx->overlap;
  if (pt != 0 && pt != 32 && pt != 64) return fail(ctx, EPIK2_E_INVALID, "pair_tile must be 0, 32 or 64");
  if (ov < 0 || ov > 2) return fail(ctx, EPIK2_E_INVALID, "overlap must be 0, 1 or 2");
  if (engine == EPIK2_ENGINE_TC_FP4 && !fp4_exact(d))
    return fail(ctx, EPIK2_E_TOO_LARGE, "FP4 tensor-core engine: a class of 2^24 samples or more");
  const bool can_overlap = fp4_exact(d) && pipe_fits(d.n_controls, d.n_cases);
  if (ov == 2 && !can_overlap)
    return fail(ctx, EPIK2_E_TOO_LARGE, "overlapped kernel: classes of at most 65535 samples");
  if (engine == 0 || ((engine == 2 || engine == 3) && kw == 0)) {
    epik2_tune t{};
    int r = tuned(ctx, d, &t);
    if (r) return r;
    if (engine == 0) {  // a requested option that one format alone takes picks that format
      if (kw == 4 && ov != 2) engine = EPIK2_ENGINE_TC;
      else if (kw == 16 || pt == 64 || ov == 2) engine = fp4_exact(d) ? EPIK2_ENGINE_TC_FP4 : EPIK2_ENGINE_TC;
    }
    complete_config(t, fp4_exact(d), can_overlap, engine, kw, pt, ov);
  }
  if (pt == 0) pt = (engine == EPIK2_ENGINE_TC_FP4 && (kw == 16 || ov == 2)) ? 64 : 32;  // not given: by depth
  if (engine == 2 || engine == 3) {
    if (!config_valid(engine, kw, pt == 64, ov == 2))
      return fail(ctx, EPIK2_E_INVALID,
                  "tensor-core configuration: int8 takes 4 or 8 words per stage on 32-SNP tiles; FP4 takes 8 or 16 "
                  "(32- or 64-SNP tiles), or 4 or 8 overlapped on 64-SNP tiles");
    return run_scan_tc(ctx, d, ib, ie, top_k, dump_tables, dump_scores, best_out, opts, kw, engine == 3, pt == 64,
                       ov == 2);
  }

  const int64_t n_first = std::max<int64_t>(ie - ib, 1);
  std::vector<int64_t> off((size_t)n_first + 1, 0);
  for (int64_t t = 0; t < n_first; t++) off[(size_t)t + 1] = off[(size_t)t] + (ib + t < ie ? groups_of(m, ib + t) : 0);
  int r = ensure_pgoff(ctx, n_first + 1);
  if (r) return r;
  CK(ctx, cudaMemcpyAsync(ctx->d_pgoff, off.data(), off.size() * 8, cudaMemcpyHostToDevice, ctx->stream),
     "upload pair-group offsets");
  ctx->stats.h2d_bytes += off.size() * 8;
  CK(ctx, cudaMemsetAsync(ctx->d_counter, 0, 8, ctx->stream), "reset counter");
  ScanParams p{};
  p.planes = d.planes;
  p.singles = d.singles;
  p.pairs = d.pairs;
  p.lut = d.lut;
  p.pg_off = ctx->d_pgoff;
  p.n_groups = off.back();
  p.tri = d.tri;
  p.n_first = (int32_t)n_first;
  p.i_begin = (int32_t)ib;
  p.m = (int32_t)m;
  p.m_pad = (int32_t)d.m_pad;
  p.w0 = (int32_t)d.w0;
  p.w1 = (int32_t)d.w1;
  p.n0 = (int32_t)d.n_controls;
  p.n1 = (int32_t)d.n_cases;
  p.counter = ctx->d_counter;
  p.slots = ctx->d_slots;
  p.top_k = top_k;
  p.cand = ctx->d_cand;
  p.dump_tables = dump_tables;
  p.dump_scores = dump_scores;
  const bool dump = dump_tables != nullptr;
  CK(ctx, cudaEventRecord(ctx->ev_start, ctx->stream), "event");
  CK(ctx, launch_scan_int(p, ctx->scan_blocks, dump, ctx->stream), "scan kernel");
  CK(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream), "event");
  const int n_warps = ctx->scan_blocks * (kScanThreads / 32);
  CK(ctx, launch_reduce_best(ctx->d_slots, n_warps, ctx->d_best, ctx->stream), "reduce kernel");
  ctx->stats.kernel_launches += 2;
  CK(ctx, cudaMemcpyAsync(ctx->h_best, ctx->d_best, sizeof(BestSlot), cudaMemcpyDeviceToHost, ctx->stream),
     "read result");
  ctx->stats.d2h_bytes += sizeof(BestSlot);
  CK(ctx, cudaStreamSynchronize(ctx->stream), "scan");
  float kms = 0.0f;
  CK(ctx, cudaEventElapsedTime(&kms, ctx->ev_start, ctx->ev_stop), "event time");
  ctx->stats.last_scan_kernel_ms = kms;
  int64_t trip = 0;
  for (int64_t i = ib; i < ie; i++) {
    const int64_t r = m - 1 - i;
    trip += r * (r - 1) / 2;
  }
  ctx->stats.last_scan_triplets = trip;
  ctx->stats.last_scan_words = d.w0 + d.w1;
  *best_out = *ctx->h_best;
  return collect_topk(ctx, d, opts, top_k, n_warps);
}

int collect_topk(epik2_ctx* ctx, DevDataset& d, const epik2_opts* opts, int top_k, int n_warps) {
  const bool rescore = opts && opts->rescore_fp64;
  if (top_k > 1 && rescore) {
    const int64_t nc = (int64_t)n_warps * 32;
    CK(ctx, launch_rescore(d, ctx->d_cand, nc, ctx->d_resc, ctx->stream), "rescore kernel");
    ctx->stats.kernel_launches += 1;
    std::vector<Rescored> res((size_t)nc);
    CK(ctx, cudaMemcpyAsync(res.data(), ctx->d_resc, res.size() * sizeof(Rescored), cudaMemcpyDeviceToHost,
                            ctx->stream),
       "read rescored");
    CK(ctx, cudaStreamSynchronize(ctx->stream), "rescore");
    ctx->stats.d2h_bytes += res.size() * sizeof(Rescored);
    std::sort(res.begin(), res.end(), [](const Rescored& a, const Rescored& b) {
      const bool va = a.key != ~0ull, vb = b.key != ~0ull;
      if (va != vb) return va;
      return a.s64 < b.s64 || (a.s64 == b.s64 && a.key < b.key);
    });
    ctx->last_topk.clear();
    for (const Rescored& c : res) {
      if ((int)ctx->last_topk.size() >= top_k || c.key == ~0ull) break;
      epik2_best e{};
      e.score = c.s32;
      e.score_fp64 = c.s64;
      decode_key(c.key, e.i, e.j, e.k);
      ctx->last_topk.push_back(e);
    }
  } else if (top_k > 1) {
    std::vector<BestSlot> cand((size_t)n_warps * 32);
    CK(ctx, cudaMemcpyAsync(cand.data(), ctx->d_cand, cand.size() * sizeof(BestSlot), cudaMemcpyDeviceToHost,
                            ctx->stream),
       "read candidates");
    CK(ctx, cudaStreamSynchronize(ctx->stream), "read candidates");
    ctx->stats.d2h_bytes += cand.size() * sizeof(BestSlot);
    std::sort(cand.begin(), cand.end(), [](const BestSlot& a, const BestSlot& b) {
      return a.score < b.score || (a.score == b.score && a.key < b.key);
    });
    ctx->last_topk.clear();
    for (const BestSlot& c : cand) {
      if ((int)ctx->last_topk.size() >= top_k || c.key == ~0ull) break;
      epik2_best e{};
      e.score = c.score;
      e.score_fp64 = std::numeric_limits<double>::quiet_NaN();
      decode_key(c.key, e.i, e.j, e.k);
      ctx->last_topk.push_back(e);
    }
  }
  return EPIK2_OK;
}

// Pair margins on tensor cores: the CTA-pair FP4 kernel in its pair-margin form over pair
// blocks (0, j0), j0 = 0, 64, ..., each with the k blocks of 112 SNPs from (j0 + 1) / 112
// on; every (j, k), j < k < m_pad, is written once.  Waits for the result (stream sync).
int run_pairs_tc(epik2_ctx* ctx, DevDataset& d) {
  const int64_t m_pad = d.m_pad, kk = tc_k_per_tile(true);
  std::vector<uint32_t> ij;
  std::vector<int64_t> off(1, 0);
  for (int64_t j0 = 0; j0 <= m_pad - 2; j0 += 64) {
    ij.push_back(0);
    ij.push_back((uint32_t)j0);
    off.push_back(off.back() + tiles_of_pair_block(j0, m_pad, kk));
  }
  const int64_t n_pb = (int64_t)off.size() - 1;
  int r = ensure_pb(ctx, std::max<int64_t>(n_pb, 1));
  if (r) return r;
  r = ensure_tiles(ctx, std::max<int64_t>(off.back(), 1));
  if (r) return r;
  CK(ctx, cudaMemcpyAsync(ctx->d_pb_off, off.data(), off.size() * 8, cudaMemcpyHostToDevice, ctx->stream),
     "upload pair-margin tiles");
  CK(ctx, cudaMemcpyAsync(ctx->d_pb_ij, ij.data(), ij.size() * 4, cudaMemcpyHostToDevice, ctx->stream),
     "upload pair-margin tiles");
  CK(ctx, launch_expand_tiles(ctx->d_pb_off, ctx->d_pb_ij, n_pb, true, 0, ctx->d_tiles, ctx->stream),
     "expand pair-margin tiles");
  CK(ctx, cudaMemsetAsync(ctx->d_counter, 0, 8, ctx->stream), "reset counter");
  CK(ctx, cudaMemsetAsync(ctx->d_err, 0, 4, ctx->stream), "reset error word");
  TcParams p{};
  p.planes = d.planes;
  p.singles = d.singles;
  p.pairs = d.pairs;
  p.lut = d.lut;
  p.tiles = ctx->d_tiles;
  p.n_tiles = off.back();
  p.tri = d.tri;
  p.m = (int32_t)d.n_snps;
  p.m_pad = (int32_t)d.m_pad;
  p.w0 = (int32_t)d.w0;
  p.w1 = (int32_t)d.w1;
  p.n0 = (int32_t)d.n_controls;
  p.n1 = (int32_t)d.n_cases;
  p.counter = ctx->d_counter;
  p.slots = ctx->d_slots;
  p.err = ctx->d_err;
  p.wait_limit = ctx->wait_limit;
  p.pairs_out = d.pairs;
  CK(ctx, launch_pairs_tc(p, tc_pair_blocks(ctx->tc_blocks), ctx->stream), "pair-margin kernel");
  ctx->stats.kernel_launches += 2;
  int err_word = 0;
  CK(ctx, cudaMemcpyAsync(&err_word, ctx->d_err, 4, cudaMemcpyDeviceToHost, ctx->stream), "read error word");
  CK(ctx, cudaStreamSynchronize(ctx->stream), "encode");
  if (err_word) return fail(ctx, EPIK2_E_TIMEOUT, "pair margins: a bounded wait expired");
  return EPIK2_OK;
}

// Tile descriptors of the search of first indices [ib, ie) of an m-SNP dataset into
// ctx->d_tiles (expanded on the GPU from the pair-block list); *n_tiles receives their count.
int prepare_tiles(epik2_ctx* ctx, int64_t m, int64_t ib, int64_t ie, bool fp4, bool pair, int64_t* n_tiles) {
  const int64_t kk = tc_k_per_tile(fp4);
  const int64_t jstep = pair ? 64 : 32;  // SNPs j per tile (a CTA pair takes 64)
  std::vector<uint32_t> ij;
  std::vector<int64_t> off(1, 0);
  // Pair blocks in the order (u, i) with j0 = i + 1 + jstep*u: consecutive pair blocks (and
  // the CTAs working on them at the same time) cover nearly the same SNPs j and k, so the
  // (j, k) pair margins and the k planes they read are shared through L2 instead of being
  // swept from HBM once per first index.
  for (int64_t u = 0; ib + 1 + jstep * u <= m - 2; u++)
    for (int64_t i = ib; i < ie; i++) {
      const int64_t j0 = i + 1 + jstep * u;
      if (j0 > m - 2) break;
      ij.push_back((uint32_t)i);
      ij.push_back((uint32_t)j0);
      off.push_back(off.back() + tiles_of_pair_block(j0, m, kk));
    }
  const int64_t n_pb = (int64_t)off.size() - 1;
  if (n_pb > ctx->pb_cap || off.back() > ctx->tiles_cap) {
    // grow once to the whole search of this dataset, so that its shards never reallocate
    // (a reallocation synchronises the device)
    int64_t all_pb = 0, all_tiles = 0;
    for (int64_t i = 0; i < m; i++)
      for (int64_t j0 = i + 1; j0 <= m - 2; j0 += jstep) {
        all_pb++;
        all_tiles += tiles_of_pair_block(j0, m, kk);
      }
    int r0 = ensure_pb(ctx, std::max<int64_t>(all_pb, 1));
    if (r0) return r0;
    r0 = ensure_tiles(ctx, std::max<int64_t>(all_tiles, 1));
    if (r0) return r0;
  }
  int r = ensure_pb(ctx, std::max<int64_t>(n_pb, 1));
  if (r) return r;
  r = ensure_tiles(ctx, std::max<int64_t>(off.back(), 1));
  if (r) return r;
  if (n_pb > 0) {
    CK(ctx, cudaMemcpyAsync(ctx->d_pb_off, off.data(), off.size() * 8, cudaMemcpyHostToDevice, ctx->stream),
       "upload tile list");
    CK(ctx, cudaMemcpyAsync(ctx->d_pb_ij, ij.data(), ij.size() * 4, cudaMemcpyHostToDevice, ctx->stream),
       "upload tile list");
    ctx->stats.h2d_bytes += off.size() * 8 + ij.size() * 4;
    CK(ctx, launch_expand_tiles(ctx->d_pb_off, ctx->d_pb_ij, n_pb, fp4, 0, ctx->d_tiles, ctx->stream),
       "tile descriptors");
    ctx->stats.kernel_launches += 1;
  }
  *n_tiles = off.back();
  return EPIK2_OK;
}

// Tensor-core engine: one CTA per SM, tiles = pair blocks (i, j0..j0+31) x k blocks of
// 128 (int8 format) or 112 (FP4 format) SNPs.
int run_scan_tc(epik2_ctx* ctx, DevDataset& d, int64_t ib, int64_t ie, int top_k, uint32_t* dump_tables,
                float* dump_scores, BestSlot* best_out, const epik2_opts* opts, int kw, bool fp4, bool pair,
                bool overlap) {
  const int64_t m = d.n_snps;
  pair = pair && fp4;
  overlap = overlap && pair;
  const int grid = pair ? tc_pair_blocks(ctx->tc_blocks) : ctx->tc_blocks;
  int64_t n_tiles = 0;
  int r = prepare_tiles(ctx, m, ib, ie, fp4, pair, &n_tiles);
  if (r) return r;
  CK(ctx, cudaMemsetAsync(ctx->d_counter, 0, 8, ctx->stream), "reset counter");
  CK(ctx, cudaMemsetAsync(ctx->d_err, 0, 4, ctx->stream), "reset error word");
  TcParams p{};
  p.planes = d.planes;
  p.singles = d.singles;
  p.pairs = d.pairs;
  p.lut = d.lut;
  p.tiles = ctx->d_tiles;
  p.n_tiles = n_tiles;
  p.tri = d.tri;
  p.m = (int32_t)m;
  p.m_pad = (int32_t)d.m_pad;
  p.w0 = (int32_t)d.w0;
  p.w1 = (int32_t)d.w1;
  p.n0 = (int32_t)d.n_controls;
  p.n1 = (int32_t)d.n_cases;
  p.counter = ctx->d_counter;
  p.slots = ctx->d_slots;
  p.top_k = top_k;
  p.cand = ctx->d_cand;
  p.dump_tables = dump_tables;
  p.dump_scores = dump_scores;
  p.err = ctx->d_err;
  p.wait_limit = ctx->wait_limit;
  p.test_withhold = pair ? 0 : ctx->test_withhold;
  if (!pair) ctx->test_withhold = 0;
  CK(ctx, cudaEventRecord(ctx->ev_start, ctx->stream), "event");
  if (overlap)
    CK(ctx, launch_scan_pipe(p, grid, kw, dump_tables != nullptr, ctx->stream), "overlapped tensor-core kernel");
  else
    CK(ctx, launch_scan_tc(p, grid, kw, fp4, pair, dump_tables != nullptr, ctx->stream), "tensor-core scan kernel");
  CK(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream), "event");
  const int n_warps = grid * tc_warps_per_block();
  CK(ctx, launch_reduce_best(ctx->d_slots, n_warps, ctx->d_best, ctx->stream), "reduce kernel");
  ctx->stats.kernel_launches += 2;
  CK(ctx, cudaMemcpyAsync(ctx->h_best, ctx->d_best, sizeof(BestSlot), cudaMemcpyDeviceToHost, ctx->stream),
     "read result");
  int err_word = 0;
  CK(ctx, cudaMemcpyAsync(&err_word, ctx->d_err, 4, cudaMemcpyDeviceToHost, ctx->stream), "read error word");
  ctx->stats.d2h_bytes += sizeof(BestSlot) + 4;
  CK(ctx, cudaStreamSynchronize(ctx->stream), "scan");
  if (err_word) return fail(ctx, EPIK2_E_TIMEOUT, "tensor-core scan: a bounded wait expired");
  float kms = 0.0f;
  CK(ctx, cudaEventElapsedTime(&kms, ctx->ev_start, ctx->ev_stop), "event time");
  ctx->stats.last_scan_kernel_ms = kms;
  int64_t trip = 0;
  for (int64_t i = ib; i < ie; i++) {
    const int64_t rr = m - 1 - i;
    trip += rr * (rr - 1) / 2;
  }
  ctx->stats.last_scan_triplets = trip;
  ctx->stats.last_scan_words = d.w0 + d.w1;
  *best_out = *ctx->h_best;
  return collect_topk(ctx, d, opts, top_k, n_warps);
}

// Triplets with first index in [0, ie).
int64_t triplets_before(int64_t m, int64_t ie) {
  int64_t t = 0;
  for (int64_t i = 0; i < ie; i++) t += (m - 1 - i) * (m - 2 - i) / 2;
  return t;
}

// Autotuner: time each candidate on a slice of the dataset (first indices [0, ie) holding
// about 1/64 of the triplets, grown until the tensor-core engine has >= 4 tiles per SM)
// and keep the fastest per shape bucket.  Each candidate runs twice; the second run is
// timed (the first absorbs first-launch costs).
int autotune_now(epik2_ctx* ctx, DevDataset& d, epik2_tune* out) {
  const int64_t m = d.n_snps, total = triplets_before(m, m);
  int64_t ie = 1;
  while (ie < m && (triplets_before(m, ie) * 64 < total || triplets_before(m, ie) < 4ll * ctx->tc_blocks * 4096)) ie++;
  const double ts = (double)triplets_before(m, ie) * (double)d.n_samples;
  // candidates: integer; int8 tensor cores, 4 or 8 words per stage (pair tile 32); FP4 tensor
  // cores, 8 or 16 words per stage, pair tile 32 (one CTA) or 64 (CTA pairs); the overlapped
  // FP4 CTA-pair kernel at 4 and 8 words per stage
  constexpr int kCand = 1 + kNumTcConfigs;
  double rate[kCand] = {};
  const bool can_fp4 = fp4_exact(d), can_overlap = can_fp4 && pipe_fits(d.n_controls, d.n_cases);
  for (int c = 0; c < kCand; c++) {
    epik2_opts o{};
    if (c == 0) {
      o.engine = EPIK2_ENGINE_INT;
    } else {
      const TcConfig& tc = kTcConfigs[c - 1];
      if (!config_fits(tc, can_fp4, can_overlap)) continue;
      o.engine = tc.engine;
      o.stage_words = tc.kw;
      o.pair_tile = tc.pair ? 64 : 32;
      o.overlap = tc.overlap ? 2 : 1;
    }
    o.snp_begin = 0;
    o.snp_end = ie;
    BestSlot b{};
    for (int rep = 0; rep < 2; rep++) {
      int r = run_scan(ctx, d, &o, nullptr, nullptr, &b);
      if (r) return r;
    }
    rate[c] = ts / (ctx->stats.last_scan_kernel_ms * 1e-3);
  }
  epik2_tune t{};
  t.rate_int = rate[0];
  t.rate_tc4 = rate[1];
  t.rate_tc8 = rate[2];
  t.rate_fp4_8 = rate[3];
  t.rate_fp4_8_pair = rate[4];
  t.rate_fp4_16_single = rate[5];
  t.rate_fp4_16 = rate[6];
  t.rate_fp4_4_overlap = rate[7];
  t.rate_fp4_8_overlap = rate[8];
  int best = 0;
  for (int c = 1; c < kCand; c++)
    if (rate[c] > rate[best]) best = c;
  if (best == 0) {  // the integer engine; the stage depth is the faster int8 one
    t.engine = EPIK2_ENGINE_INT;
    t.stage_words = rate[2] > rate[1] ? 8 : 4;
    t.pair_tile = 32;
    t.overlap = 0;
  } else {
    t.engine = kTcConfigs[best - 1].engine;
    t.stage_words = kTcConfigs[best - 1].kw;
    t.pair_tile = kTcConfigs[best - 1].pair ? 64 : 32;
    t.overlap = kTcConfigs[best - 1].overlap ? 1 : 0;
  }
  *out = t;
  return EPIK2_OK;
}

std::pair<int, int> shape_bucket(const DevDataset& d) {
  int sb = 0, mb = 0;
  while ((2ll << sb) <= d.n_samples) sb++;
  while ((2ll << mb) <= d.n_snps) mb++;
  return {sb, mb};
}

int tuned(epik2_ctx* ctx, DevDataset& d, epik2_tune* out) {
  const auto key = shape_bucket(d);
  auto it = ctx->tune_cache.find(key);
  if (it != ctx->tune_cache.end()) {
    *out = it->second;
    return EPIK2_OK;
  }
  int r = autotune_now(ctx, d, out);
  if (r) return r;
  ctx->tune_cache[key] = *out;
  return EPIK2_OK;
}

// Batched form: build (or reuse) the plan for these datasets, refresh the job table from
// the datasets' current class split, replay the captured launch sequence.  codes[b] =
// tc_code() of dataset b's configuration; datasets with the same code form a group, one
// persistent tensor-core launch per group (inside the one graph), each group with its own
// tile queue (datasets with the most samples first).  epik2_scan_batch gives every dataset
// the same code: one group, one launch.
int run_batch(epik2_ctx* ctx, const std::vector<DevDataset*>& ds, const std::vector<int32_t>& ids,
              const std::vector<int>& codes, bool rescore, epik2_best* out) {
  (void)ids;
  std::vector<int64_t> key;
  for (const DevDataset* d : ds) key.push_back(d->n_snps);
  for (int c : codes) key.push_back(c);
  key.push_back(rescore ? 1 : 0);
  BatchPlan* plan = nullptr;
  auto it = ctx->plans.find(key);
  const int32_t n = (int32_t)ds.size();
  const int grid = ctx->tc_blocks;
  auto touch = [&](const std::vector<int64_t>& k) {
    auto pos = std::find(ctx->plan_lru.begin(), ctx->plan_lru.end(), k);
    if (pos != ctx->plan_lru.end()) ctx->plan_lru.erase(pos);
    ctx->plan_lru.push_back(k);
  };
  if (it != ctx->plans.end()) {
    plan = it->second.get();
    touch(key);
  } else {
    if (ctx->plans.size() >= kMaxPlans && !ctx->plan_lru.empty()) {  // drop the least recently used
      CK(ctx, cudaStreamSynchronize(ctx->stream), "plan eviction");
      ctx->plans.erase(ctx->plan_lru.front());
      ctx->plan_lru.erase(ctx->plan_lru.begin());
    }
    std::unique_ptr<BatchPlan> pl(new BatchPlan());
    pl->n_jobs = n;
    pl->rescore = rescore;
    // groups in order of first appearance
    std::vector<int> group_code;
    std::vector<int> group_of(n);
    for (int32_t b = 0; b < n; b++) {
      auto g = std::find(group_code.begin(), group_code.end(), codes[b]);
      if (g == group_code.end()) {
        group_code.push_back(codes[b]);
        g = group_code.end() - 1;
      }
      group_of[b] = (int)(g - group_code.begin());
    }
    const int n_groups = (int)group_code.size();
    // pair-block lists depend on the SNP count and the k-block size: one list per pair
    std::vector<int64_t> pb_off_all;
    std::vector<uint32_t> pb_ij_all;
    std::vector<int64_t> job_pb_base(n), job_ij_base(n), job_n_pb(n), job_tiles(n);
    struct ListInfo {
      int64_t off_base, ij_base, n_pb, tiles;
    };
    std::map<std::pair<int64_t, int64_t>, ListInfo> lists;
    for (int32_t b = 0; b < n; b++) {
      const bool fp4 = codes[b] & 1;
      const int64_t m = ds[b]->n_snps, kk = tc_k_per_tile(fp4);
      const int64_t jstep = (codes[b] & 2) ? 64 : 32;  // CTA pairs (both kernels)
      auto li = lists.find({m, kk * 2 + (jstep == 64 ? 1 : 0)});
      if (li == lists.end()) {
        ListInfo L{(int64_t)pb_off_all.size(), (int64_t)pb_ij_all.size(), 0, 0};
        pb_off_all.push_back(0);
        for (int64_t u = 0; 1 + jstep * u <= m - 2; u++)  // (u, i) order, as in run_scan_tc
          for (int64_t i = 0; i < m; i++) {
            const int64_t j0 = i + 1 + jstep * u;
            if (j0 > m - 2) break;
            pb_ij_all.push_back((uint32_t)i);
            pb_ij_all.push_back((uint32_t)j0);
            L.tiles += tiles_of_pair_block(j0, m, kk);
            pb_off_all.push_back(L.tiles);
            L.n_pb++;
          }
        li = lists.emplace(std::make_pair(m, kk * 2 + (jstep == 64 ? 1 : 0)), L).first;
      }
      job_pb_base[b] = li->second.off_base;
      job_ij_base[b] = li->second.ij_base;
      job_n_pb[b] = li->second.n_pb;
      job_tiles[b] = li->second.tiles;
      pl->h_jobs.push_back(TcJob{});
    }
    // tile queue: group after group; inside a group, datasets with the most samples first
    // (their tiles are the longest), so the short tiles fill the end of each launch
    std::vector<int32_t> order(n);
    for (int32_t b = 0; b < n; b++) order[b] = b;
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
      if (group_of[a] != group_of[b]) return group_of[a] < group_of[b];
      return ds[a]->n_samples > ds[b]->n_samples;
    });
    std::vector<int64_t> job_off(n, 0);
    pl->group_off.assign(n_groups + 1, 0);
    pl->n_tiles = 0;
    for (int32_t b : order) {
      job_off[b] = pl->n_tiles;
      pl->n_tiles += job_tiles[b];
      pl->group_off[group_of[b] + 1] = pl->n_tiles;
    }
    for (int g = 1; g <= n_groups; g++) pl->group_off[g] = std::max(pl->group_off[g], pl->group_off[g - 1]);
    pl->group_code = group_code;
    const size_t pb_ij_bytes = std::max<size_t>(pb_ij_all.size(), 2) * 4;
    if (cudaMalloc(&pl->d_jobs, sizeof(TcJob) * n) ||
        cudaMalloc(&pl->d_tiles, 8 * (size_t)std::max<int64_t>(pl->n_tiles, 1)) ||
        cudaMalloc(&pl->d_counters, 8 * (size_t)n_groups) ||
        cudaMalloc(&pl->d_pb_off, 8 * pb_off_all.size()) || cudaMalloc(&pl->d_pb_ij, pb_ij_bytes) ||
        cudaMalloc(&pl->d_job_slots, sizeof(BestSlot) * (size_t)n * grid) ||
        cudaMalloc(&pl->d_results, sizeof(BestSlot) * n) || cudaMallocHost(&pl->h_results, sizeof(BestSlot) * n) ||
        cudaMallocHost(&pl->h_err, sizeof(int)) || cudaMalloc(&pl->d_resc, sizeof(Rescored) * n) ||
        cudaMallocHost(&pl->h_resc, sizeof(Rescored) * n))
      return fail(ctx, EPIK2_E_NOMEM, "batched plan: device memory");
    CK(ctx, cudaMemcpyAsync(pl->d_pb_off, pb_off_all.data(), 8 * pb_off_all.size(), cudaMemcpyHostToDevice,
                            ctx->stream),
       "upload batch");
    if (!pb_ij_all.empty())
      CK(ctx, cudaMemcpyAsync(pl->d_pb_ij, pb_ij_all.data(), 4 * pb_ij_all.size(), cudaMemcpyHostToDevice,
                              ctx->stream),
         "upload batch");
    ctx->stats.h2d_bytes += 8 * pb_off_all.size() + 4 * pb_ij_all.size();
    for (int32_t b = 0; b < n; b++) {
      CK(ctx, launch_expand_tiles(pl->d_pb_off + job_pb_base[b], pl->d_pb_ij + job_ij_base[b], job_n_pb[b],
                                  codes[b] & 1, b, pl->d_tiles + job_off[b], ctx->stream),
         "tile descriptors");
      ctx->stats.kernel_launches += 1;
    }
    CK(ctx, cudaStreamSynchronize(ctx->stream), "upload batch");
    // capture: reset slots, counters and error word; one batched search per group;
    // per-dataset reduce; optional FP64 rescore; read back
    CK(ctx, tc_configure(), "configure");
    CK(ctx, pipe_configure(), "configure");
    CK(ctx, launch_fill_slots(pl->d_job_slots, (int64_t)n * grid, ctx->stream), "configure");  // also loads modules
    CK(ctx, cudaStreamSynchronize(ctx->stream), "configure");
    CK(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
    cudaError_t e = launch_fill_slots(pl->d_job_slots, (int64_t)n * grid, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(pl->d_counters, 0, 8 * (size_t)n_groups, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_err, 0, 4, ctx->stream);
    for (int g = 0; g < n_groups && e == cudaSuccess; g++) {
      const int64_t nt = pl->group_off[g + 1] - pl->group_off[g];
      if (nt == 0) continue;
      TcParams p{};
      p.counter = pl->d_counters + g;
      p.err = ctx->d_err;
      p.wait_limit = ctx->wait_limit;
  p.wait_limit = ctx->wait_limit;
      p.jobs = pl->d_jobs;
      p.tiles = pl->d_tiles + pl->group_off[g];
      p.n_jobs = n;
      p.job_slots = pl->d_job_slots;
      p.n_tiles = nt;
      const bool gp = (group_code[g] & 2) != 0, gov = (group_code[g] & 4) != 0;
      if (gov)
        e = launch_scan_pipe(p, tc_pair_blocks(grid), group_code[g] >> 3, false, ctx->stream);
      else
        e = launch_scan_tc(p, gp ? tc_pair_blocks(grid) : grid, group_code[g] >> 3, group_code[g] & 1, gp, false,
                           ctx->stream);
    }
    if (e == cudaSuccess) e = launch_reduce_jobs(pl->d_job_slots, n, grid, pl->d_results, ctx->stream);
    if (e == cudaSuccess && rescore) e = launch_rescore_jobs(pl->d_jobs, pl->d_results, n, pl->d_resc, ctx->stream);
    if (e == cudaSuccess && rescore)
      e = cudaMemcpyAsync(pl->h_resc, pl->d_resc, sizeof(Rescored) * n, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(pl->h_results, pl->d_results, sizeof(BestSlot) * n, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(pl->h_err, ctx->d_err, 4, cudaMemcpyDeviceToHost, ctx->stream);
    cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &pl->graph);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&pl->exec, pl->graph, 0);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batched graph");
    plan = pl.get();
    ctx->plans[key] = std::move(pl);
    touch(key);
  }
  // refresh the job table (class splits may have changed since the plan was built)
  for (int32_t b = 0; b < n; b++) {
    const DevDataset& d = *ds[b];
    TcJob& j = plan->h_jobs[b];
    j.planes = d.planes;
    j.singles = d.singles;
    j.pairs = d.pairs;
    j.lut = d.lut;
    j.lut64 = d.lut64;
    j.tri = d.tri;
    j.m = (int32_t)d.n_snps;
    j.m_pad = (int32_t)d.m_pad;
    j.w0 = (int32_t)d.w0;
    j.w1 = (int32_t)d.w1;
    j.n0 = (int32_t)d.n_controls;
    j.n1 = (int32_t)d.n_cases;
  }
  CK(ctx, cudaMemcpyAsync(plan->d_jobs, plan->h_jobs.data(), sizeof(TcJob) * n, cudaMemcpyHostToDevice, ctx->stream),
     "upload job table");
  ctx->stats.h2d_bytes += sizeof(TcJob) * n;
  CK(ctx, cudaEventRecord(ctx->ev_start, ctx->stream), "event");
  CK(ctx, cudaGraphLaunch(plan->exec, ctx->stream), "batched graph launch");
  CK(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream), "event");
  CK(ctx, cudaStreamSynchronize(ctx->stream), "batched search");
  ctx->stats.kernel_launches += 2 + (uint64_t)plan->group_code.size() + (rescore ? 1 : 0);
  ctx->stats.d2h_bytes += sizeof(BestSlot) * n + 4;
  if (*plan->h_err) return fail(ctx, EPIK2_E_TIMEOUT, "batched search: a bounded wait expired");
  float kms = 0.0f;
  CK(ctx, cudaEventElapsedTime(&kms, ctx->ev_start, ctx->ev_stop), "event time");
  ctx->stats.last_scan_kernel_ms = kms;
  int64_t trip = 0;
  for (auto* d : ds) trip += triplets_before(d->n_snps, d->n_snps);
  ctx->stats.last_scan_triplets = trip;
  ctx->stats.last_scan_words = 0;
  for (int32_t b = 0; b < n; b++) {
    const BestSlot& r = plan->h_results[b];
    out[b].score = r.score;
    out[b].score_fp64 = rescore ? plan->h_resc[b].s64 : std::numeric_limits<double>::quiet_NaN();
    decode_key(r.key, out[b].i, out[b].j, out[b].k);
  }
  return EPIK2_OK;
}

}  // namespace

extern "C" {

const char* epik2_strerror(int status) {
  switch (status) {
    case EPIK2_OK: return "ok";
    case EPIK2_E_INVALID: return "invalid argument";
    case EPIK2_E_CUDA: return "CUDA error";
    case EPIK2_E_NOMEM: return "out of device memory";
    case EPIK2_E_NOT_FOUND: return "not found";
    case EPIK2_E_TOO_LARGE: return "size beyond limit";
    case EPIK2_E_TIMEOUT: return "timeout";
    case EPIK2_E_NO_DEVICE: return "no suitable CUDA device";
    case EPIK2_E_BUSY: return "busy";
    case EPIK2_E_CANCELLED: return "cancelled";
    default: return "unknown status";
  }
}

const char* epik2_last_error(const epik2_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int epik2_create(epik2_ctx** out, int device) {
  if (!out) return EPIK2_E_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return EPIK2_E_NO_DEVICE;
  if (device < 0 || device >= n) return EPIK2_E_INVALID;
  std::unique_ptr<epik2_ctx> ctx(new epik2_ctx());
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess) return EPIK2_E_NO_DEVICE;
  if (cudaGetDeviceProperties(&ctx->prop, device) != cudaSuccess) return EPIK2_E_NO_DEVICE;
  if (ctx->prop.major != 10) return EPIK2_E_NO_DEVICE;  // built for sm_100a only
  if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) return EPIK2_E_CUDA;
  ctx->stream = ctx->own_stream;
  if (cudaEventCreate(&ctx->ev_start) != cudaSuccess || cudaEventCreate(&ctx->ev_stop) != cudaSuccess ||
      cudaEventCreate(&ctx->ev_load[0]) != cudaSuccess || cudaEventCreate(&ctx->ev_load[1]) != cudaSuccess ||
      cudaEventCreate(&ctx->ev_load[2]) != cudaSuccess) {
    epik2_destroy(ctx.release());
    return EPIK2_E_CUDA;
  }
  ctx->scan_blocks = ctx->prop.multiProcessorCount * scan_blocks_per_sm();
  ctx->tc_blocks = ctx->prop.multiProcessorCount;
  const int n_warps = std::max(ctx->scan_blocks * (kScanThreads / 32), ctx->tc_blocks * tc_warps_per_block());
  ctx->n_slots = n_warps;
  if (cudaMalloc(&ctx->d_counter, 64) != cudaSuccess || cudaMalloc(&ctx->d_err, 64) != cudaSuccess || cudaMalloc(&ctx->d_slots, sizeof(BestSlot) * n_warps) ||
      cudaMalloc(&ctx->d_best, sizeof(BestSlot)) || cudaMalloc(&ctx->d_cand, sizeof(BestSlot) * n_warps * 32) ||
      cudaMalloc(&ctx->d_resc, sizeof(Rescored) * n_warps * 32) ||
      cudaMallocHost(&ctx->h_best, sizeof(BestSlot))) {
    epik2_destroy(ctx.release());
    return EPIK2_E_NOMEM;
  }
  *out = ctx.release();
  return EPIK2_OK;
}

void epik2_destroy(epik2_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  ctx->plans.clear();
  for (auto& kv : ctx->datasets) cudaFree(kv.second->block);
  ctx->datasets.clear();
  cudaFree(ctx->spare_block);
  cudaFree(ctx->d_counter);
  cudaFree(ctx->d_slots);
  cudaFree(ctx->d_best);
  cudaFree(ctx->d_cand);
  cudaFree(ctx->d_resc);
  cudaFree(ctx->d_pgoff);
  cudaFree(ctx->d_err);
  cudaFree(ctx->d_pb_off);
  cudaFree(ctx->d_pb_ij);
  cudaFree(ctx->d_tiles);
  cudaFree(ctx->d_rep_jobs);
  cudaFree(ctx->d_rep_slots);
  cudaFree(ctx->d_rep_res);
  cudaFree(ctx->d_rep_resc);
  cudaFreeHost(ctx->h_best);
  if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
  if (ctx->ev_stop) cudaEventDestroy(ctx->ev_stop);
  for (cudaEvent_t e : ctx->ev_load)
    if (e) cudaEventDestroy(e);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
}

int epik2_device_name(const epik2_ctx* ctx, char* buf, size_t len) {
  if (!ctx || !buf || len == 0) return EPIK2_E_INVALID;
  snprintf(buf, len, "%s", ctx->prop.name);
  return EPIK2_OK;
}

int epik2_mem_info(const epik2_ctx* ctx, size_t* free_bytes, size_t* total_bytes) {
  if (!ctx || !free_bytes || !total_bytes) return EPIK2_E_INVALID;
  cudaSetDevice(ctx->device);
  if (cudaMemGetInfo(free_bytes, total_bytes) != cudaSuccess) return EPIK2_E_CUDA;
  *free_bytes += ctx->spare_bytes;  // the context's spare allocation is reused or released on demand
  return EPIK2_OK;
}

int epik2_set_stream(epik2_ctx* ctx, void* cuda_stream) {
  if (!ctx) return EPIK2_E_INVALID;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx->stream = cuda_stream ? (cudaStream_t)cuda_stream : ctx->own_stream;
  return EPIK2_OK;
}

int epik2_set_engine(epik2_ctx* ctx, int engine) {
  if (!ctx) return EPIK2_E_INVALID;
  if (engine < EPIK2_ENGINE_AUTO || engine > EPIK2_ENGINE_TC_FP4) return fail(ctx, EPIK2_E_INVALID, "unknown engine");
  ctx->engine = engine;
  return EPIK2_OK;
}

int epik2_set_stage_words(epik2_ctx* ctx, int stage_words) {
  if (!ctx) return EPIK2_E_INVALID;
  if (stage_words != 0 && stage_words != 4 && stage_words != 8 && stage_words != 16)
    return fail(ctx, EPIK2_E_INVALID, "stage_words must be 0, 4, 8 or 16");
  ctx->stage_words = stage_words;
  return EPIK2_OK;
}

int epik2_set_wait_limit(epik2_ctx* ctx, int64_t sm_clocks) {
  if (!ctx) return EPIK2_E_INVALID;
  if (sm_clocks < 0) return fail(ctx, EPIK2_E_INVALID, "wait limit must be >= 0");
  ctx->wait_limit = sm_clocks;
  return EPIK2_OK;
}

int epik2_test_withhold_arrival(epik2_ctx* ctx) {
  if (!ctx) return EPIK2_E_INVALID;
  ctx->test_withhold = 1;
  return EPIK2_OK;
}

int epik2_set_overlap(epik2_ctx* ctx, int overlap) {
  if (!ctx) return EPIK2_E_INVALID;
  if (overlap < 0 || overlap > 2) return fail(ctx, EPIK2_E_INVALID, "overlap must be 0, 1 or 2");
  ctx->overlap = overlap;
  return EPIK2_OK;
}

int epik2_set_pair_tile(epik2_ctx* ctx, int pair_tile) {
  if (!ctx) return EPIK2_E_INVALID;
  if (pair_tile != 0 && pair_tile != 32 && pair_tile != 64) return fail(ctx, EPIK2_E_INVALID, "pair_tile must be 0, 32 or 64");
  ctx->pair_tile = pair_tile;
  return EPIK2_OK;
}

int epik2_get_stream(const epik2_ctx* ctx, void** cuda_stream) {
  if (!ctx || !cuda_stream) return EPIK2_E_INVALID;
  *cuda_stream = (void*)ctx->stream;
  return EPIK2_OK;
}

int epik2_get_stats(const epik2_ctx* ctx, epik2_stats* out) {
  if (!ctx || !out) return EPIK2_E_INVALID;
  *out = ctx->stats;
  return EPIK2_OK;
}

int epik2_reset_stats(epik2_ctx* ctx) {
  if (!ctx) return EPIK2_E_INVALID;
  ctx->stats = epik2_stats{};
  return EPIK2_OK;
}

int epik2_generate_reference(int64_t n_samples, int64_t n_snps, uint8_t* geno, uint8_t* pheno) {
  if (n_samples < 1 || n_snps < 1 || !geno || !pheno || n_samples > INT32_MAX) return EPIK2_E_INVALID;
  generate_reference(n_samples, n_snps, geno, pheno);
  return EPIK2_OK;
}

int epik2_generate_hwe(uint64_t seed, int64_t n_samples, int64_t n_snps, int64_t n_cases, double maf_lo,
                       double maf_hi, int32_t n_planted, const int64_t* planted, const double* effects, uint8_t* geno,
                       uint8_t* pheno) {
  if (n_samples < 1 || n_snps < 1 || !geno || !pheno || n_cases < 0 || n_cases > n_samples) return EPIK2_E_INVALID;
  if (!(maf_lo >= 0.0 && maf_hi <= 1.0 && maf_lo <= maf_hi)) return EPIK2_E_INVALID;
  if (n_planted < 0 || (n_planted > 0 && (!planted || !effects))) return EPIK2_E_INVALID;
  for (int t = 0; t < n_planted; t++) {
    for (int q = 0; q < 3; q++)
      if (planted[3 * t + q] < 0 || planted[3 * t + q] >= n_snps) return EPIK2_E_INVALID;
    if (!(effects[t] > 0.0 && effects[t] < 1.0)) return EPIK2_E_INVALID;
  }
  generate_hwe(seed, n_samples, n_snps, n_cases, maf_lo, maf_hi, n_planted, planted, effects, geno, pheno);
  return EPIK2_OK;
}

int64_t epik2_dataset_bytes(int64_t n_samples, int64_t n_snps) {
  if (n_samples < 1 || n_snps < 1) return -1;
  return (int64_t)dataset_layout(n_samples, n_snps).total;
}

int epik2_load_u8(epik2_ctx* ctx, const uint8_t* geno, const uint8_t* pheno, int64_t n_samples, int64_t n_snps,
                  int32_t* dataset_id) {
  if (!ctx) return EPIK2_E_INVALID;
  if (!geno || !pheno || !dataset_id) return fail(ctx, EPIK2_E_INVALID, "null pointer");
  if (n_samples < 1 || n_snps < 1) return fail(ctx, EPIK2_E_INVALID, "n_samples and n_snps must be >= 1");
  if (n_samples > EPIK2_MAX_SAMPLES || n_snps > EPIK2_MAX_SNPS)
    return fail(ctx, EPIK2_E_TOO_LARGE, "n_samples or n_snps beyond limit");
  CK(ctx, cudaSetDevice(ctx->device), "set device");
  const Layout L = dataset_layout(n_samples, n_snps);
  // the spare allocation serves when it fits without doubling the footprint (take_block):
  // then nothing new is allocated and free memory need not be asked for
  const bool reuse = ctx->spare_block && ctx->spare_bytes >= L.total && ctx->spare_bytes <= 2 * L.total;
  if (!reuse) {
    size_t fr = 0, tot = 0;
    CK(ctx, cudaMemGetInfo(&fr, &tot), "mem info");
    if (L.total + (size_t)(256u << 20) > fr + ctx->spare_bytes)
      return fail(ctx, EPIK2_E_NOMEM, "dataset does not fit in free device memory");
  }
  std::unique_ptr<DevDataset> d(new DevDataset());
  CK(ctx, take_block(ctx, L.total, &d->block, &d->block_bytes), "alloc dataset");
  char* b = (char*)d->block;
  d->bytes = L.total;
  d->n_samples = n_samples;
  d->n_snps = n_snps;
  d->m_pad = (n_snps + 31) / 32 * 32;
  d->tri = tri_size(d->m_pad);
  d->geno = (uint8_t*)(b + L.geno);
  d->perm = (int32_t*)(b + L.perm);
  d->planes = (uint2*)(b + L.planes);
  d->singles = (uint32_t*)(b + L.singles);
  d->pairs = (uint4*)(b + L.pairs);
  d->lut = (float*)(b + L.lut);
  d->lut64 = (double*)(b + L.lut64);
  const auto t_load = std::chrono::steady_clock::now();
  if (ctx->lut_samples != n_samples) {
    ctx->lut_host.assign((size_t)n_samples + 2, 0.0f);
    build_k2_lut(n_samples + 1, ctx->lut_host.data());
    ctx->lut64_host.assign((size_t)n_samples + 2, 0.0);
    build_k2_lut64(n_samples + 1, ctx->lut64_host.data());
    ctx->lut_samples = n_samples;
  }
  const std::vector<float>& lut = ctx->lut_host;
  const std::vector<double>& lut64 = ctx->lut64_host;
  cudaEventRecord(ctx->ev_load[0], ctx->stream);
  cudaError_t e = cudaMemcpyAsync(d->geno, geno, (size_t)(n_samples * n_snps), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d->lut, lut.data(), lut.size() * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d->lut64, lut64.data(), lut64.size() * 8, cudaMemcpyHostToDevice, ctx->stream);
  ctx->stats.h2d_bytes += (uint64_t)(n_samples * n_snps) + lut.size() * 4 + lut64.size() * 8;
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_load[1], ctx->stream);
  if (e != cudaSuccess) {
    cudaFree(d->block);
    return cuda_fail(ctx, e, "upload dataset");
  }
  int r = encode_with(ctx, *d, pheno);
  if (r) {
    cudaFree(d->block);
    return r;
  }
  // load breakdown: host -> device copies, then encode + margins (encode_with waited for them)
  float up_ms = 0.0f, prep_ms = 0.0f;
  if (cudaEventRecord(ctx->ev_load[2], ctx->stream) == cudaSuccess && cudaEventSynchronize(ctx->ev_load[2]) == cudaSuccess) {
    cudaEventElapsedTime(&up_ms, ctx->ev_load[0], ctx->ev_load[1]);
    cudaEventElapsedTime(&prep_ms, ctx->ev_load[1], ctx->ev_load[2]);
  }
  ctx->stats.last_upload_ms = up_ms;
  ctx->stats.last_prepare_ms = prep_ms;
  ctx->stats.last_load_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_load).count();
  const int32_t id = ctx->next_id++;
  ctx->datasets[id] = std::move(d);
  *dataset_id = id;
  return EPIK2_OK;
}

int epik2_set_pheno(epik2_ctx* ctx, int32_t dataset_id, const uint8_t* pheno) {
  if (!ctx) return EPIK2_E_INVALID;
  DevDataset* d = find(ctx, dataset_id);
  if (!d) return fail(ctx, EPIK2_E_NOT_FOUND, "unknown dataset");
  if (!pheno) return fail(ctx, EPIK2_E_INVALID, "null phenotype");
  CK(ctx, cudaSetDevice(ctx->device), "set device");
  return encode_with(ctx, *d, pheno);
}

int64_t epik2_replicate_bytes(int64_t n_samples, int64_t n_snps) {
  if (n_samples < 1 || n_snps < 1) return -1;
  return (int64_t)dataset_layout(n_samples, n_snps, false).total;
}

int epik2_load_replicate(epik2_ctx* ctx, int32_t base_dataset_id, const uint8_t* pheno, int32_t* dataset_id) {
  if (!ctx) return EPIK2_E_INVALID;
  if (!pheno || !dataset_id) return fail(ctx, EPIK2_E_INVALID, "null pointer");
  DevDataset* base = find(ctx, base_dataset_id);
  if (!base) return fail(ctx, EPIK2_E_NOT_FOUND, "unknown dataset");
  int32_t root_id = base->base_id >= 0 ? base->base_id : base_dataset_id;
  DevDataset* root = find(ctx, root_id);
  if (!root) return fail(ctx, EPIK2_E_NOT_FOUND, "genotype owner no longer loaded");
  CK(ctx, cudaSetDevice(ctx->device), "set device");
  const Layout L = dataset_layout(root->n_samples, root->n_snps, false);
  if (!(ctx->spare_block && ctx->spare_bytes >= L.total && ctx->spare_bytes <= 2 * L.total)) {
    size_t fr = 0, tot = 0;  // a new allocation: ask for free memory (about a millisecond)
    CK(ctx, cudaMemGetInfo(&fr, &tot), "mem info");
    if (L.total + (size_t)(256u << 20) > fr + ctx->spare_bytes)
      return fail(ctx, EPIK2_E_NOMEM, "replicate does not fit in free device memory");
  }
  std::unique_ptr<DevDataset> d(new DevDataset());
  CK(ctx, take_block(ctx, L.total, &d->block, &d->block_bytes), "alloc replicate");
  char* b = (char*)d->block;
  d->bytes = L.total;
  d->n_samples = root->n_samples;
  d->n_snps = root->n_snps;
  d->m_pad = root->m_pad;
  d->tri = root->tri;
  d->geno = root->geno;
  d->perm = (int32_t*)(b + L.perm);
  d->planes = (uint2*)(b + L.planes);
  d->singles = (uint32_t*)(b + L.singles);
  d->pairs = (uint4*)(b + L.pairs);
  d->lut = (float*)(b + L.lut);
  d->lut64 = (double*)(b + L.lut64);
  d->base_id = root_id;
  cudaError_t e = cudaMemcpyAsync(d->lut, root->lut, (size_t)(root->n_samples + 2) * 4, cudaMemcpyDeviceToDevice,
                                  ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d->lut64, root->lut64, (size_t)(root->n_samples + 2) * 8, cudaMemcpyDeviceToDevice,
                        ctx->stream);
  if (e != cudaSuccess) {
    cudaFree(d->block);
    return cuda_fail(ctx, e, "replicate tables");
  }
  int r = encode_with(ctx, *d, pheno);
  if (r) {
    cudaFree(d->block);
    return r;
  }
  root->n_replicates++;
  const int32_t id = ctx->next_id++;
  ctx->datasets[id] = std::move(d);
  *dataset_id = id;
  return EPIK2_OK;
}

namespace {
// keep: the allocation becomes the context's spare block (the one-call entry point)
int unload_dataset(epik2_ctx* ctx, int32_t dataset_id, bool keep) {
  if (!ctx) return EPIK2_E_INVALID;
  auto it = ctx->datasets.find(dataset_id);
  if (it == ctx->datasets.end()) return fail(ctx, EPIK2_E_NOT_FOUND, "unknown dataset");
  if (it->second->n_replicates > 0) return fail(ctx, EPIK2_E_BUSY, "dataset still has live replicates");
  if (it->second->base_id >= 0) {
    DevDataset* root = find(ctx, it->second->base_id);
    if (root) root->n_replicates--;
  }
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (keep) {
    drop_spare(ctx);
    ctx->spare_block = it->second->block;
    ctx->spare_bytes = it->second->block_bytes;
  } else {
    cudaFree(it->second->block);
  }
  ctx->datasets.erase(it);
  return EPIK2_OK;
}
}  // namespace

int epik2_unload(epik2_ctx* ctx, int32_t dataset_id) { return unload_dataset(ctx, dataset_id, false); }

int epik2_dataset_info(const epik2_ctx* ctx, int32_t dataset_id, int64_t* n_samples, int64_t* n_snps,
                       int64_t* n_cases, int64_t* device_bytes) {
  if (!ctx) return EPIK2_E_INVALID;
  auto it = ctx->datasets.find(dataset_id);
  if (it == ctx->datasets.end()) return EPIK2_E_NOT_FOUND;
  const DevDataset& d = *it->second;
  if (n_samples) *n_samples = d.n_samples;
  if (n_snps) *n_snps = d.n_snps;
  if (n_cases) *n_cases = d.n_cases;
  if (device_bytes) *device_bytes = (int64_t)d.bytes;
  return EPIK2_OK;
}

int epik2_scan(epik2_ctx* ctx, int32_t dataset_id, const epik2_opts* opts, epik2_best* out) {
  if (!ctx) return EPIK2_E_INVALID;
  if (!out) return fail(ctx, EPIK2_E_INVALID, "null output");
  DevDataset* d = find(ctx, dataset_id);
  if (!d) return fail(ctx, EPIK2_E_NOT_FOUND, "unknown dataset");
  if (d->n_snps < 3) return fail(ctx, EPIK2_E_INVALID, "need at least 3 SNPs");
  CK(ctx, cudaSetDevice(ctx->device), "set device");
  BestSlot b{};
  epik2_opts o{};
  if (opts) o = *opts;
  if (o.rescore_fp64 && o.top_k < 2) o.top_k = 32;
  const auto t_scan = std::chrono::steady_clock::now();
  int r = run_scan(ctx, *d, &o, nullptr, nullptr, &b);
  ctx->stats.last_scan_wall_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_scan).count();
  if (r) return r;
  if (b.key == ~0ull) return fail(ctx, EPIK2_E_INVALID, "no triplet in the requested range");
  if (o.rescore_fp64) {
    if (ctx->last_topk.empty()) return fail(ctx, EPIK2_E_CUDA, "rescore produced no candidate");
    *out = ctx->last_topk[0];  // best by FP64 score
    return EPIK2_OK;
  }
  out->score = b.score;
  out->score_fp64 = std::numeric_limits<double>::quiet_NaN();
  decode_key(b.key, out->i, out->j, out->k);
  return EPIK2_OK;
}

int epik2_scan_topk(epik2_ctx* ctx, int32_t dataset_id, const epik2_opts* opts, epik2_best* out, int32_t capacity,
                    int32_t* n_out) {
  if (!ctx) return EPIK2_E_INVALID;
  if (!out || !n_out || capacity < 1) return fail(ctx, EPIK2_E_INVALID, "bad output buffer");
  epik2_opts o{};
  if (opts) o = *opts;
  if (o.top_k < 2) o.top_k = std::min(capacity, 32);
  epik2_best best{};
  int r = epik2_scan(ctx, dataset_id, &o, &best);
  if (r) return r;
  const int n = std::min<int>(capacity, (int)ctx->last_topk.size());
  for (int t = 0; t < n; t++) out[t] = ctx->last_topk[(size_t)t];
  *n_out = n;
  return EPIK2_OK;
}

int epik2_scan_u8(epik2_ctx* ctx, const uint8_t* geno, const uint8_t* pheno, int64_t n_samples, int64_t n_snps,
                  const epik2_opts* opts, epik2_best* out) {
  int32_t id = 0;
  int r = epik2_load_u8(ctx, geno, pheno, n_samples, n_snps, &id);
  if (r) return r;
  r = epik2_scan(ctx, id, opts, out);
  unload_dataset(ctx, id, true);
  return r;
}

int epik2_autotune(epik2_ctx* ctx, int32_t dataset_id, epik2_tune* out) {
  if (!ctx) return EPIK2_E_INVALID;
  if (!out) return fail(ctx, EPIK2_E_INVALID, "null output");
  DevDataset* d = find(ctx, dataset_id);
  if (!d) return fail(ctx, EPIK2_E_NOT_FOUND, "unknown dataset");
  if (d->n_snps < 3) return fail(ctx, EPIK2_E_INVALID, "need at least 3 SNPs");
  CK(ctx, cudaSetDevice(ctx->device), "set device");
  int r = autotune_now(ctx, *d, out);
  if (r) return r;
  ctx->tune_cache[shape_bucket(*d)] = *out;
  return EPIK2_OK;
}

int epik2_scan_batch(epik2_ctx* ctx, const int32_t* dataset_ids, int32_t n, const epik2_opts* opts, epik2_best* out) {
  if (!ctx) return EPIK2_E_INVALID;
  if (!dataset_ids || !out || n < 1) return fail(ctx, EPIK2_E_INVALID, "bad dataset list");
  if (n > kMaxBatchJobs) return fail(ctx, EPIK2_E_TOO_LARGE, "at most 512 datasets per batched launch");
  std::vector<DevDataset*> ds;
  std::vector<int32_t> ids(dataset_ids, dataset_ids + n);
  for (int32_t b = 0; b < n; b++) {
    DevDataset* d = find(ctx, dataset_ids[b]);
    if (!d) return fail(ctx, EPIK2_E_NOT_FOUND, "unknown dataset in batch");
    if (d->n_snps < 3) return fail(ctx, EPIK2_E_INVALID, "every dataset needs at least 3 SNPs");
    ds.push_back(d);
  }
  CK(ctx, cudaSetDevice(ctx->device), "set device");
  // One configuration (format, stage depth, pair tile) for every dataset, so that all the
  // tiles drain from one queue in one persistent launch: the requested one, else, among the
  // tensor-core configurations every dataset can take that match what was requested, the
  // one with the least predicted time: sum over datasets of work / the autotuner's rate for
  // the dataset's shape.
  const int engine_req = opts ? opts->engine : 0;
  const int kw_req = opts ? opts->stage_words : 0;
  const int pt_req = opts ? opts->pair_tile : 0;
  const int ov_req = opts ? opts->overlap : 0;
  if (engine_req == EPIK2_ENGINE_INT) return fail(ctx, EPIK2_E_INVALID, "the batched form runs on the tensor cores");
  if (engine_req < 0 || engine_req > EPIK2_ENGINE_TC_FP4) return fail(ctx, EPIK2_E_INVALID, "unknown engine");
  if (pt_req != 0 && pt_req != 32 && pt_req != 64) return fail(ctx, EPIK2_E_INVALID, "pair_tile must be 0, 32 or 64");
  if (ov_req < 0 || ov_req > 2) return fail(ctx, EPIK2_E_INVALID, "overlap must be 0, 1 or 2");
  bool all_fp4 = true, all_overlap = true;
  for (DevDataset* d : ds) {
    all_fp4 = all_fp4 && fp4_exact(*d);
    all_overlap = all_overlap && fp4_exact(*d) && pipe_fits(d->n_controls, d->n_cases);
  }
  if (engine_req == EPIK2_ENGINE_TC_FP4 && !all_fp4)
    return fail(ctx, EPIK2_E_TOO_LARGE, "FP4 tensor-core engine: a class of 2^24 samples or more");
  if (ov_req == 2 && !all_overlap)
    return fail(ctx, EPIK2_E_TOO_LARGE, "overlapped kernel: classes of at most 65535 samples");
  TcConfig pick{0, 0, false, false};
  bool have = false;
  if (engine_req != 0 && kw_req != 0 && (pt_req != 0 || engine_req == EPIK2_ENGINE_TC) && ov_req != 0) {
    pick = TcConfig{engine_req, kw_req, pt_req == 64, ov_req == 2};
    have = true;
  } else if (engine_req == EPIK2_ENGINE_TC && kw_req != 0) {
    pick = TcConfig{engine_req, kw_req, false, false};
    have = true;
  } else if (engine_req == EPIK2_ENGINE_TC_FP4 && kw_req != 0 && pt_req == 0 && ov_req == 0) {
    pick = TcConfig{engine_req, kw_req, kw_req == 16, false};  // stage depth given, nothing else
    have = true;
  } else {
    std::vector<epik2_tune> tunes;
    for (DevDataset* d : ds) {
      epik2_tune t{};
      int r = tuned(ctx, *d, &t);
      if (r) return r;
      tunes.push_back(t);
    }
    double best_time = 0.0;
    for (const TcConfig& c : kTcConfigs) {
      if (engine_req && c.engine != engine_req) continue;
      if (kw_req && c.kw != kw_req) continue;
      if (pt_req && c.pair != (pt_req == 64)) continue;
      if (ov_req && c.overlap != (ov_req == 2)) continue;
      if (!config_fits(c, all_fp4, all_overlap)) continue;
      double time = 0.0;
      bool ok = true;
      for (size_t b = 0; b < ds.size() && ok; b++) {
        const double rate = tune_rate(tunes[b], c.engine, c.kw, c.pair, c.overlap);
        const double m = (double)ds[b]->n_snps;
        ok = rate > 0.0;
        time += m * (m - 1) * (m - 2) / 6.0 * (double)ds[b]->n_samples / (ok ? rate : 1.0);
      }
      if (ok && (!have || time < best_time)) {
        best_time = time;
        pick = c;
        have = true;
      }
    }
  }
  if (!have) return fail(ctx, EPIK2_E_INVALID, "no tensor-core configuration matches the request");
  const bool fp4 = pick.engine == EPIK2_ENGINE_TC_FP4;
  if (!config_valid(pick.engine, pick.kw, pick.pair, pick.overlap))
    return fail(ctx, EPIK2_E_INVALID,
                "tensor-core configuration: int8 takes 4 or 8 words per stage on 32-SNP tiles; FP4 takes 8 or 16 "
                "(32- or 64-SNP tiles), or 4 or 8 overlapped on 64-SNP tiles");
  const std::vector<int> codes(ds.size(), tc_code(pick.kw, fp4, pick.pair && fp4, pick.overlap));
  return run_batch(ctx, ds, ids, codes, opts && opts->rescore_fp64, out);
}

int epik2_scan_replicates(epik2_ctx* ctx, int32_t dataset_id, const uint8_t* phenos, int32_t n_reps,
                          const epik2_opts* opts, epik2_best* out) {
  if (!ctx) return EPIK2_E_INVALID;
  if (!phenos || !out || n_reps < 1) return fail(ctx, EPIK2_E_INVALID, "bad replicate list");
  DevDataset* base = find(ctx, dataset_id);
  if (!base) return fail(ctx, EPIK2_E_NOT_FOUND, "unknown dataset");
  if (base->n_snps < 3) return fail(ctx, EPIK2_E_INVALID, "need at least 3 SNPs");
  if (!fp4_exact(*base))
    return fail(ctx, EPIK2_E_TOO_LARGE, "replicate form (FP4 on CTA pairs): a class of 2^24 samples or more");
  CK(ctx, cudaSetDevice(ctx->device), "set device");
  const int64_t S = base->n_samples, m = base->n_snps;
  const int grid = tc_pair_blocks(ctx->tc_blocks);
  // replicates per launch: as many as fit in free device memory above 1 GiB, at most 256.
  // Their class orders, planes and margins live in one allocation for the whole call, kept
  // afterwards as the context's spare allocation (the next call of the same shape reuses it;
  // any other allocation of the context releases it first); their genotypes and ln n! tables
  // are the base dataset's.
  const auto t_call = std::chrono::steady_clock::now();
  const Layout L = dataset_layout(S, m, false);
  const size_t rep_bytes = align_up(L.total, 256);
  const int64_t want = std::min<int64_t>(n_reps, 256);
  int64_t fit = want;  // a spare allocation that holds them all needs no free-memory query
  if (!(ctx->spare_block && ctx->spare_bytes >= rep_bytes * (size_t)want)) {
    size_t fr = 0, tot = 0;
    CK(ctx, cudaMemGetInfo(&fr, &tot), "mem info");
    fr += ctx->spare_bytes;
    fit = ((int64_t)fr - ((int64_t)1 << 30)) / (int64_t)rep_bytes;
  }
  const int32_t group = (int32_t)std::max<int64_t>(1, std::min<int64_t>(fit, want));
  int r = EPIK2_OK;
  const bool rescore = opts && opts->rescore_fp64;
  char* arena = nullptr;
  size_t arena_bytes = 0;
  cudaError_t e = cudaSuccess;
  const size_t need = rep_bytes * (size_t)group;
  if (ctx->spare_block && ctx->spare_bytes >= need) {  // a larger spare serves too: it is returned
    arena = static_cast<char*>(ctx->spare_block);
    arena_bytes = ctx->spare_bytes;
    ctx->spare_block = nullptr;
    ctx->spare_bytes = 0;
  } else {
    e = take_block(ctx, need, reinterpret_cast<void**>(&arena), &arena_bytes);
  }
  if (e == cudaSuccess && (group > ctx->rep_cap || (int64_t)group * grid > ctx->rep_slot_cap)) {
    cudaFree(ctx->d_rep_jobs);
    cudaFree(ctx->d_rep_slots);
    cudaFree(ctx->d_rep_res);
    cudaFree(ctx->d_rep_resc);
    ctx->d_rep_jobs = nullptr;
    ctx->d_rep_slots = nullptr;
    ctx->d_rep_res = nullptr;
    ctx->d_rep_resc = nullptr;
    ctx->rep_cap = ctx->rep_slot_cap = 0;
    const int64_t cap = std::max<int64_t>(group, 64);
    e = cudaMalloc(&ctx->d_rep_jobs, sizeof(TcJob) * cap);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_rep_slots, sizeof(BestSlot) * (size_t)cap * grid);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_rep_res, sizeof(BestSlot) * cap);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_rep_resc, sizeof(Rescored) * cap);
    if (e == cudaSuccess) {
      ctx->rep_cap = cap;
      ctx->rep_slot_cap = cap * grid;
    }
  }
  TcJob* d_jobs = ctx->d_rep_jobs;
  BestSlot *d_rslots = ctx->d_rep_slots, *d_res = ctx->d_rep_res;
  Rescored* d_resc = ctx->d_rep_resc;
  const double alloc_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_call).count();
  double encode_ms = 0.0;
  auto release = [&]() {
    cudaStreamSynchronize(ctx->stream);
    if (arena) {  // becomes the context's spare allocation
      drop_spare(ctx);
      ctx->spare_block = arena;
      ctx->spare_bytes = arena_bytes;
    }
  };
  if (e != cudaSuccess) {
    release();
    if (e == cudaErrorMemoryAllocation) {
      cudaGetLastError();
      return fail(ctx, EPIK2_E_NOMEM, "replicate buffers do not fit in free device memory");
    }
    return cuda_fail(ctx, e, "replicate buffers");
  }
  double kms_total = 0.0;
  std::vector<TcJob> jobs((size_t)group);
  std::vector<BestSlot> res((size_t)group);
  std::vector<Rescored> resc((size_t)group);
  std::vector<DevDataset> reps((size_t)group);
  for (int32_t done = 0; done < n_reps; done += group) {
    const int32_t g = std::min<int32_t>(group, n_reps - done);
    const auto t_enc = std::chrono::steady_clock::now();
    for (int32_t t = 0; t < g; t++) {  // each replicate's class order, planes, margins
      DevDataset& R = reps[(size_t)t];
      char* b = arena + rep_bytes * (size_t)t;
      R = DevDataset{};
      R.n_samples = S;
      R.n_snps = m;
      R.m_pad = base->m_pad;
      R.tri = base->tri;
      R.geno = base->geno;
      R.lut = base->lut;
      R.lut64 = base->lut64;
      R.perm = (int32_t*)(b + L.perm);
      R.planes = (uint2*)(b + L.planes);
      R.singles = (uint32_t*)(b + L.singles);
      R.pairs = (uint4*)(b + L.pairs);
      R.bytes = L.total;
      r = encode_with(ctx, R, phenos + (size_t)(done + t) * (size_t)S);
      if (r) {
        release();
        return r;
      }
      jobs[(size_t)t] = TcJob{R.planes, R.singles, R.pairs, R.lut, R.lut64, R.tri, (int32_t)R.n_snps,
                              (int32_t)R.m_pad, (int32_t)R.w0, (int32_t)R.w1, (int32_t)R.n_controls,
                              (int32_t)R.n_cases};
    }
    encode_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_enc).count();
    // the search's tile descriptors, after the replicates' loads (their pair margins use the
    // same descriptor buffer)
    int64_t n_tiles = 0;
    r = prepare_tiles(ctx, m, 0, m, true, true, &n_tiles);
    if (r) {
      release();
      return r;
    }
    e = cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(TcJob) * g, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = launch_fill_slots(d_rslots, (int64_t)g * grid, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_counter, 0, 8, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_err, 0, 4, ctx->stream);
    TcParams p{};
    p.planes = base->planes;  // pass 0: all samples of the base dataset
    p.singles = base->singles;
    p.pairs = base->pairs;
    p.lut = base->lut;
    p.tiles = ctx->d_tiles;
    p.n_tiles = n_tiles;
    p.tri = base->tri;
    p.m = (int32_t)m;
    p.m_pad = (int32_t)base->m_pad;
    p.w0 = (int32_t)base->w0;
    p.w1 = (int32_t)base->w1;
    p.n0 = (int32_t)base->n_controls;
    p.n1 = (int32_t)base->n_cases;
    p.counter = ctx->d_counter;
    p.slots = ctx->d_slots;
    p.err = ctx->d_err;
    p.wait_limit = ctx->wait_limit;
    p.jobs = d_jobs;
    p.n_jobs = g;
    p.n_reps = g;
    p.job_slots = d_rslots;
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_start, ctx->stream);
    if (e == cudaSuccess) e = launch_scan_reps(p, grid, ctx->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_stop, ctx->stream);
    if (e == cudaSuccess) e = launch_reduce_jobs(d_rslots, g, grid, d_res, ctx->stream);
    if (e == cudaSuccess && rescore) e = launch_rescore_jobs(d_jobs, d_res, g, d_resc, ctx->stream);
    if (e == cudaSuccess && rescore)
      e = cudaMemcpyAsync(resc.data(), d_resc, sizeof(Rescored) * g, cudaMemcpyDeviceToHost, ctx->stream);
    int err_word = 0;
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(res.data(), d_res, sizeof(BestSlot) * g, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err_word, ctx->d_err, 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    float kms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&kms, ctx->ev_start, ctx->ev_stop);
    if (e != cudaSuccess) {
      release();
      return cuda_fail(ctx, e, "replicate search");
    }
    if (err_word) {
      release();
      return fail(ctx, EPIK2_E_TIMEOUT, "replicate search: a bounded wait expired");
    }
    ctx->stats.kernel_launches += 3;
    ctx->stats.h2d_bytes += sizeof(TcJob) * g;
    ctx->stats.d2h_bytes += sizeof(BestSlot) * g + 4;
    kms_total += kms;
    for (int32_t t = 0; t < g; t++) {
      epik2_best& b = out[done + t];
      b.score = res[(size_t)t].score;
      b.score_fp64 = rescore ? resc[(size_t)t].s64 : std::numeric_limits<double>::quiet_NaN();
      decode_key(res[(size_t)t].key, b.i, b.j, b.k);
    }
  }
  release();
  ctx->stats.last_scan_kernel_ms = kms_total;
  ctx->stats.last_load_ms = alloc_ms;
  ctx->stats.last_prepare_ms = encode_ms;
  ctx->stats.last_scan_wall_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_call).count();
  ctx->stats.last_scan_triplets = triplets_before(m, m) * n_reps;
  ctx->stats.last_scan_words = 0;
  return EPIK2_OK;
}

int epik2_dump_tables(epik2_ctx* ctx, int32_t dataset_id, uint32_t* tables, float* scores) {
  if (!ctx) return EPIK2_E_INVALID;
  DevDataset* d = find(ctx, dataset_id);
  if (!d) return fail(ctx, EPIK2_E_NOT_FOUND, "unknown dataset");
  const int64_t m = d->n_snps;
  if (m < 3) return fail(ctx, EPIK2_E_INVALID, "need at least 3 SNPs");
  if (m > 512) return fail(ctx, EPIK2_E_TOO_LARGE, "dump limited to 512 SNPs");
  CK(ctx, cudaSetDevice(ctx->device), "set device");
  const int64_t T = m * (m - 1) * (m - 2) / 6;
  uint32_t* dt = nullptr;
  float* ds = nullptr;
  CK(ctx, cudaMalloc(&dt, (size_t)T * 54 * 4), "alloc dump");
  cudaError_t e = cudaMalloc(&ds, (size_t)T * 4);
  if (e != cudaSuccess) {
    cudaFree(dt);
    return cuda_fail(ctx, e, "alloc dump");
  }
  BestSlot b{};
  int r = run_scan(ctx, *d, nullptr, dt, ds, &b);
  if (r == EPIK2_OK) {
    e = cudaSuccess;
    if (tables) e = cudaMemcpy(tables, dt, (size_t)T * 54 * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && scores) e = cudaMemcpy(scores, ds, (size_t)T * 4, cudaMemcpyDeviceToHost);
    ctx->stats.d2h_bytes += (tables ? (uint64_t)T * 54 * 4 : 0) + (scores ? (uint64_t)T * 4 : 0);
    if (e != cudaSuccess) r = cuda_fail(ctx, e, "read dump");
  }
  cudaFree(dt);
  cudaFree(ds);
  return r;
}

int epik2_tables(epik2_ctx* ctx, int32_t dataset_id, const uint32_t* triplets, int64_t n, uint32_t* tables) {
  if (!ctx) return EPIK2_E_INVALID;
  DevDataset* d = find(ctx, dataset_id);
  if (!d) return fail(ctx, EPIK2_E_NOT_FOUND, "unknown dataset");
  if (n < 0 || (n > 0 && (!triplets || !tables))) return fail(ctx, EPIK2_E_INVALID, "bad triplet list");
  if (n == 0) return EPIK2_OK;
  for (int64_t t = 0; t < n; t++) {
    const uint32_t i = triplets[3 * t], j = triplets[3 * t + 1], k = triplets[3 * t + 2];
    if (!(i < j && j < k && (int64_t)k < d->n_snps)) return fail(ctx, EPIK2_E_INVALID, "triplet out of range");
  }
  CK(ctx, cudaSetDevice(ctx->device), "set device");
  uint32_t *dtrip = nullptr, *dout = nullptr;
  CK(ctx, cudaMalloc(&dtrip, (size_t)n * 12), "alloc triplets");
  cudaError_t e = cudaMalloc(&dout, (size_t)n * 54 * 4);
  if (e == cudaSuccess) e = cudaMemcpy(dtrip, triplets, (size_t)n * 12, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = launch_tables(*d, dtrip, n, dout, ctx->stream);
  ctx->stats.kernel_launches += 1;
  ctx->stats.h2d_bytes += (uint64_t)n * 12;
  ctx->stats.d2h_bytes += (uint64_t)n * 54 * 4;
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpy(tables, dout, (size_t)n * 54 * 4, cudaMemcpyDeviceToHost);
  cudaFree(dtrip);
  cudaFree(dout);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tables");
  return EPIK2_OK;
}

int epik2_k2_lut(int64_t n_max, float* lut) {
  if (n_max < 0 || !lut) return EPIK2_E_INVALID;
  build_k2_lut(n_max, lut);
  return EPIK2_OK;
}

}  // extern "C"
