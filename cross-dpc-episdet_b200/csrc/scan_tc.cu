// Tensor-core engine of the triplet search (tcgen05, sm_100a): kind::i8 and block-scaled
// kind::mxf4 (FP4), single CTAs or CTA pairs (cta_group::2).
//
// Same result as the integer engine (scan_int.cu) and as the reference's kernel_epi
// (GPU/v4.cpp:295-594): the 8 cells of each triplet with g_i, g_j, g_k in {0,1} are
// counted exactly, the other 19 per class follow by inclusion-exclusion, K2 is scored in
// the reference's FP32 order, and the lowest (score, i, j, k) wins.
//
// Counting as a matrix product.  For a fixed SNP i, a block of 32 SNPs j and a block of kK
// SNPs k (128 in the int8 format, 112 in FP4), with 0/1 indicators x_{s,g}(snp) =
// [genotype of snp in sample s is g]:
//     D[(j, a, b)][(k, c)] = sum over samples s of class C of
//                            x_{s,a}(i) * x_{s,b}(j)  *  x_{s,c}(k)
//                          = count of (g_i=a, g_j=b, g_k=c) in class C.
// A (128 x S_C) holds the pair indicators of the 32 pairs (i, j) x (a, b), B (2kK x S_C)
// the single indicators of the kK SNPs k x c; both are expanded from the bit planes (int8
// 0 or -1; E2M1 0 or 0.5 with scale factors 2), 32*kW samples per pipeline stage, straight
// into shared memory in the no-swizzle K-major layout the tensor core reads (8-row x
// 16-byte core matrices; K-neighbours 128 B apart).  Warp roles: 16 warps expand operands
// (and later run the epilogue); one more warp only issues tcgen05.mma (int8: M=128, N=256,
// K=32, int32 accumulators; FP4: N=224, K=64, FP32 accumulators exact below 2^24; class 0
// and class 1 into separate halves of tensor memory).  An MMA issue blocks its thread for
// about the MMA's execution time, so the issuing thread does nothing else.  Hand-off per
// stage: each producing warp fences its stores for the async proxy and arrives once on the
// stage's "full" mbarrier; the issuer waits on it, issues the stage's MMAs and commits them
// to the stage's "empty" mbarrier, which the producers wait on before refilling the slot
// (and, at the end of a tile, to the accumulator barrier).  CTA pairs compute 64 pairs j at
// once (M=256), each CTA expanding half of A and half of B.  The epilogue moves the
// accumulators TMEM -> registers -> shared memory and completes, scores and selects the
// triplets of the tile, with the ln n! table copied into the then idle stage ring.
//
// Every wait on an mbarrier is bounded (about 2 s of SM clock); on expiry the kernel sets
// an error word, stops taking tiles, frees its tensor memory and returns.
#include <algorithm>
#include <cfloat>

#include "epik2_internal.h"
#include "scan_common.cuh"
#include "tc_ptx.cuh"

namespace epik2 {

constexpr int kTcThreads = 512;  // 16 operand-producing / epilogue warps
constexpr int kTcWarps = kTcThreads / 32;
constexpr int kTcThreadsAll = kTcThreads + 32;  // + one warp that only issues the MMAs
constexpr int kRingBytes = 16 * 384 * 32;  // stage ring: kStages x 384 rows x (32 * kW) bytes = 192 KiB
constexpr int kTcSmemBytes = 230400;        // ring (or epilogue staging + ln n! table), mbarriers at the end
constexpr int kBarOff = kTcSmemBytes - 256;
constexpr int kEStride = 132;  // words per row of the epilogue staging buffer (16-byte rows: 128-bit stores)
// During a tile's epilogue the ring is idle: it holds the staging buffer E (2 classes x 128
// rows x kEStride words) and, behind it, a copy of the dataset's ln n! table when the table
// has at most kLutCapacity entries (samples + 2; larger tables are read from global memory).
constexpr int kLutOff = 2 * 128 * kEStride * 4;
constexpr int kLutCapacity = (kBarOff - kLutOff) / 4;
static_assert(kRingBytes <= kBarOff && kLutOff % 16 == 0, "shared-memory layout");

// One dataset's view for a tile: the plain search has one, the batched search reads the
// tile's dataset from the job table.
struct JobView {
  const uint2* planes;
  const uint32_t* singles;
  const uint4* pairs;
  const float* lut;
  int64_t tri;
  int32_t m, m_pad, w0, w1, n0, n1;
};

// kFp4 selects the operand format: int8 (kind::i8, 128 SNPs k per tile, kW = 4 or 8 words
// per stage: 4 stages of 48 KiB or 2 of 96 KiB) or E2M1 (kind::mxf4, 112 SNPs k per tile so
// that the scale factors fit in tensor memory beside the two accumulators, kW = 8 or 16:
// 4 stages of 44 KiB or 2 of 88 KiB).  kW = class words (32 samples each) per stage.
// kPair (FP4 only): a cluster of two CTAs computes one tile of 64 pairs (M = 256,
// cta_group::2): CTA r holds the A rows of pairs j0+32r.. and the B rows of SNPs
// k0+56r..k0+56r+55 (both values of g_k), so each CTA expands 128 + 112 operand rows per
// stage instead of 128 + 224; D column 112h + 56c + kp is SNP k0 + 56h + kp, g_k = c.
// The even CTA issues.
// kBatched: tiles of many datasets on one queue, per-dataset results.
// kMarg (CTA pairs only): the pair-margin form.  Operand A's g_i = 0 rows are all ones and
// its g_i = 1 rows zero, so D[(j, 0, b)][(k, c)] is the count of (g_j = b, g_k = c): tiles
// (0, j0, k block) write the pair margins of every j < k < m_pad instead of scoring.
// kRepl (CTA pairs, 16 words per stage): the replicate form.  The tile's passes share one
// pair operand expansion scheme and the tensor memory: pass 0 counts all samples of the base
// dataset (its two classes' words as one range) into the class-0 accumulators, where they stay;
// pass r = 1..p.n_reps counts the cases of replicate r (p.jobs[r-1]) into the class-1
// accumulators and scores replicate r with controls = totals - cases, its best folded into
// p.job_slots[r-1].  Permutation replicates of one matrix thus share the all-sample counts.
template <int kW, bool kFp4, bool kPair, bool kBatched, bool kDump, bool kTopK, bool kMarg = false,
          bool kRepl = false>
__global__ void __launch_bounds__(kTcThreadsAll, 1) k_scan_tc(const TcParams p) {
  static_assert(!kPair || kFp4, "CTA pairs use the FP4 format");
  static_assert(!kMarg || (kPair && !kBatched && !kDump && !kTopK), "pair margins: plain CTA-pair kernel");
  static_assert(!kRepl || (kPair && kW == 16 && !kBatched && !kDump && !kTopK && !kMarg), "replicates: CTA pairs");
  constexpr int kK = kFp4 ? 112 : 128;                // SNPs k per tile -> 2*kK rows of B
  constexpr int kRowBytes = (kFp4 ? 16 : 32) * kW;    // operand bytes per row per stage
  constexpr int kBRows = kPair ? kK : 2 * kK;         // B rows held by this CTA
  constexpr int kStageA = 128 * kRowBytes;
  constexpr int kStageBytes = (128 + kBRows) * kRowBytes;
  constexpr int kStages = (kRingBytes / kStageBytes) < 4 ? (kRingBytes / kStageBytes) : 4;
  constexpr uint32_t kSbo = 8 * kRowBytes;            // bytes between 8-row groups
  constexpr int kMmas = kFp4 ? kW / 2 : kW;           // MMAs per stage (K = 64 E2M1 or 32 int8)
  constexpr int kU = kW / 4;                          // units of each kind per thread per stage
  constexpr int kUB = kPair ? kW / 8 : kU;            // 8-byte B plane loads per thread per stage
  static_assert(kStages >= 2 && kStages <= 4, "stage ring");
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint32_t s_tmem;
  __shared__ long long s_tile;
  __shared__ int s_abort;
  __shared__ float s_red_s[kTcWarps];
  __shared__ unsigned long long s_red_k[kTcWarps];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kBarOff);  // [stages] empty + acc
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t stage0 = smem_u32(smem);
  const uint32_t bar0 = smem_u32(bars);
  const uint32_t bar_acc = bar0 + 8 * kStages;
  const uint32_t bar_full0 = bar_acc + 8;  // [stages]: one arrival per producing warp (+1 forwarded)
  const uint32_t bar_tile = bar_full0 + 8 * kStages;  // CTA pairs: the odd CTA's "next tile is set"
  const uint32_t bar_final = bar_tile + 8;  // the issuer's last commit: every product has completed
  volatile int* abort_flag = &s_abort;
  const bool worker = warp < kTcWarps;
  const long long wl = p.wait_limit > 0 ? p.wait_limit : kWaitLimit;  // clocks a bounded wait lasts
  // test hook (single CTAs only): warp 0 of CTA 0 leaves out its "stage stored" arrival of
  // the first stage, so the issuing warp's wait on that stage expires and the kernel takes
  // its error exit before any MMA was issued
  const bool hold_first = !kPair && p.test_withhold != 0 && blockIdx.x == 0 && warp == 0;
  const uint32_t crank = kPair ? cluster_rank() : 0u;  // rank in the CTA pair
  const bool issuer_cta = crank == 0;

  if (tid == 0) {
    for (int s = 0; s < kStages; s++) bar_init(bar0 + 8 * s, 1);
    bar_init(bar_acc, 1);
    // full: the CTA's producing warps, and in a pair's issuing CTA one forwarded arrival
    for (int s = 0; s < kStages; s++) bar_init(bar_full0 + 8 * s, kTcWarps + ((kPair && crank == 0) ? 1 : 0));
    bar_init(bar_tile, 1);
    bar_init(bar_final, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
  }
  if (kPair) cluster_sync_all();  // the pair's barriers are initialised before any remote arrival
  if (warp == 0) {
    if (kPair) {
      asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                   "r"(512u)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    } else {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                   "r"(512u)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  if (kFp4) {  // scale factors: every byte of columns [224, 256) = 0x80 (2^1), all 128 lanes
    if (warp < 4) {
      const uint32_t ta = tmem + ((uint32_t)(32 * warp) << 16) + kSfaCol;
      tmem_st16_fill(ta, 0x80808080u);
      tmem_st16_fill(ta + 16, 0x80808080u);
      tmem_wait_st();
    }
    tc_fence_before();
    __syncthreads();
    if (kPair) cluster_sync_all();  // both CTAs' scale factors are in place before the first MMA
    tc_fence_after();
  }

  float best_s = FLT_MAX;
  unsigned long long best_k = ~0ull;
  float list_s = FLT_MAX;
  unsigned long long list_k = ~0ull;
  uint32_t g_chunk = 0, n_tile = 0, n_fetch = 0;
  unsigned long long pf_t = 0;  // thread 0: ticket and descriptor of the next tile
  long long pf_d = -1;
  const uint32_t* E = reinterpret_cast<const uint32_t*>(smem);  // epilogue staging, reuses the stages

  // Batched form: fold the CTA's candidates for dataset jb into its slot of that dataset.
  // Called by every thread when the dataset of the next tile differs (the queue holds each
  // dataset's tiles together, so this happens about once per dataset and CTA).
  auto flush_job = [&](int jb) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const float os = __shfl_xor_sync(kFull, best_s, off);
      const unsigned long long ok = __shfl_xor_sync(kFull, best_k, off);
      if (better(os, ok, best_s, best_k)) {
        best_s = os;
        best_k = ok;
      }
    }
    if (lane == 0 && worker) {
      s_red_s[warp] = best_s;
      s_red_k[warp] = best_k;
    }
    __syncthreads();
    if (tid == 0) {
      float bs = s_red_s[0];
      unsigned long long bk = s_red_k[0];
      for (int w = 1; w < kTcWarps; w++)
        if (better(s_red_s[w], s_red_k[w], bs, bk)) {
          bs = s_red_s[w];
          bk = s_red_k[w];
        }
      BestSlot& slot = p.job_slots[(int64_t)jb * gridDim.x + blockIdx.x];
      if (better(bs, bk, slot.score, slot.key)) {
        slot.score = bs;
        slot.key = bk;
      }
    }
    __syncthreads();
    best_s = FLT_MAX;
    best_k = ~0ull;
  };
  int cur_job = -1;

  for (;;) {
    // next tile from the shared queue; its descriptor (one 8-byte load) gives the dataset,
    // the first index, the pair block and the k block.  Thread 0 takes the ticket and the
    // descriptor of the tile after it right away, so their latency overlaps this tile.
    if (tid == 0) {
      if (issuer_cta) {
        if (n_fetch == 0) {
          pf_t = atomicAdd(p.counter, 1ull);
          pf_d = pf_t < (unsigned long long)p.n_tiles ? (long long)__ldg(p.tiles + pf_t) : -1ll;
        }
        const long long d = s_abort ? -1ll : pf_d;
        if (d >= 0) {
          pf_t = atomicAdd(p.counter, 1ull);
          pf_d = pf_t < (unsigned long long)p.n_tiles ? (long long)__ldg(p.tiles + pf_t) : -1ll;
        }
        s_tile = d;
        if (kPair) {  // hand the tile to the odd CTA: store, then release-arrive on its barrier
          st_cluster_s64(map_cta(smem_u32(&s_tile), 1), d);
          bar_arrive_cluster(map_cta(bar_tile, 1));
        }
      } else if (!bar_wait_cluster(bar_tile, n_fetch & 1u, wl)) {
        s_abort = 1;
        s_tile = -1;
      }
    }
    ++n_fetch;
    __syncthreads();
    const long long desc = s_tile;
    if (kBatched) {  // desc is the same for every thread: the flush is uniform
      const int next_job = desc < 0 ? -1 : tile_job(desc);
      if (next_job != cur_job) {
        if (cur_job >= 0) flush_job(cur_job);
        cur_job = next_job;
      }
    }
    if (desc < 0) break;
    // this CTA's pairs: j0 .. j0+31 (pairs of a CTA pair: 32*rank further)
    const int i = tile_i(desc), j0 = tile_j0(desc) + 32 * (int)crank, k0 = tile_k0(desc, kK);
    const int job = kBatched ? tile_job(desc) : 0;
    JobView jv;
    if (kBatched) {
      const TcJob& J = p.jobs[job];
      jv = JobView{J.planes, J.singles, J.pairs, J.lut, J.tri, J.m, J.m_pad, J.w0, J.w1, J.n0, J.n1};
    } else {
      jv = JobView{p.planes, p.singles, p.pairs, p.lut, p.tri, p.m, p.m_pad, p.w0, p.w1, p.n0, p.n1};
    }
    const int n_pass = kRepl ? 1 + p.n_reps : 1;
    for (int pass = 0; pass < n_pass; pass++) {
    if (kRepl && pass > 0) {  // replicate `pass`: its planes, class split, margins and table
      const TcJob& R = p.jobs[pass - 1];
      jv = JobView{R.planes, R.singles, R.pairs, R.lut, R.tri, R.m, R.m_pad, R.w0, R.w1, R.n0, R.n1};
    }
    const int64_t m_pad = jv.m_pad;
    const int m = jv.m;
    // words counted into class 0 and class 1 in this pass (class-1 words start at jv.w0)
    const int lim0 = kRepl ? (pass == 0 ? jv.w0 + jv.w1 : 0) : jv.w0;
    const int lim1 = kRepl ? (pass == 0 ? 0 : jv.w1) : jv.w1;
    const int nc0 = (lim0 + kW - 1) / kW, nc1 = (lim1 + kW - 1) / kW, nct = nc0 + nc1;

    // ---- operand expansion and MMA, 32*kW samples per stage ----
    // Work of a stage per thread:
    //   A: pair q = lane, word wA = warp % kW: loads the i and j words once and writes rows
    //      32*ab + q (g_i = ab>>1, g_j = ab&1) for kAb = kW/4 consecutive ab
    //   B: words w = (tid>>7) + 4r (r < kU), kl = tid&127 (< kK) -> rows kK*c + kl (g_k = c)
    //      of both c; CTA pairs: words w = (tid>>6) + 8r (r < kW/8), kp = tid&63 (< kK/2) ->
    //      rows (kK/2)*c + kp for SNP k0 + (kK/2)*rank + kp (one 8-byte load gives both c)
    // A warp writes 32 consecutive rows of one 16-byte K group per store (conflict-free).
    // The words of stage cc+1 are loaded while stage cc is expanded.
    constexpr int kAb = kW / 4;
    const int wA = warp % kW, ab0 = (warp / kW) * kAb, w_base = tid >> 7;
    const int a_j = min(j0 + lane, (int)m_pad - 1);
    const int b_kl = tid & 127;
    const bool b_on = b_kl < kK;
    const int b_k = k0 + b_kl;
    const uint32_t offb0 = (b_kl >> 3) * kSbo + (b_kl & 7) * 16;  // + (kK/8)*kSbo for c = 1
    // CTA pairs: B rows (kK/2)*c + kp of this CTA hold SNP k0 + (kK/2)*rank + kp, kp < kK/2
    const int p_kl = tid & 63;
    const bool p_on = p_kl < kK / 2;
    const int p_k = k0 + (kK / 2) * (int)crank + p_kl;
    const uint32_t offp0 = (p_kl >> 3) * kSbo + (p_kl & 7) * 16;  // + (kK/16)*kSbo for c = 1
    const int p_wbase = tid >> 6;  // words p_wbase + 8r, r < kW/8
    auto load_words = [&](int cc, uint2& gi, uint2& gj, uint2 (&gk)[kUB]) {
      const bool c1 = cc >= nc0;
      const int c_in = c1 ? cc - nc0 : cc;
      const int wcls = c1 ? lim1 : lim0;
      const int64_t wb = (c1 ? (int64_t)jv.w0 : 0) + (int64_t)kW * c_in;
      gi = make_uint2(0, 0);
      gj = gi;
      if (kW * c_in + wA < wcls) {
        const uint2* row = jv.planes + (wb + wA) * m_pad;
        gi = kMarg ? make_uint2(~0u, 0u) : __ldg(row + i);
        gj = __ldg(row + a_j);
      }
#pragma unroll
      for (int r = 0; r < kUB; r++) gk[r] = make_uint2(0, 0);
      if constexpr (kPair) {
#pragma unroll
        for (int r = 0; r < kW / 8; r++) {
          const int w = p_wbase + 8 * r;
          if (kW * c_in + w < wcls && p_on && p_k < m_pad) gk[r] = __ldg(jv.planes + (wb + w) * m_pad + p_k);
        }
      } else {
#pragma unroll
        for (int r = 0; r < kU; r++) {
          const int w = w_base + 4 * r;
          if (kW * c_in + w < wcls && b_on && b_k < m_pad) gk[r] = __ldg(jv.planes + (wb + w) * m_pad + b_k);
        }
      }
    };
    if (worker) {
      uint2 ci, cj, ck[kUB];
      if (nct > 0) load_words(0, ci, cj, ck);
      for (int cc = 0; cc < nct; ++cc) {
        const uint32_t g = g_chunk + (uint32_t)cc;
        uint2 ni = make_uint2(0, 0), nj = ni, nk[kUB];
#pragma unroll
        for (int r = 0; r < kUB; r++) nk[r] = make_uint2(0, 0);
        if (cc + 1 < nct) load_words(cc + 1, ni, nj, nk);
        const int s = (int)(g % kStages);
        const uint32_t use = g / kStages;
        const bool late =
            use > 0 && !(kPair ? bar_wait_cluster(bar0 + 8 * s, (use & 1u) ^ 1u, wl) : bar_wait(bar0 + 8 * s, (use & 1u) ^ 1u, wl));
        if (__any_sync(kFull, late)) *abort_flag = 1;
        if (__shfl_sync(kFull, *abort_flag, 0)) break;  // warp-uniform
        const uint32_t sA = stage0 + s * kStageBytes, sB = sA + kStageA;
#pragma unroll
        for (int t = 0; t < kAb; t++) {
          const int ab = ab0 + t, row = 32 * ab + lane;
          const uint32_t wa = ((ab >> 1) ? ci.y : ci.x) & ((ab & 1) ? cj.y : cj.x);
          const uint32_t offa = sA + (row >> 3) * kSbo + (row & 7) * 16;
          if (kFp4) {
            sts128(offa + wA * 128, expand32_fp4(wa));
          } else {
            sts128(offa + (2 * wA) * 128, expand16(wa));
            sts128(offa + (2 * wA) * 128 + 128, expand16(wa >> 16));
          }
        }
        if constexpr (kPair) {
#pragma unroll
          for (int r = 0; r < kW / 8; r++) {
            const int w = p_wbase + 8 * r;
            if (p_on) {
              const uint32_t offb = sB + offp0 + w * 128;
              sts128(offb, expand32_fp4(ck[r].x));
              sts128(offb + (kK / 16) * kSbo, expand32_fp4(ck[r].y));
            }
          }
        } else {
#pragma unroll
          for (int r = 0; r < kU; r++) {
            const int w = w_base + 4 * r;
            if (kFp4) {
              if (b_on) {
                const uint32_t offb = sB + offb0 + w * 128;
                sts128(offb, expand32_fp4(ck[r].x));
                sts128(offb + (kK / 8) * kSbo, expand32_fp4(ck[r].y));
              }
            } else {
              const uint32_t offb = sB + offb0 + (2 * w) * 128;
              sts128(offb, expand16(ck[r].x));
              sts128(offb + 128, expand16(ck[r].x >> 16));
              sts128(offb + (kK / 8) * kSbo, expand16(ck[r].y));
              sts128(offb + (kK / 8) * kSbo + 128, expand16(ck[r].y >> 16));
            }
          }
        }
        ci = ni;
        cj = nj;
#pragma unroll
        for (int r = 0; r < kUB; r++) ck[r] = nk[r];
        fence_proxy_async();
        __syncwarp();
        if (lane == 0 && !(hold_first && g == 0)) bar_arrive(bar_full0 + 8 * s);
      }
    } else if (kPair && lane == 0 && !issuer_cta) {
      // the odd CTA of a pair forwards "stage stored" to the issuing CTA: one cluster-scope
      // arrival per stage once all its producing warps have arrived locally
      for (int cc = 0; cc < nct; ++cc) {
        const uint32_t g = g_chunk + (uint32_t)cc;
        const int s = (int)(g % kStages);
        if (!bar_wait(bar_full0 + 8 * s, (g / kStages) & 1u, wl)) {
          *abort_flag = 1;
          break;
        }
        bar_arrive_cluster(map_cta(bar_full0 + 8 * s, 0));
      }
    } else if (lane == 0 && issuer_cta) {
      // the issuing warp: wait for each stage's operands, issue its MMAs, release it
      for (int cc = 0; cc < nct; ++cc) {
        const uint32_t g = g_chunk + (uint32_t)cc;
        const int s = (int)(g % kStages);
        const uint32_t use = g / kStages;
        if (!(kPair ? bar_wait_cluster(bar_full0 + 8 * s, use & 1u, wl) : bar_wait(bar_full0 + 8 * s, use & 1u, wl))) {
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        const bool c1 = cc >= nc0;
        const int c_in = c1 ? cc - nc0 : cc;
        const uint32_t sA = stage0 + s * kStageBytes, sB = sA + kStageA;
        const uint32_t d = tmem + (c1 ? 256u : 0u);
        const uint64_t da = smem_desc(sA, kSbo), db = smem_desc(sB, kSbo);
#pragma unroll
        for (int kk = 0; kk < kMmas; kk++) {  // each MMA reads 32 bytes of every row: 256 B on
          const uint32_t acc = (c_in > 0 || kk > 0) ? 1u : 0u;
          if (kPair)
            mma_fp4_pair(d, da + (uint64_t)(16 * kk), db + (uint64_t)(16 * kk), acc, tmem + kSfaCol, tmem + kSfbCol);
          else if (kFp4)
            mma_fp4(d, da + (uint64_t)(16 * kk), db + (uint64_t)(16 * kk), acc, tmem + kSfaCol, tmem + kSfbCol);
          else
            mma_i8(d, da + (uint64_t)(16 * kk), db + (uint64_t)(16 * kk), acc);
        }
        if (kPair) {
          mma_commit_pair(bar0 + 8 * s);
          if (cc == nct - 1 && !(kRepl && pass == 0)) mma_commit_pair(bar_acc);  // pass 0 is not scored
        } else {
          mma_commit(bar0 + 8 * s);
          if (cc == nct - 1) mma_commit(bar_acc);
        }
      }
      // a replicate without cases has no products of its own: the accumulator barrier still
      // completes, once the totals of pass 0 are in
      if (kRepl && pass > 0 && nct == 0 && !*abort_flag) mma_commit_pair(bar_acc);
    }
    g_chunk += (uint32_t)nct;
    __syncwarp();
    __syncthreads();  // every thread has left the stage loop (done, or an expired wait)
    if (*abort_flag) break;
    if (kRepl && pass == 0) continue;  // the totals stay in tensor memory for the replicates

    // ---- epilogue: TMEM -> shared -> complete tables, score, select ----
    {
      const bool ok = kPair ? bar_wait_cluster(bar_acc, n_tile & 1u, wl) : bar_wait(bar_acc, n_tile & 1u, wl);
      if (!ok) *abort_flag = 1;
      __syncthreads();
      if (*abort_flag) break;
    }
    tc_fence_after();
    ++n_tile;
    // Accumulator layout: TMEM lane = 32*ab + q, column = kK*c + kl (per class: +256*cls).
    // Per half h (kl in [64h, min(64h+64, kK))) each warp copies lanes 32*(warp&3).. and up
    // to 32 columns of both c into E[cls][lane][64*c + kl - 64h] (row stride kEStride
    // words); FP32 accumulators (FP4 format) are converted to the integer counts they hold.
    const int quarter = warp & 3, cgrp = warp >> 2;
    const int row = 32 * quarter + lane;
    const int e_c = cgrp >> 1, e_sub = cgrp & 1;
    const int64_t tri = jv.tri;
    const uint2 si0 = *reinterpret_cast<const uint2*>(jv.singles + ((int64_t)i) * 2);
    const uint2 si1 = *reinterpret_cast<const uint2*>(jv.singles + (m_pad + i) * 2);
    // ln n! table into the idle ring (in flight during the accumulator copy below); the
    // device table is padded to 256 bytes, so whole 16-byte pieces stay inside it
    const float* lut_s = reinterpret_cast<const float*>(smem + kLutOff);
    const bool lut_shared = jv.n0 + jv.n1 + 2 <= kLutCapacity;
    if (!kMarg && lut_shared && worker) {
      const int n16 = (jv.n0 + jv.n1 + 2 + 3) / 4;
      for (int x = tid; x < n16; x += kTcThreads) cp_async16(stage0 + kLutOff + 16 * x, jv.lut + 4 * x);
    }
    for (int h = 0; h < 2; h++) {
      if (kPair) {
        // CTA pairs: columns 112h + 56c + kp (kp < 56) hold SNP k0 + 56h + kp, g_k = c; they
        // go to E[cls][lane][56c + kp], 7 groups of 16 columns per class and lane quarter
#pragma unroll
        for (int cls = 0; cls < 2; cls++) {
          const bool has = (cls ? nc1 > 0 : (kRepl || nc0 > 0)) && worker;
#pragma unroll
          for (int t = 0; t < 2; t++) {
            const int u = cgrp + 4 * t;  // warp-uniform
            if (u < 7 && worker) {
              uint32_t v[16];
              if (has) {
                tmem_ld16(tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(cls * 256 + 112 * h + 16 * u), v);
                tmem_wait_ld();
#pragma unroll
                for (int t2 = 0; t2 < 16; t2++) v[t2] = __float2uint_rn(__uint_as_float(v[t2]));
              } else {
#pragma unroll
                for (int t2 = 0; t2 < 16; t2++) v[t2] = 0;
              }
              const uint32_t dst = stage0 + 4 * ((cls * 128 + row) * kEStride + 16 * u);
#pragma unroll
              for (int t2 = 0; t2 < 4; t2++) sts128(dst + 16 * t2, make_uint4(v[4 * t2], v[4 * t2 + 1], v[4 * t2 + 2], v[4 * t2 + 3]));
            }
          }
        }
      }
#pragma unroll
      for (int cls = 0; cls < (kPair ? 0 : 2); cls++) {  // single CTAs: columns kK*c + kl
        const bool has = (cls ? nc1 > 0 : nc0 > 0) && worker;
#pragma unroll
        for (int part = 0; part < 2; part++) {
          const int kin = 64 * h + 32 * e_sub + 16 * part;  // first k of the 16 columns
          const int col = kK * e_c + kin;                     // inside the class accumulator
          uint32_t v[16];
          if (has && kin < kK) {  // warp-uniform
            tmem_ld16(tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(cls * 256 + col), v);
            tmem_wait_ld();
            if (kFp4) {
#pragma unroll
              for (int t = 0; t < 16; t++) v[t] = __float2uint_rn(__uint_as_float(v[t]));
            }
          } else {
#pragma unroll
            for (int t = 0; t < 16; t++) v[t] = 0;
          }
          const uint32_t dst = stage0 + 4 * ((cls * 128 + row) * kEStride + 64 * e_c + 32 * e_sub + 16 * part);
          if (worker) {
#pragma unroll
            for (int t = 0; t < 4; t++) sts128(dst + 16 * t, make_uint4(v[4 * t], v[4 * t + 1], v[4 * t + 2], v[4 * t + 3]));
          }
        }
      }
      cp_async_wait_all();
      tc_fence_before();
      __syncthreads();
      // 32 pairs x nk k of this half (nk = 64, or 48 in the FP4 tile's second half; 56 in
      // both halves of a CTA pair's tile): triplet x = tid + 512u -> kl = x % nk, q = x / nk
      const int nk = kPair ? kK / 2 : ((64 * h + 64 <= kK) ? 64 : kK - 64 * h);
      const int kbase = kPair ? (kK / 2) * h : 64 * h;
      constexpr int kEc = kPair ? kK / 2 : 64;  // staging column of (c, kl): kEc * c + kl
      if constexpr (kMarg) {
        // pair margins (n00, n01, n10, n11) of (j, k): staging rows ab = g_j (g_i = 0), c = g_k
#pragma unroll 1
        for (int u = 0; u < (worker ? (32 * nk + kTcThreads - 1) / kTcThreads : 0); u++) {
          const int x = tid + kTcThreads * u;
          const int q = x / nk, kl = x - q * nk;
          const int j = j0 + q, k = k0 + kbase + kl;
          if (q < 32 && j < k && k < m_pad) {
            const int64_t o = tri_offset(m_pad, j, k);
#pragma unroll
            for (int cls = 0; cls < 2; cls++) {
              const uint32_t* Er = E + (cls * 128 + q) * kEStride + kl;
              p.pairs_out[cls * tri + o] = make_uint4(Er[0], Er[kEc], Er[32 * kEStride], Er[32 * kEStride + kEc]);
            }
          }
        }
      }
#pragma unroll 1
      for (int u = 0; u < (worker && !kMarg ? (32 * nk + kTcThreads - 1) / kTcThreads : 0); u++) {
        const int x = tid + kTcThreads * u;
        const int q = x / nk, kl = x - q * nk;
        const int j = j0 + q;
        const int k = k0 + kbase + kl;
        const bool valid = (q < 32) && (j < m) && (k > j) && (k < m);
        float sc = FLT_MAX;
        unsigned long long key = ~0ull;
        if (valid) {
          uint32_t t80[8], t81[8];
#pragma unroll
          for (int ab = 0; ab < 4; ab++)
#pragma unroll
            for (int c = 0; c < 2; c++) {
              t80[2 * ab + c] = E[(0 * 128 + 32 * ab + q) * kEStride + kEc * c + kl];
              t81[2 * ab + c] = E[(1 * 128 + 32 * ab + q) * kEStride + kEc * c + kl];
            }
          if (kRepl) {  // class 0 holds all samples: the replicate's controls are the rest
#pragma unroll
            for (int x = 0; x < 8; x++) t80[x] -= t81[x];
          }
          const uint2 sj0 = *reinterpret_cast<const uint2*>(jv.singles + ((int64_t)j) * 2);
          const uint2 sj1 = *reinterpret_cast<const uint2*>(jv.singles + (m_pad + j) * 2);
          const uint2 sk0 = *reinterpret_cast<const uint2*>(jv.singles + ((int64_t)k) * 2);
          const uint2 sk1 = *reinterpret_cast<const uint2*>(jv.singles + (m_pad + k) * 2);
          const int64_t oij = tri_offset(m_pad, i, j), oik = tri_offset(m_pad, i, k), ojk = tri_offset(m_pad, j, k);
          const uint4 pij0 = __ldg(jv.pairs + oij), pij1 = __ldg(jv.pairs + tri + oij);
          const uint4 pik0 = __ldg(jv.pairs + oik), pik1 = __ldg(jv.pairs + tri + oik);
          const uint4 pjk0 = __ldg(jv.pairs + ojk), pjk1 = __ldg(jv.pairs + tri + ojk);
          uint32_t T0[27], T1[27];
          complete_table(t80, (uint32_t)jv.n0, si0, sj0, sk0, pij0, pik0, pjk0, T0);
          complete_table(t81, (uint32_t)jv.n1, si1, sj1, sk1, pij1, pik1, pjk1, T1);
          sc = lut_shared ? k2_score_shared(T0, T1, lut_s) : k2_score(T0, T1, jv.lut);
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
          const float ts = __shfl_sync(kFull, list_s, 31);
          const unsigned long long tk = __shfl_sync(kFull, list_k, 31);
          unsigned want = __ballot_sync(kFull, valid && better(sc, key, ts, tk));
          while (want) {
            const int src = __ffs(want) - 1;
            want &= want - 1;
            const float cs = __shfl_sync(kFull, sc, src);
            const unsigned long long ck2 = __shfl_sync(kFull, key, src);
            const float ts2 = __shfl_sync(kFull, list_s, 31);
            const unsigned long long tk2 = __shfl_sync(kFull, list_k, 31);
            if (better(cs, ck2, ts2, tk2)) warp_list_insert(list_s, list_k, cs, ck2, lane);
          }
        }
      }
      __syncthreads();  // the staging buffer is rewritten by the next half / next tile
    }
    if (kRepl) flush_job(pass - 1);  // replicate `pass`'s best of this tile into its slot
    }  // passes
    if (*abort_flag) break;
  }

  // ---- teardown ----
  // Tensor memory is released only after every product has completed.  A search that ran to
  // its end waited for each tile's products already; after an expired wait the issuer may
  // have left its last stages running.  So the issuing thread commits once more and that
  // commit is waited for (bounded) in each CTA it arrives in.
  if (!worker && lane == 0) {
    if (issuer_cta) {
      if (kPair) mma_commit_pair(bar_final);
      else mma_commit(bar_final);
    }
    if (!(kPair ? bar_wait_cluster(bar_final, 0, wl) : bar_wait(bar_final, 0, wl))) *abort_flag = 1;
  }
  tc_fence_before();
  __syncthreads();
  if (s_abort && tid == 0) atomicExch(p.err, 1);
  if (kPair) cluster_sync_all();  // the pair's MMAs and remote arrivals are over
  if (warp == 0) {
    tc_fence_after();
    if (kPair)
      asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
    else
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
  }
  if (!kBatched && !kRepl && worker) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const float os = __shfl_xor_sync(kFull, best_s, off);
      const unsigned long long ok = __shfl_xor_sync(kFull, best_k, off);
      if (better(os, ok, best_s, best_k)) {
        best_s = os;
        best_k = ok;
      }
    }
    const int64_t gwarp = (int64_t)blockIdx.x * kTcWarps + warp;
    if (lane == 0) {
      p.slots[gwarp].score = best_s;
      p.slots[gwarp].key = best_k;
    }
    if (kTopK) {
      p.cand[gwarp * 32 + lane].score = list_s;
      p.cand[gwarp * 32 + lane].key = list_k;
    }
  }
}

// Tile descriptors of one pair-block list: pair block b = (i, j0) holds the tiles
// [pb_off[b], pb_off[b+1]) with k blocks t = 0, 1, ... (k from j0 + 1 + kK*t); one thread
// per pair block writes them to out[pb_off[b] ...].
__global__ void k_expand_tiles(const int64_t* __restrict__ pb_off, const uint32_t* __restrict__ pb_ij, int64_t n_pb,
                               int kK, int job, uint64_t* __restrict__ out) {
  (void)kK;
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n_pb) return;
  const uint32_t i = pb_ij[2 * b], j0 = pb_ij[2 * b + 1];
  const int64_t t0 = pb_off[b], n = pb_off[b + 1] - t0;
  for (int64_t t = 0; t < n; t++) out[t0 + t] = pack_tile(i, j0, (uint32_t)t, (uint32_t)job);
}

cudaError_t launch_expand_tiles(const int64_t* pb_off, const uint32_t* pb_ij, int64_t n_pb, bool fp4, int job,
                                uint64_t* out, cudaStream_t stream) {
  if (n_pb <= 0) return cudaSuccess;
  k_expand_tiles<<<(unsigned)((n_pb + 255) / 256), 256, 0, stream>>>(pb_off, pb_ij, n_pb, tc_k_per_tile(fp4), job,
                                                                     out);
  return cudaGetLastError();
}

// Per-dataset reduction of the batched search's per-CTA slots: block b reduces dataset b.
__global__ void k_reduce_jobs(const BestSlot* __restrict__ slots, int per_job, BestSlot* __restrict__ out) {
  __shared__ float ss[32];
  __shared__ unsigned long long sk[32];
  const BestSlot* js = slots + (int64_t)blockIdx.x * per_job;
  float bs = FLT_MAX;
  unsigned long long bk = ~0ull;
  for (int t = threadIdx.x; t < per_job; t += blockDim.x)
    if (better(js[t].score, js[t].key, bs, bk)) {
      bs = js[t].score;
      bk = js[t].key;
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
      out[blockIdx.x].score = bs;
      out[blockIdx.x].key = bk;
    }
  }
}

__global__ void k_fill_slots(BestSlot* __restrict__ slots, int64_t n) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) {
    slots[t].score = FLT_MAX;
    slots[t].key = ~0ull;
  }
}

int tc_warps_per_block() { return kTcWarps; }

template <int kW, bool kF, bool kP, bool kB, bool kD, bool kT, bool kM = false, bool kR = false>
static cudaError_t set_smem() {
  return cudaFuncSetAttribute(k_scan_tc<kW, kF, kP, kB, kD, kT, kM, kR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kTcSmemBytes);
}

template <int kW, bool kF, bool kP>
static cudaError_t set_smem_all() {
  cudaError_t e = set_smem<kW, kF, kP, false, false, false>();
  if (e == cudaSuccess) e = set_smem<kW, kF, kP, false, true, false>();
  if (e == cudaSuccess) e = set_smem<kW, kF, kP, false, false, true>();
  if (e == cudaSuccess) e = set_smem<kW, kF, kP, true, false, false>();
  return e;
}

cudaError_t tc_configure() {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = set_smem_all<4, false, false>();
    if (e == cudaSuccess) e = set_smem_all<8, false, false>();
    if (e == cudaSuccess) e = set_smem_all<8, true, false>();
    if (e == cudaSuccess) e = set_smem_all<16, true, false>();
    if (e == cudaSuccess) e = set_smem_all<8, true, true>();
    if (e == cudaSuccess) e = set_smem_all<16, true, true>();
    if (e == cudaSuccess) e = set_smem<16, true, true, false, false, false, true>();         // pair margins
    if (e == cudaSuccess) e = set_smem<16, true, true, false, false, false, false, true>();  // replicates
    if (e != cudaSuccess) return e;
    configured = true;
  }
  return cudaSuccess;
}

template <int kW, bool kF>
static void launch_variant(const TcParams& p, int blocks, bool batched, bool dump, bool topk, cudaStream_t stream) {
  if (batched) k_scan_tc<kW, kF, false, true, false, false><<<blocks, kTcThreadsAll, kTcSmemBytes, stream>>>(p);
  else if (dump) k_scan_tc<kW, kF, false, false, true, false><<<blocks, kTcThreadsAll, kTcSmemBytes, stream>>>(p);
  else if (topk) k_scan_tc<kW, kF, false, false, false, true><<<blocks, kTcThreadsAll, kTcSmemBytes, stream>>>(p);
  else k_scan_tc<kW, kF, false, false, false, false><<<blocks, kTcThreadsAll, kTcSmemBytes, stream>>>(p);
}

// CTA-pair kernels: clusters of two CTAs
template <int kW, bool kB, bool kD, bool kT, bool kM = false, bool kR = false>
static cudaError_t launch_pair(const TcParams& p, int blocks, cudaStream_t stream) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)blocks);
  cfg.blockDim = dim3(kTcThreadsAll);
  cfg.dynamicSmemBytes = kTcSmemBytes;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_scan_tc<kW, true, true, kB, kD, kT, kM, kR>, p);
}

template <int kW>
static cudaError_t launch_pair_variant(const TcParams& p, int blocks, bool batched, bool dump, bool topk,
                                       cudaStream_t stream) {
  if (batched) return launch_pair<kW, true, false, false>(p, blocks, stream);
  if (dump) return launch_pair<kW, false, true, false>(p, blocks, stream);
  if (topk) return launch_pair<kW, false, false, true>(p, blocks, stream);
  return launch_pair<kW, false, false, false>(p, blocks, stream);
}

int tc_k_per_tile(bool fp4) { return fp4 ? 112 : 128; }

// CTAs of the CTA-pair kernel that can be resident at once (even; at most one per SM).
int tc_pair_blocks(int sms) {
  static int blocks = -1;
  if (blocks < 0) {
    blocks = sms & ~1;
    if (tc_configure() == cudaSuccess) {
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3((unsigned)(sms & ~1));
      cfg.blockDim = dim3(kTcThreadsAll);
      cfg.dynamicSmemBytes = kTcSmemBytes;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = 2;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int clusters = 0;
      if (cudaOccupancyMaxActiveClusters(&clusters, k_scan_tc<16, true, true, false, false, false>, &cfg) ==
              cudaSuccess &&
          clusters > 0)
        blocks = std::min(blocks, 2 * clusters);
    }
    cudaGetLastError();
  }
  return blocks;
}

cudaError_t launch_scan_tc(const TcParams& p, int blocks, int words_per_stage, bool fp4, bool pair, bool dump,
                           cudaStream_t stream) {
  const cudaError_t ce = tc_configure();
  if (ce != cudaSuccess) return ce;
  const bool topk = p.top_k > 1;
  const bool batched = p.jobs != nullptr;
  if (fp4 && pair) {
    const cudaError_t e = words_per_stage == 16
                              ? launch_pair_variant<16>(p, blocks & ~1, batched, dump, topk, stream)
                              : launch_pair_variant<8>(p, blocks & ~1, batched, dump, topk, stream);
    if (e != cudaSuccess) return e;
  } else if (fp4) {
    if (words_per_stage == 16) launch_variant<16, true>(p, blocks, batched, dump, topk, stream);
    else launch_variant<8, true>(p, blocks, batched, dump, topk, stream);
  } else {
    if (words_per_stage == 8) launch_variant<8, false>(p, blocks, batched, dump, topk, stream);
    else launch_variant<4, false>(p, blocks, batched, dump, topk, stream);
  }
  return cudaGetLastError();
}

cudaError_t launch_scan_reps(const TcParams& p, int blocks, cudaStream_t stream) {
  const cudaError_t ce = tc_configure();
  if (ce != cudaSuccess) return ce;
  const cudaError_t e = launch_pair<16, false, false, false, false, true>(p, blocks & ~1, stream);
  return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t launch_pairs_tc(const TcParams& p, int blocks, cudaStream_t stream) {
  const cudaError_t ce = tc_configure();
  if (ce != cudaSuccess) return ce;
  const cudaError_t e = launch_pair<16, false, false, false, true>(p, blocks & ~1, stream);
  return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t launch_reduce_jobs(const BestSlot* slots, int n_jobs, int per_job, BestSlot* out, cudaStream_t stream) {
  if (n_jobs <= 0) return cudaSuccess;
  k_reduce_jobs<<<n_jobs, 256, 0, stream>>>(slots, per_job, out);
  return cudaGetLastError();
}

cudaError_t launch_fill_slots(BestSlot* slots, int64_t n, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  k_fill_slots<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(slots, n);
  return cudaGetLastError();
}

}  // namespace epik2
