// Overlapped tensor-core search (tcgen05, sm_100a): the CTA-pair FP4 kernel of scan_tc.cu
// restructured so that a tile's scoring runs while the tensor cores count the next tile.
//
// Same result as k_scan_tc and the integer engine (and the reference's kernel_epi,
// GPU/v4.cpp:295-594): 8 cells per class counted exactly as a block-scaled FP4 matrix
// product on CTA pairs (cta_group::2, M=256 N=224 K=64, 64 SNPs j x 112 SNPs k per tile),
// the other 19 cells by inclusion-exclusion, K2 in the reference's FP32 order, lowest
// (score, i, j, k) wins.
//
// In k_scan_tc every warp first produces operands for a tile and then scores it, so the
// tensor cores idle through the epilogue (about 40 % of a tile at 16384 samples).  Here the
// warps of a CTA have fixed roles and run concurrently:
//   * 8 producing warps expand the bit-plane words of every stage into the operand ring,
//     tile after tile (they fetch the tile descriptors and publish them);
//   * 1 issuing warp (one lane; in the odd CTA of a pair the lane forwards arrivals to the
//     even CTA) issues the matrix products of each stage once its operands are stored;
//   * 8 scoring warps wait for a tile's accumulators, copy them from tensor memory into a
//     16-bit staging buffer (which frees the accumulators for the next tile's products),
//     and then complete, score and select that tile's triplets while the next tile counts.
// Shared memory holds the operand ring (kW = 4 words per stage: 3 stages of 15 KiB; kW = 8:
// 2 of 30 KiB), the staging buffer (2 classes x 128 rows x 224 counts, 16 bits each, rows
// padded to 456 bytes) and the dataset's ln n! table for the whole launch.  The staging
// buffer holds counts below 2^16: classes of at most 65535 samples (the host checks).
//
// Hand-offs (all mbarriers, every wait bounded; an expired wait sets an error word, every
// role stops at its next check, tensor memory is freed, the host returns E_TIMEOUT):
//   tile[t%4]  even CTA's producer thread 0 -> odd CTA's: tile t's descriptor
//   desc[t%4]  producer thread 0 -> issuer/forwarder and scorers of its CTA: tile t's
//              descriptor
//   full[s]    8 producing warps (+1 forwarded from the odd CTA) -> issuer: stage stored
//   empty[s]   issuer's commit (both CTAs) -> producers: stage consumed
//   acc        issuer's commit after a tile's last products (both CTAs) -> scorers
//   drained    8 scoring warps (+1 forwarded) -> issuer: accumulators copied out; the next
//              tile's first product may overwrite them
// Named barriers: 1 = the 256 scoring threads, 2 = the 256 producing threads.  A group leaves
// its loop only on a value that every one of its threads reads after such a barrier and
// that no thread changes before all of them have passed the group's next barrier.
#include <cfloat>

#include "epik2_internal.h"
#include "scan_common.cuh"
#include "tc_ptx.cuh"

namespace epik2 {

constexpr int kPipeThreads = 544;          // 8 producing + 8 scoring warps + 1 issuing warp
constexpr int kPipeSmemBytes = 230400;
constexpr int kPipeBarOff = kPipeSmemBytes - 256;
constexpr int kPipeK = 112;                // SNPs k per tile (56 in each CTA's half of B)
constexpr int kERow = 456;                 // staging row: 224 16-bit counts + 8 bytes padding
constexpr int kEBytes = 2 * 128 * kERow;   // both classes

template <int kW>
struct PipeShape {
  static constexpr int kRowBytes = 16 * kW;               // E2M1 operand bytes per row per stage
  static constexpr int kStageBytes = 240 * kRowBytes;     // 128 A rows + 112 B rows
  static constexpr int kStages = kW == 4 ? 3 : 2;
  static constexpr int kEOff = kStages * kStageBytes;
  static constexpr int kLutOff = kEOff + kEBytes;
  static constexpr int kLutCap = (kPipeBarOff - kLutOff) / 4;  // ln n! entries that fit
};
static_assert(PipeShape<4>::kLutOff % 16 == 0 && PipeShape<8>::kLutOff % 16 == 0, "table alignment");
static_assert(PipeShape<4>::kLutCap % 4 == 0 && PipeShape<8>::kLutCap % 4 == 0, "whole 16-byte table pieces");
static_assert(PipeShape<4>::kLutCap >= 16388, "16384 samples keep their table in shared memory");

// barrier slots (8 bytes each) at kPipeBarOff
constexpr int kBFull = 0, kBEmpty = 4, kBAcc = 8, kBTile = 9, kBDrained = 13, kBDesc = 14, kBFinal = 18;
static_assert((kBFinal + 1) * 8 <= 256, "barrier area");

// One dataset's view for a tile (the batched form reads the tile's dataset from the job table).
struct JobRef {
  const uint2* planes;
  const uint32_t* singles;
  const uint4* pairs;
  const float* lut;
  int64_t tri;
  int32_t m, m_pad, w0, w1, n0, n1;
};

__device__ __forceinline__ void named_sync(int id, int threads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

__device__ __forceinline__ void sts64(uint32_t saddr, uint32_t a, uint32_t b) {
  asm volatile("st.shared.v2.b32 [%0], {%1, %2};" ::"r"(saddr), "r"(a), "r"(b) : "memory");
}

template <int kW, bool kBatched, bool kDump, bool kTopK>
__global__ void __launch_bounds__(kPipeThreads, 1) k_scan_pipe(const TcParams p) {
  using S = PipeShape<kW>;
  constexpr int kRowBytes = S::kRowBytes, kStageBytes = S::kStageBytes, kStages = S::kStages;
  constexpr uint32_t kSbo = 8 * kRowBytes;  // bytes between 8-row groups
  constexpr int kMmas = kW / 2;             // K = 64 samples per MMA
  constexpr int kAb = kW / 2;               // A rows (g_i, g_j) per producing thread per stage
  constexpr int kUB = kW / 4;               // 8-byte B plane loads per producing thread per stage
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint32_t s_tmem;
  __shared__ long long s_hand[4];           // odd CTA: descriptors handed over by the even CTA
  __shared__ long long s_desc[4];           // this CTA's descriptor of tile t at t % 4
  __shared__ int s_abort, s_pfail, s_sfail;
  __shared__ float s_red_s[8];
  __shared__ unsigned long long s_red_k[8];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t crank = cluster_rank();
  const bool even = crank == 0;
  const uint32_t stage0 = smem_u32(smem), bar0 = smem_u32(smem + kPipeBarOff);
  auto bar = [&](int slot) { return bar0 + 8u * (uint32_t)slot; };
  const long long wl = p.wait_limit > 0 ? p.wait_limit : kWaitLimit;
  volatile int* abort_flag = &s_abort;
  volatile int* pfail = &s_pfail;
  volatile int* sfail = &s_sfail;

  if (tid == 0) {
    for (int s = 0; s < kStages; s++) {
      bar_init(bar(kBFull + s), 8 + (even ? 1 : 0));
      bar_init(bar(kBEmpty + s), 1);
    }
    bar_init(bar(kBAcc), 1);
    for (int d = 0; d < 4; d++) {
      bar_init(bar(kBTile + d), 1);
      bar_init(bar(kBDesc + d), 1);
    }
    bar_init(bar(kBDrained), 8 + (even ? 1 : 0));
    bar_init(bar(kBFinal), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
    s_pfail = 0;
    s_sfail = 0;
  }
  cluster_sync_all();  // both CTAs' barriers exist before any remote arrival
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(512u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  if (warp < 4) {  // scale factors: every byte of columns [224, 256) = 0x80 (2^1), all 128 lanes
    const uint32_t ta = tmem + ((uint32_t)(32 * warp) << 16) + kSfaCol;
    tmem_st16_fill(ta, 0x80808080u);
    tmem_st16_fill(ta + 16, 0x80808080u);
    tmem_wait_st();
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // both CTAs' scale factors are in place before the first product
  tc_fence_after();

  auto job_of = [&](long long desc) -> JobRef {
    if (kBatched) {
      const TcJob& J = p.jobs[tile_job((uint64_t)desc)];
      return JobRef{J.planes, J.singles, J.pairs, J.lut, J.tri, J.m, J.m_pad, J.w0, J.w1, J.n0, J.n1};
    }
    (void)desc;
    return JobRef{p.planes, p.singles, p.pairs, p.lut, p.tri, p.m, p.m_pad, p.w0, p.w1, p.n0, p.n1};
  };

  if (warp < 8) {
    // ================= producing warps =================
    const int pw = warp;  // 0..7
    uint32_t g = 0;       // stages produced so far (ring position)
    unsigned long long pf_t = 0;
    long long pf_d = -1;
    for (uint32_t t = 0;; t++) {
      if (tid == 0) {  // tile t's descriptor: fetched by the even CTA, handed to the odd one
        long long d = -1;
        if (even) {
          if (t == 0) {
            pf_t = atomicAdd(p.counter, 1ull);
            pf_d = pf_t < (unsigned long long)p.n_tiles ? (long long)__ldg(p.tiles + pf_t) : -1ll;
          }
          d = (*abort_flag || *pfail) ? -1ll : pf_d;
          if (d >= 0) {
            pf_t = atomicAdd(p.counter, 1ull);
            pf_d = pf_t < (unsigned long long)p.n_tiles ? (long long)__ldg(p.tiles + pf_t) : -1ll;
          }
          st_cluster_s64(map_cta(smem_u32(&s_hand[t % 4]), 1), d);
          bar_arrive_cluster(map_cta(bar(kBTile + (int)(t % 4)), 1));
        } else if (bar_wait_cluster(bar(kBTile + (int)(t % 4)), (t / 4) & 1u, wl)) {
          d = *reinterpret_cast<volatile long long*>(&s_hand[t % 4]);
        } else {
          *abort_flag = 1;
        }
        if (*pfail || *abort_flag) d = -1;  // a failed wait of any producing warp ends the production
        s_desc[t % 4] = d;
        bar_arrive(bar(kBDesc + (int)(t % 4)));  // release: the descriptor is visible to its waiters
      }
      named_sync(2, 256);
      // leave only on the descriptor: thread 0 wrote it before the barrier and rewrites the
      // slot four tiles later, after every producing thread has passed the next barriers
      const long long desc = *reinterpret_cast<volatile long long*>(&s_desc[t % 4]);
      if (desc < 0) break;
      const JobRef jv = job_of(desc);
      const int i = tile_i((uint64_t)desc), j0 = tile_j0((uint64_t)desc) + 32 * (int)crank;
      const int k0 = tile_k0((uint64_t)desc, kPipeK);
      const int64_t m_pad = jv.m_pad;
      const int nc0 = (jv.w0 + kW - 1) / kW, nc1 = (jv.w1 + kW - 1) / kW, nct = nc0 + nc1;
      // A: pair q = lane, word wA = pw % kW, rows (g_i, g_j) = ab0 .. ab0 + kAb - 1
      const int wA = pw % kW, ab0 = (pw / kW) * kAb;
      const int a_j = min(j0 + lane, (int)m_pad - 1);
      // B: SNP k0 + 56*crank + kp (kp = tid & 63 < 56), words (tid >> 6) + 4r, r < kUB
      const int kp = tid & 63;
      const bool b_on = kp < kPipeK / 2;
      const int b_k = k0 + (kPipeK / 2) * (int)crank + kp;
      const uint32_t offb0 = (kp >> 3) * kSbo + (kp & 7) * 16;  // + 7*kSbo for g_k = 1
      auto load_words = [&](int cc, uint2& gi, uint2& gj, uint2 (&gk)[kUB]) {
        const bool c1 = cc >= nc0;
        const int c_in = c1 ? cc - nc0 : cc;
        const int wcls = c1 ? jv.w1 : jv.w0;
        const int64_t wb = (c1 ? (int64_t)jv.w0 : 0) + (int64_t)kW * c_in;
        gi = make_uint2(0, 0);
        gj = gi;
        if (kW * c_in + wA < wcls) {
          const uint2* row = jv.planes + (wb + wA) * m_pad;
          gi = __ldg(row + i);
          gj = __ldg(row + a_j);
        }
#pragma unroll
        for (int r = 0; r < kUB; r++) {
          const int w = (tid >> 6) + 4 * r;
          gk[r] = make_uint2(0, 0);
          if (kW * c_in + w < wcls && b_on && b_k < m_pad) gk[r] = __ldg(jv.planes + (wb + w) * m_pad + b_k);
        }
      };
      uint2 ci, cj, ck[kUB];
      if (nct > 0) load_words(0, ci, cj, ck);
      for (int cc = 0; cc < nct; ++cc) {
        const uint32_t gg = g + (uint32_t)cc;
        uint2 ni = make_uint2(0, 0), nj = ni, nk[kUB];
#pragma unroll
        for (int r = 0; r < kUB; r++) nk[r] = make_uint2(0, 0);
        if (cc + 1 < nct) load_words(cc + 1, ni, nj, nk);
        const int s = (int)(gg % kStages);
        const uint32_t use = gg / kStages;
        const bool late = use > 0 && !bar_wait_cluster(bar(kBEmpty + s), (use & 1u) ^ 1u, wl);
        if (__any_sync(kFull, late)) {
          if (lane == 0) *pfail = 1;
          break;
        }
        const uint32_t sA = stage0 + s * kStageBytes, sB = sA + 128 * kRowBytes;
#pragma unroll
        for (int t2 = 0; t2 < kAb; t2++) {
          const int ab = ab0 + t2, row = 32 * ab + lane;
          const uint32_t wa = ((ab >> 1) ? ci.y : ci.x) & ((ab & 1) ? cj.y : cj.x);
          sts128(sA + (row >> 3) * kSbo + (row & 7) * 16 + wA * 128, expand32_fp4(wa));
        }
#pragma unroll
        for (int r = 0; r < kUB; r++) {
          const int w = (tid >> 6) + 4 * r;
          if (b_on) {
            const uint32_t offb = sB + offb0 + w * 128;
            sts128(offb, expand32_fp4(ck[r].x));
            sts128(offb + 7 * kSbo, expand32_fp4(ck[r].y));
          }
        }
        ci = ni;
        cj = nj;
#pragma unroll
        for (int r = 0; r < kUB; r++) ck[r] = nk[r];
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) bar_arrive(bar(kBFull + s));
      }
      g += (uint32_t)nct;
    }
  } else if (warp < 16) {
    // ================= scoring warps =================
    const int sw = warp - 8, st = tid - 256;  // 0..7, 0..255
    const int quarter = warp & 3, half = sw >> 2;
    const float* lut_s = reinterpret_cast<const float*>(smem + S::kLutOff);
    const uint16_t* E = reinterpret_cast<const uint16_t*>(smem + S::kEOff);
    float best_s = FLT_MAX, list_s = FLT_MAX;
    unsigned long long best_k = ~0ull, list_k = ~0ull;
    int cur_job = -1;
    bool lut_shared = false;
    // fold the scorers' best of job jb into its slot (batched form)
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
      if (lane == 0) {
        s_red_s[sw] = best_s;
        s_red_k[sw] = best_k;
      }
      named_sync(1, 256);
      if (st == 0) {
        float bs = s_red_s[0];
        unsigned long long bk = s_red_k[0];
        for (int w = 1; w < 8; w++)
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
      named_sync(1, 256);
      best_s = FLT_MAX;
      best_k = ~0ull;
    };
    auto load_lut = [&](const JobRef& jv) {  // the dataset's ln n! table into shared memory, if it fits
      lut_shared = (jv.n0 + jv.n1 + 2 + 3) / 4 * 4 <= S::kLutCap;  // whole 16-byte pieces
      if (lut_shared) {  // the device table is padded to 256 bytes: whole 16-byte pieces stay inside
        const int n16 = (jv.n0 + jv.n1 + 2 + 3) / 4;
        for (int x = st; x < n16; x += 256) cp_async16(stage0 + S::kLutOff + 16 * x, jv.lut + 4 * x);
        cp_async_wait_all();
      }
      named_sync(1, 256);
    };
    if (!kBatched) load_lut(job_of(0));
    for (uint32_t t = 0;; t++) {
      const bool got = bar_wait(bar(kBDesc + (int)(t % 4)), (t / 4) & 1u, wl);
      const long long desc = got ? *reinterpret_cast<volatile long long*>(&s_desc[t % 4]) : -1ll;
      bool ok = got;
      if (ok && desc >= 0) ok = bar_wait_cluster(bar(kBAcc), t & 1u, wl);
      if (!ok || *abort_flag) *sfail = 1;  // written only here, before the barrier
      named_sync(1, 256);
      if (desc < 0 || *sfail) break;
      const int job = kBatched ? tile_job((uint64_t)desc) : 0;
      const JobRef jv = job_of(desc);
      if (kBatched && job != cur_job) {
        if (cur_job >= 0) flush_job(cur_job);
        cur_job = job;
        load_lut(jv);
      }
      tc_fence_after();
      // accumulators -> 16-bit staging rows: warp (quarter, half) copies class `half` for its
      // 32 lanes (rows 32*quarter + lane), columns in 14 groups of 16
      {
        const bool has = half ? jv.w1 > 0 : jv.w0 > 0;
        const int row = 32 * quarter + lane;
        const uint32_t dst_row = stage0 + S::kEOff + (uint32_t)((half * 128 + row) * kERow);
#pragma unroll 1
        for (int u = 0; u < 14; u++) {
          uint32_t v[16];
          if (has) {
            tmem_ld16(tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(half * 256 + 16 * u), v);
            tmem_wait_ld();
#pragma unroll
            for (int x = 0; x < 16; x++) v[x] = __float2uint_rn(__uint_as_float(v[x]));
          } else {
#pragma unroll
            for (int x = 0; x < 16; x++) v[x] = 0;
          }
#pragma unroll
          for (int x = 0; x < 4; x++)
            sts64(dst_row + 32 * u + 8 * x, v[4 * x] | (v[4 * x + 1] << 16), v[4 * x + 2] | (v[4 * x + 3] << 16));
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) bar_arrive(bar(kBDrained));
      named_sync(1, 256);  // every warp's staging rows are written
      // complete, score and select: slot x = st + 256u -> pair q = x / 112, k offset kk
      const int i = tile_i((uint64_t)desc), j0 = tile_j0((uint64_t)desc) + 32 * (int)crank;
      const int k0 = tile_k0((uint64_t)desc, kPipeK);
      const int m = jv.m;
      const int64_t m_pad = jv.m_pad, tri = jv.tri;
      const uint2 si0 = *reinterpret_cast<const uint2*>(jv.singles + ((int64_t)i) * 2);
      const uint2 si1 = *reinterpret_cast<const uint2*>(jv.singles + (m_pad + i) * 2);
#pragma unroll 1
      for (int u = 0; u < 14; u++) {
        const int x = st + 256 * u;
        const int q = x / kPipeK, kk = x - q * kPipeK;
        const int j = j0 + q, k = k0 + kk;
        const bool valid = (j < m) && (k > j) && (k < m);
        float sc = FLT_MAX;
        unsigned long long key = ~0ull;
        if (valid) {
          const int hh = kk >= kPipeK / 2 ? 1 : 0;
          const int col = 112 * hh + (kk - (kPipeK / 2) * hh);  // g_k = 0; g_k = 1 is 56 further
          uint32_t t80[8], t81[8];
#pragma unroll
          for (int ab = 0; ab < 4; ab++)
#pragma unroll
            for (int c = 0; c < 2; c++) {
              t80[2 * ab + c] = E[(0 * 128 + 32 * ab + q) * (kERow / 2) + col + 56 * c];
              t81[2 * ab + c] = E[(1 * 128 + 32 * ab + q) * (kERow / 2) + col + 56 * c];
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
            const int64_t ti = triplet_index(m, i, j, k);
            uint32_t* dt = p.dump_tables + ti * 54;
#pragma unroll
            for (int c = 0; c < 27; c++) {
              dt[c] = T0[c];
              dt[27 + c] = T1[c];
            }
            p.dump_scores[ti] = sc;
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
    }
    if (kBatched && cur_job >= 0) flush_job(cur_job);
    if (!kBatched) {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const float os = __shfl_xor_sync(kFull, best_s, off);
        const unsigned long long ok = __shfl_xor_sync(kFull, best_k, off);
        if (better(os, ok, best_s, best_k)) {
          best_s = os;
          best_k = ok;
        }
      }
      const int64_t gwarp = (int64_t)blockIdx.x * 16 + warp;
      if (lane == 0) {
        p.slots[gwarp].score = best_s;
        p.slots[gwarp].key = best_k;
      }
      if (kTopK) {
        p.cand[gwarp * 32 + lane].score = list_s;
        p.cand[gwarp * 32 + lane].key = list_k;
      }
    }
  } else if (lane == 0) {
    // ================= issuing lane (even CTA) / forwarding lane (odd CTA) =================
    uint32_t g = 0;
    for (uint32_t t = 0;; t++) {
      if (!bar_wait(bar(kBDesc + (int)(t % 4)), (t / 4) & 1u, wl)) {
        *abort_flag = 1;
        break;
      }
      const long long desc = *reinterpret_cast<volatile long long*>(&s_desc[t % 4]);
      if (desc < 0) break;
      const JobRef jv = job_of(desc);
      const int nc0 = (jv.w0 + kW - 1) / kW, nc1 = (jv.w1 + kW - 1) / kW, nct = nc0 + nc1;
      bool fail = false;
      if (t > 0) {  // the previous tile's accumulators have been copied out
        if (even) {
          fail = !bar_wait_cluster(bar(kBDrained), (t - 1) & 1u, wl);
        } else {
          fail = !bar_wait(bar(kBDrained), (t - 1) & 1u, wl);
          if (!fail) bar_arrive_cluster(map_cta(bar(kBDrained), 0));
        }
      }
      for (int cc = 0; cc < nct && !fail; ++cc) {
        const uint32_t gg = g + (uint32_t)cc;
        const int s = (int)(gg % kStages);
        const uint32_t use = gg / kStages;
        if (!even) {  // forward "stage stored" to the issuing CTA
          if (!bar_wait(bar(kBFull + s), use & 1u, wl)) {
            fail = true;
            break;
          }
          bar_arrive_cluster(map_cta(bar(kBFull + s), 0));
          continue;
        }
        if (!bar_wait_cluster(bar(kBFull + s), use & 1u, wl)) {
          fail = true;
          break;
        }
        tc_fence_after();
        const bool c1 = cc >= nc0;
        const int c_in = c1 ? cc - nc0 : cc;
        const uint32_t sA = stage0 + s * kStageBytes, sB = sA + 128 * kRowBytes;
        const uint32_t d = tmem + (c1 ? 256u : 0u);
        const uint64_t da = smem_desc(sA, kSbo), db = smem_desc(sB, kSbo);
#pragma unroll
        for (int kk = 0; kk < kMmas; kk++) {
          const uint32_t acc = (c_in > 0 || kk > 0) ? 1u : 0u;
          mma_fp4_pair(d, da + (uint64_t)(16 * kk), db + (uint64_t)(16 * kk), acc, tmem + kSfaCol, tmem + kSfbCol);
        }
        mma_commit_pair(bar(kBEmpty + s));
        if (cc == nct - 1) mma_commit_pair(bar(kBAcc));
      }
      if (fail) {
        *abort_flag = 1;
        break;
      }
      g += (uint32_t)nct;
    }
  }
  if (warp < 8 && !kBatched) {  // producing warps hold no candidates
    const int64_t gwarp = (int64_t)blockIdx.x * 16 + warp;
    if (lane == 0) {
      p.slots[gwarp].score = FLT_MAX;
      p.slots[gwarp].key = ~0ull;
    }
    if (kTopK) {
      p.cand[gwarp * 32 + lane].score = FLT_MAX;
      p.cand[gwarp * 32 + lane].key = ~0ull;
    }
  }

  // ---- teardown: every role has left its loop ----
  // Tensor memory is released only after every product has completed (after an expired wait
  // the issuer may have left its last stages running): the issuing lane commits once more and
  // each CTA's lane 0 of the issuing warp waits for that commit, bounded.
  if (warp == 16 && lane == 0) {
    if (even) mma_commit_pair(bar(kBFinal));
    if (!bar_wait_cluster(bar(kBFinal), 0, wl)) s_abort = 1;
  }
  tc_fence_before();
  __syncthreads();
  if ((s_abort || s_pfail || s_sfail) && tid == 0) atomicExch(p.err, 1);
  cluster_sync_all();  // the pair's products and remote arrivals are over
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
  }
}

template <int kW, bool kB, bool kD, bool kT>
static cudaError_t pipe_set_smem() {
  return cudaFuncSetAttribute(k_scan_pipe<kW, kB, kD, kT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kPipeSmemBytes);
}

// Dynamic shared-memory limit of every variant, once (outside any stream capture).
cudaError_t pipe_configure() {
  static bool configured = false;
  if (configured) return cudaSuccess;
  cudaError_t e = pipe_set_smem<4, false, false, false>();
  if (e == cudaSuccess) e = pipe_set_smem<4, false, true, false>();
  if (e == cudaSuccess) e = pipe_set_smem<4, false, false, true>();
  if (e == cudaSuccess) e = pipe_set_smem<4, true, false, false>();
  if (e == cudaSuccess) e = pipe_set_smem<8, false, false, false>();
  if (e == cudaSuccess) e = pipe_set_smem<8, false, true, false>();
  if (e == cudaSuccess) e = pipe_set_smem<8, false, false, true>();
  if (e == cudaSuccess) e = pipe_set_smem<8, true, false, false>();
  if (e == cudaSuccess) configured = true;
  return e;
}

template <int kW, bool kB, bool kD, bool kT>
static cudaError_t launch_pipe_kernel(const TcParams& p, int blocks, cudaStream_t stream) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)blocks);
  cfg.blockDim = dim3(kPipeThreads);
  cfg.dynamicSmemBytes = kPipeSmemBytes;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_scan_pipe<kW, kB, kD, kT>, p);
}

template <int kW>
static cudaError_t launch_pipe_variant(const TcParams& p, int blocks, bool batched, bool dump, bool topk,
                                       cudaStream_t stream) {
  if (batched) return launch_pipe_kernel<kW, true, false, false>(p, blocks, stream);
  if (dump) return launch_pipe_kernel<kW, false, true, false>(p, blocks, stream);
  if (topk) return launch_pipe_kernel<kW, false, false, true>(p, blocks, stream);
  return launch_pipe_kernel<kW, false, false, false>(p, blocks, stream);
}

bool pipe_fits(int64_t n_controls, int64_t n_cases) { return n_controls <= 65535 && n_cases <= 65535; }

cudaError_t launch_scan_pipe(const TcParams& p, int blocks, int words_per_stage, bool dump, cudaStream_t stream) {
  const cudaError_t ce = pipe_configure();
  if (ce != cudaSuccess) return ce;
  const bool topk = p.top_k > 1;
  const bool batched = p.jobs != nullptr;
  const cudaError_t e = words_per_stage == 8 ? launch_pipe_variant<8>(p, blocks & ~1, batched, dump, topk, stream)
                                             : launch_pipe_variant<4>(p, blocks & ~1, batched, dump, topk, stream);
  return e != cudaSuccess ? e : cudaGetLastError();
}

}  // namespace epik2
