// epik2_scan_u8_noalloc: the one-call search (same result as epik2_scan_u8) for callers
// that cannot allocate device memory -- code running where cudaMalloc is unavailable or
// forbidden, such as a plugin inside a host application that owns the device heap, or
// a process whose memory budget is fixed before this library is reached.  No context
// is created: every intermediate buffer (uploaded matrix, class order, bit planes,
// margins, ln n! table, work counter, per-warp results) lives in one file-scope
// __device__ array of EPIK2_NOALLOC_SCRATCH_BYTES, which every GPU that loads this
// library holds until the process exits.
//
// Rules of use:
//   * Every call resolves the array's device address on the current device with
//     cudaGetSymbolAddress (the host-side symbol is only a stand-in, never a device
//     pointer), so the address stays right after a device reset or a new primary
//     context.  No call may run under stream capture: each one waits for its stream and
//     copies through pageable host buffers, which capture forbids; a capturing stream is
//     refused with EPIK2_E_INVALID before anything is enqueued.
//   * All calls share the one array and it keeps the last call's contents; everything
//     that must start at zero is cleared by each call.  Calls whose GPU work overlaps
//     (two host threads, or two streams) race on the array; the host side serialises
//     calls from one process with a mutex, but work on different streams still must not
//     overlap on the device.
//   * Shapes whose buffers exceed the array are rejected with EPIK2_E_TOO_LARGE.
//   * A call that fails after it has enqueued work waits for its stream before it
//     returns, so the array is idle when the next call starts.
//   * Nothing here calls cudaMalloc, cudaFree or any allocating routine; host staging
//     uses fixed static buffers.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "../../include/epik2.h"
#include "epik2_internal.h"

namespace epik2 {
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[EPIK2_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
constexpr int64_t kLutChunk = 16384;
constexpr int64_t kMaxFirst = 4096;

std::mutex g_mu;
int g_blocks[kMaxDevices] = {};
float g_lut_chunk[kLutChunk];
int64_t g_pgoff[kMaxFirst + 1];
BestSlot g_best;

// Class-sorted sample order (controls, then cases), one block: each thread owns a
// contiguous slice of samples; a block-wide exclusive scan of per-slice case counts
// gives every sample its destination.
__global__ void k_class_order(const uint8_t* __restrict__ pheno, int64_t s, int64_t n_controls,
                              int32_t* __restrict__ perm) {
  __shared__ int64_t part[1024];
  const int t = threadIdx.x;
  const int64_t chunk = (s + blockDim.x - 1) / blockDim.x;
  const int64_t lo = std::min<int64_t>(s, (int64_t)t * chunk), hi = std::min<int64_t>(s, lo + chunk);
  int64_t c1 = 0;
  for (int64_t q = lo; q < hi; q++) c1 += (pheno[q] == 1);
  part[t] = c1;
  __syncthreads();
  for (int off = 1; off < (int)blockDim.x; off <<= 1) {  // inclusive Hillis-Steele scan
    const int64_t v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int64_t cases_before = part[t] - c1;
  int64_t controls_before = lo - cases_before;
  for (int64_t q = lo; q < hi; q++) {
    if (pheno[q] == 1) perm[n_controls + cases_before++] = (int32_t)q;
    else perm[controls_before++] = (int32_t)q;
  }
}

size_t up256(size_t v) { return (v + 255) / 256 * 256; }

struct NoAllocLayout {
  size_t geno, pheno, perm, planes, singles, pairs, lut, pgoff, slots, counter, best, total;
};

NoAllocLayout noalloc_layout(int64_t s, int64_t m, int n_warps) {
  const int64_t m_pad = (m + 31) / 32 * 32;
  const int64_t words = (s + 31) / 32 + 1;
  NoAllocLayout L{};
  size_t off = 0;
  L.geno = off;    off = up256(off + (size_t)(s * m));
  L.pheno = off;   off = up256(off + (size_t)s);
  L.perm = off;    off = up256(off + (size_t)s * 4);
  L.planes = off;  off = up256(off + (size_t)(words * m_pad) * 8);
  L.singles = off; off = up256(off + (size_t)m_pad * 16);
  L.pairs = off;   off = up256(off + (size_t)(2 * tri_size(m_pad)) * 16);
  L.lut = off;     off = up256(off + (size_t)(s + 2) * 4);
  L.pgoff = off;   off = up256(off + (size_t)(m + 1) * 8);
  L.slots = off;   off = up256(off + (size_t)n_warps * sizeof(BestSlot));
  L.counter = off; off = up256(off + 8);
  L.best = off;    off = up256(off + sizeof(BestSlot));
  L.total = off;
  return L;
}

}  // namespace
}  // namespace epik2

using namespace epik2;

extern "C" int epik2_scan_u8_noalloc(const uint8_t* geno, const uint8_t* pheno, int64_t n_samples, int64_t n_snps,
                                     void* cuda_stream, epik2_best* out) {
  if (!geno || !pheno || !out || n_samples < 1 || n_snps < 3) return EPIK2_E_INVALID;
  if (n_snps > kMaxFirst) return EPIK2_E_TOO_LARGE;
  std::lock_guard<std::mutex> lock(g_mu);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return EPIK2_E_NO_DEVICE;
  cudaStream_t st = (cudaStream_t)cuda_stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) return EPIK2_E_CUDA;
  if (cap != cudaStreamCaptureStatusNone) return EPIK2_E_INVALID;  // waits and pageable copies end a capture
  if (!g_blocks[dev]) {  // grid size of this device, once
    int major = 0, sms = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess || major != 10)
      return EPIK2_E_NO_DEVICE;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return EPIK2_E_NO_DEVICE;
    g_blocks[dev] = sms * scan_blocks_per_sm();
  }
  // the array's address in the current context (looked up on every call: a device reset
  // or a new primary context moves it)
  void* sym = nullptr;
  if (cudaGetSymbolAddress(&sym, g_noalloc_scratch) != cudaSuccess || !sym) return EPIK2_E_CUDA;
  unsigned char* base = (unsigned char*)sym;
  const int n_warps = g_blocks[dev] * (kScanThreads / 32);
  const NoAllocLayout L = noalloc_layout(n_samples, n_snps, n_warps);
  if (L.total > (size_t)EPIK2_NOALLOC_SCRATCH_BYTES) return EPIK2_E_TOO_LARGE;

  int64_t n1 = 0;
  for (int64_t q = 0; q < n_samples; q++) n1 += (pheno[q] == 1);
  DevDataset d{};
  d.n_samples = n_samples;
  d.n_snps = n_snps;
  d.n_cases = n1;
  d.n_controls = n_samples - n1;
  d.m_pad = (n_snps + 31) / 32 * 32;
  d.w0 = (d.n_controls + 31) / 32;
  d.w1 = (d.n_cases + 31) / 32;
  d.tri = tri_size(d.m_pad);
  d.geno = base + L.geno;
  d.perm = (int32_t*)(base + L.perm);
  d.planes = (uint2*)(base + L.planes);
  d.singles = (uint32_t*)(base + L.singles);
  d.pairs = (uint4*)(base + L.pairs);
  d.lut = (float*)(base + L.lut);
  uint8_t* d_pheno = base + L.pheno;

  // after the first enqueue a failing step waits for the stream (ignoring its status), so
  // that no copy or kernel of this call still uses the array when the lock is released
#define NA_CK(x)                    \
  do {                              \
    if ((x) != cudaSuccess) {       \
      cudaStreamSynchronize(st);    \
      cudaGetLastError();           \
      return EPIK2_E_CUDA;          \
    }                               \
  } while (0)
  NA_CK(cudaMemcpyAsync(d.geno, geno, (size_t)(n_samples * n_snps), cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemcpyAsync(d_pheno, pheno, (size_t)n_samples, cudaMemcpyHostToDevice, st));
  for (int64_t n0 = 0; n0 < n_samples + 2; n0 += kLutChunk) {
    const int64_t n1c = std::min<int64_t>(n_samples + 2, n0 + kLutChunk);
    NA_CK(cudaStreamSynchronize(st));  // the static chunk buffer is reused
    build_k2_lut_range(n0, n1c, g_lut_chunk);
    NA_CK(cudaMemcpyAsync(d.lut + n0, g_lut_chunk, (size_t)(n1c - n0) * 4, cudaMemcpyHostToDevice, st));
  }
  k_class_order<<<1, 1024, 0, st>>>(d_pheno, n_samples, d.n_controls, d.perm);
  NA_CK(cudaGetLastError());
  NA_CK(launch_encode(d, st));
  NA_CK(launch_counts(d, st));

  // pair groups (i, j0..j0+3) per first index i, as in the context path
  g_pgoff[0] = 0;
  for (int64_t i = 0; i < n_snps; i++)
    g_pgoff[i + 1] = g_pgoff[i] + ((i <= n_snps - 3) ? (n_snps - 2 - i + kPairsPerWarp) / kPairsPerWarp : 0);
  int64_t* d_pgoff = (int64_t*)(base + L.pgoff);
  NA_CK(cudaMemcpyAsync(d_pgoff, g_pgoff, (size_t)(n_snps + 1) * 8, cudaMemcpyHostToDevice, st));
  unsigned long long* d_counter = (unsigned long long*)(base + L.counter);
  NA_CK(cudaMemsetAsync(d_counter, 0, 8, st));

  ScanParams p{};
  p.planes = d.planes;
  p.singles = d.singles;
  p.pairs = d.pairs;
  p.lut = d.lut;
  p.pg_off = d_pgoff;
  p.n_groups = g_pgoff[n_snps];
  p.tri = d.tri;
  p.n_first = (int32_t)n_snps;
  p.i_begin = 0;
  p.m = (int32_t)n_snps;
  p.m_pad = (int32_t)d.m_pad;
  p.w0 = (int32_t)d.w0;
  p.w1 = (int32_t)d.w1;
  p.n0 = (int32_t)d.n_controls;
  p.n1 = (int32_t)d.n_cases;
  p.counter = d_counter;
  p.slots = (BestSlot*)(base + L.slots);
  p.top_k = 0;
  NA_CK(launch_scan_int(p, g_blocks[dev], false, st));
  BestSlot* d_best = (BestSlot*)(base + L.best);
  NA_CK(launch_reduce_best(p.slots, n_warps, d_best, st));
  NA_CK(cudaMemcpyAsync(&g_best, d_best, sizeof(BestSlot), cudaMemcpyDeviceToHost, st));
  NA_CK(cudaStreamSynchronize(st));
#undef NA_CK
  if (g_best.key == ~0ull) return EPIK2_E_INVALID;
  out->score = g_best.score;
  out->score_fp64 = __builtin_nan("");
  out->i = (uint32_t)(g_best.key >> 42);
  out->j = (uint32_t)((g_best.key >> 21) & ((1ull << 21) - 1));
  out->k = (uint32_t)(g_best.key & ((1ull << 21) - 1));
  return EPIK2_OK;
}
