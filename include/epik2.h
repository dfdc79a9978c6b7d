/*
 * epik2.h -- C ABI of the B200 exhaustive third-order K2 epistasis search.
 *
 * Drop-in for the GPU search path of hiperbio/cross-dpc-episdet (GPU/v1.cpp-v4.cpp).
 * The reference has no library interface: its seams are the process CLI
 * (GPU/v4.cpp:210-212, 610-612) and, inside main(), the hand-off from encoding to the
 * search kernel (GPU/v4.cpp:219-297) and from the kernel to the host argmin
 * (GPU/v4.cpp:599-608).  Each entry point below names the reference code it replaces.
 *
 * Conventions
 *   - Every function returns 0 (EPIK2_OK) or a negative EPIK2_E_* status; no exception
 *     or longjmp crosses the ABI.  epik2_last_error() gives the message of the last
 *     failure on a context.
 *   - The caller owns every host buffer; the library owns every device buffer through
 *     the context and frees it in epik2_unload / epik2_destroy.
 *   - A context belongs to one host thread at a time (the serving loop in this library
 *     serialises its own use).
 *   - Genotypes are uint8 in {0,1,2}, sample-major [n_samples][n_snps], the layout of the
 *     reference's generate_data (GPU/v4.cpp:94).  As in the reference's encoder
 *     (GPU/v4.cpp:161-171) any value other than 0 or 1 counts as genotype 2.
 *   - Phenotype is uint8 [n_samples]; value 1 = case, anything else = control
 *     (GPU/v4.cpp:152).
 *   - Triplets are 0-based SNP indices i < j < k.  Ties in score go to the lowest
 *     (i, j, k) in lexicographic order.
 *   - Contingency tables are 54 uint32: cell c = 9*g_i + 3*g_j + g_k, controls in
 *     [0,27), cases in [27,54) (GPU/v4.cpp:317-319).
 */
#ifndef EPIK2_H
#define EPIK2_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EPIK2_ABI_VERSION 1

/* status codes */
#define EPIK2_OK 0
#define EPIK2_E_INVALID (-1)   /* bad argument (null pointer, size out of range, unknown option) */
#define EPIK2_E_CUDA (-2)      /* CUDA runtime error; the context stays usable unless noted */
#define EPIK2_E_NOMEM (-3)     /* device memory exhausted, or admission refused for lack of HBM */
#define EPIK2_E_NOT_FOUND (-4) /* unknown dataset or request handle */
#define EPIK2_E_TOO_LARGE (-5) /* size beyond a documented limit */
#define EPIK2_E_TIMEOUT (-6)   /* a bounded device-side or host-side wait expired */
#define EPIK2_E_NO_DEVICE (-7) /* no CUDA device, or not an sm_100 device */
#define EPIK2_E_BUSY (-8)      /* request still running (epik2_poll) */
#define EPIK2_E_CANCELLED (-9) /* request cancelled before it ran */

/* limits */
#define EPIK2_MAX_SNPS (1 << 20)      /* i, j, k packed in 21 bits each for the argmin key */
#define EPIK2_MAX_SAMPLES (1 << 26)   /* counts and LUT index fit in 32 bits with margin */
#define EPIK2_MAX_TOPK 256

typedef struct epik2_ctx epik2_ctx;

/* Best triplet.  `score` is the K2 score in the reference CPU path's FP32 arithmetic
 * (CPU/v2.cpp:514-517); `score_fp64` is the same triplet rescored in FP64 on the GPU
 * (precision form) or NaN when not requested. */
typedef struct {
  float score;
  float _pad;
  double score_fp64;
  uint32_t i, j, k;
  uint32_t _pad2;
} epik2_best;

/* Scan options.  Zero-initialise and set what you need; 0 means "default". */
typedef struct {
  int32_t engine;      /* 0 = the context's default, 1 = integer pipe (LOP3+POPC), 2 = tensor cores
                          (int8), 3 = tensor cores (block-scaled FP4) */
  int32_t top_k;       /* 0/1 = best only; >1 = keep the top_k lowest FP32 scores */
  int32_t rescore_fp64;/* 1 = rescore the kept candidates in FP64 on the GPU */
  int32_t pair_tile;   /* tuning, tensor cores: SNPs j per tile, 32 (one CTA) or 64 (a cluster of two
                          CTAs sharing one tile, FP4 only); 0 = autotuned (with stage_words given and
                          pair_tile 0: 64 for FP4 at 16 words, else 32) */
  int32_t stage_words;  /* tuning, tensor cores: 32-sample words per pipeline stage, 4 or 8 (int8),
                           8 or 16 (FP4); 0 = autotuned */
  int32_t overlap;     /* tuning, FP4 on CTA pairs: 2 = the overlapped kernel (a tile's scoring runs
                          while the next tile counts; 4 or 8 words per stage; classes of at most
                          65535 samples), 1 = the sequential one, 0 = tuned */
  int64_t snp_begin;   /* restrict the first index i to [snp_begin, snp_end); 0,0 = all */
  int64_t snp_end;
} epik2_opts;

/* --------------------------------------------------------------------------------
 * Context.  Replaces the SYCL queue/device selection of GPU/v4.cpp:243-251.
 * ------------------------------------------------------------------------------ */
int epik2_create(epik2_ctx **out, int device);
void epik2_destroy(epik2_ctx *ctx);
const char *epik2_strerror(int status);
const char *epik2_last_error(const epik2_ctx *ctx);
/* Device name as the reference prints it ("Selected device: ...", GPU/v4.cpp:251). */
int epik2_device_name(const epik2_ctx *ctx, char *buf, size_t len);
/* Bytes of device memory currently free / total on the context's device. */
int epik2_mem_info(const epik2_ctx *ctx, size_t *free_bytes, size_t *total_bytes);

/* Default search engine of the context (EPIK2_ENGINE_*).  All engines give identical
 * tables, scores and triplets; AUTO takes the autotuner's choice for the dataset's shape. */
#define EPIK2_ENGINE_AUTO 0
#define EPIK2_ENGINE_INT 1 /* integer pipe: 8 LOP3+POPC per triplet and 32-sample word */
#define EPIK2_ENGINE_TC 2  /* tcgen05 int8 matrix products on 0/1 operands, int32 accumulators */
#define EPIK2_ENGINE_TC_FP4 3 /* tcgen05 block-scaled FP4 (E2M1 0/0.5, scales 2) products, FP32
                                 accumulators: exact while every class has < 2^24 samples,
                                 else EPIK2_E_TOO_LARGE */
int epik2_set_engine(epik2_ctx *ctx, int engine);
/* Default tensor-core stage depth of the context (used when epik2_opts.stage_words is 0):
 * 0 = autotuned, else 4 or 8 (int8) / 8 or 16 (FP4; 16 runs as clusters of two CTAs that
 * share one 64-pair tile). */
int epik2_set_stage_words(epik2_ctx *ctx, int stage_words);
/* Default tensor-core pair tile of the context (used when epik2_opts.pair_tile is 0): 0 =
 * autotuned, 32 or 64 (64 = FP4 on clusters of two CTAs). */
int epik2_set_pair_tile(epik2_ctx *ctx, int pair_tile);
/* Default of epik2_opts.overlap for the context: 0 = tuned, 1 = off, 2 = on. */
int epik2_set_overlap(epik2_ctx *ctx, int overlap);

/* Run the context's work on a caller-owned stream (e.g. a PyTorch stream); NULL restores
 * the context's own stream.  The library still synchronises that stream before it
 * returns results to the host. */
int epik2_set_stream(epik2_ctx *ctx, void *cuda_stream);
int epik2_get_stream(const epik2_ctx *ctx, void **cuda_stream);

/* Bounded device-side waits.  Every mbarrier wait of the tensor-core kernels gives up after
 * this many SM clocks: the kernel sets an error word, stops taking tiles, frees its tensor
 * memory and ends; the call returns EPIK2_E_TIMEOUT and the context stays usable (the
 * reference has no device-side wait to bound).  0 = the default, about 2 s. */
int epik2_set_wait_limit(epik2_ctx *ctx, int64_t sm_clocks);
/* Test hook of that error path (no reference counterpart): in the next tensor-core search
 * that runs on single CTAs (int8, or FP4 at 8 words per stage), one producing warp of the
 * first CTA leaves out its first "stage stored" arrival, so the issuing warp's wait expires
 * before any matrix product is issued and the search returns EPIK2_E_TIMEOUT.  One-shot:
 * the search after it runs normally. */
int epik2_test_withhold_arrival(epik2_ctx *ctx);

/* Counters kept by the context (no reference counterpart: the reference's only
 * instrument is a TSC timer around its launch loop, GPU/v4.cpp:282, 609). */
typedef struct {
  uint64_t kernel_launches;     /* CUDA kernels this library launched on the context */
  uint64_t h2d_bytes;           /* bytes copied host -> device */
  uint64_t d2h_bytes;           /* bytes copied device -> host */
  double last_scan_kernel_ms;   /* device time of the last search kernel (CUDA events on its stream) */
  int64_t last_scan_triplets;   /* triplets scored by the last search */
  int64_t last_scan_words;      /* 32-sample class words per triplet in the last search (both classes) */
  double last_load_ms;          /* host wall time of the last epik2_load_u8 (upload, encode, margins) */
  double last_upload_ms;        /* device time of its host -> device copies (CUDA events) */
  double last_prepare_ms;       /* device time of its encode and margin kernels, to their completion */
  double last_scan_wall_ms;     /* host wall time of the last epik2_scan (setup, search, reduction, read-back) */
} epik2_stats;
int epik2_get_stats(const epik2_ctx *ctx, epik2_stats *out);
int epik2_reset_stats(epik2_ctx *ctx);

/* --------------------------------------------------------------------------------
 * Data sources (host).  The reference synthesises its input inside main().
 * ------------------------------------------------------------------------------ */
/* The reference's generator: srand(100), geno[s][m] = rand()%3, exactly n/2 cases by
 * rejection sampling (GPU/v4.cpp:81-110).  pheno must hold n_samples bytes. */
int epik2_generate_reference(int64_t n_samples, int64_t n_snps, uint8_t *geno, uint8_t *pheno);
/* Seeded Hardy-Weinberg generator with planted triplets (benchmark workloads; no
 * reference counterpart).  planted = n_planted*3 SNP indices, effects = case
 * probability for carriers of each planted triplet. */
int epik2_generate_hwe(uint64_t seed, int64_t n_samples, int64_t n_snps, int64_t n_cases, double maf_lo,
                       double maf_hi, int32_t n_planted, const int64_t *planted, const double *effects,
                       uint8_t *geno, uint8_t *pheno);

/* --------------------------------------------------------------------------------
 * Datasets.  Replaces data_to_binary + binary_to_tiled + masks + the USM uploads
 * (GPU/v4.cpp:112-196, 220-238, 256-262): uploads the matrix, encodes per-class bit
 * planes on the GPU and keeps them resident until epik2_unload.
 * ------------------------------------------------------------------------------ */
int epik2_load_u8(epik2_ctx *ctx, const uint8_t *geno, const uint8_t *pheno, int64_t n_samples,
                  int64_t n_snps, int32_t *dataset_id);
/* Re-encode a resident dataset with a new phenotype vector (permutation replicate). */
int epik2_set_pheno(epik2_ctx *ctx, int32_t dataset_id, const uint8_t *pheno);
/* A new dataset that shares the genotype matrix of a resident dataset (no upload) and
 * has its own phenotype: the unit of a permutation-replicate scan (no reference
 * counterpart).  The genotype owner cannot be unloaded while replicates of it live
 * (EPIK2_E_BUSY). */
int epik2_load_replicate(epik2_ctx *ctx, int32_t base_dataset_id, const uint8_t *pheno, int32_t *dataset_id);
/* Device bytes a replicate of this shape holds (its planes and margins, not the shared
 * genotypes). */
int64_t epik2_replicate_bytes(int64_t n_samples, int64_t n_snps);
int epik2_unload(epik2_ctx *ctx, int32_t dataset_id);
/* n_samples, n_snps, n_cases, and device bytes held by the dataset. */
int epik2_dataset_info(const epik2_ctx *ctx, int32_t dataset_id, int64_t *n_samples, int64_t *n_snps,
                       int64_t *n_cases, int64_t *device_bytes);
/* Device bytes a dataset of this shape would hold (admission control). */
int64_t epik2_dataset_bytes(int64_t n_samples, int64_t n_snps);

/* --------------------------------------------------------------------------------
 * Search.  Replaces the host tile loop + kernel_epi + host argmin
 * (GPU/v4.cpp:283-608; same result as GPU/v2.cpp:260-565 with its lexicographic
 * tie-break).
 * ------------------------------------------------------------------------------ */
int epik2_scan(epik2_ctx *ctx, int32_t dataset_id, const epik2_opts *opts, epik2_best *out);
/* Top-k form: after a scan with opts->top_k = K, copy the K best (ascending FP32 score,
 * ties by index) into out[0..K).  *n_out receives the number written. */
int epik2_scan_topk(epik2_ctx *ctx, int32_t dataset_id, const epik2_opts *opts, epik2_best *out,
                    int32_t capacity, int32_t *n_out);
/* --------------------------------------------------------------------------------
 * Input files (no reference counterpart: the reference reads no files; its input is the
 * synthetic generate_data, GPU/v4.cpp:81-110).  PLINK 1 binary fileset <prefix>.bed/.bim/.fam:
 * the genotype is the count of the .bim's first allele (0, 1, 2); samples whose .fam
 * phenotype (column 6) is neither 2 (case) nor 1 (control) are left out; a missing
 * genotype takes `missing_genotype`.  epik2_plink_dims gives the sizes of the matrix that
 * epik2_read_plink fills (sample-major n_samples x n_snps bytes, n_samples phenotypes).
 * ------------------------------------------------------------------------------ */
int epik2_plink_dims(const char *prefix, int64_t *n_samples, int64_t *n_snps);
int epik2_read_plink(const char *prefix, uint8_t missing_genotype, uint8_t *geno, uint8_t *pheno);

/* Permutation test (no reference counterpart): p-value of an observed best score against
 * the best scores of phenotype-permutation replicates (epik2_load_replicate / the server's
 * replicate requests): (1 + #{replicate best <= observed}) / (1 + n_replicates); lower K2
 * is the stronger association.  -1 on invalid arguments. */
double epik2_perm_pvalue(float observed, const float *replicate_best, int64_t n_replicates);

/* One call from host buffers to the best triplet: load + scan + unload.  The context keeps
 * the dataset's device allocation for its next load (reused when it fits within twice the
 * size, else released first); epik2_destroy releases it. */
int epik2_scan_u8(epik2_ctx *ctx, const uint8_t *geno, const uint8_t *pheno, int64_t n_samples,
                  int64_t n_snps, const epik2_opts *opts, epik2_best *out);

/* --------------------------------------------------------------------------------
 * Batched form (no reference counterpart).  One persistent tensor-core launch over many
 * resident datasets: the triplet tiles of all of them go on one shared queue (datasets with
 * the most samples first), each CTA folds its candidates into per-dataset slots, and a
 * per-dataset reduction writes out[0..n).  The launch sequence is captured once per set of
 * dataset shapes into a CUDA graph and replayed (phenotype re-encodings via epik2_set_pheno
 * and new datasets of the same shapes are picked up).  One configuration (format, stage
 * depth, pair tile) serves the whole call: the requested one, else the one with the least
 * predicted time, sum over datasets of work / the autotuner's rate for the dataset's shape.
 * Each result equals epik2_scan on that dataset alone.  At most 512 datasets per call
 * (EPIK2_E_TOO_LARGE beyond).
 * ------------------------------------------------------------------------------ */
int epik2_scan_batch(epik2_ctx *ctx, const int32_t *dataset_ids, int32_t n, const epik2_opts *opts,
                     epik2_best *out);

/* Replicate form (no reference counterpart; the phenotype-mask idea of GPU/v1.cpp:264-289 on
 * tensor cores): the best triplet of each of n_reps phenotype-permutation replicates of a
 * resident dataset (phenos: n_reps x n_samples bytes, 1 = case).  Each tile of the search
 * counts the all-sample contingency cells of the base matrix once, then for every replicate
 * only its cases; its controls are the totals minus its cases.  Runs the FP4 CTA-pair kernel
 * (EPIK2_E_TOO_LARGE for classes of 2^24 samples or more), as many replicates per launch as
 * free device memory allows (at most 256).  out[r] equals epik2_scan of the dataset with
 * phenotype r; with opts->rescore_fp64, out[r].score_fp64 is its best triplet rescored in FP64
 * on the GPU (other options are ignored). */
int epik2_scan_replicates(epik2_ctx *ctx, int32_t dataset_id, const uint8_t *phenos, int32_t n_reps,
                          const epik2_opts *opts, epik2_best *out);

/* Autotuner (no reference counterpart).  Times nine configurations on a slice of the
 * dataset (about 1/64 of its triplets, at least a few tiles per SM): the integer engine; the
 * int8 tensor-core engine at 4 and 8 words (128 and 256 samples) per stage; and, when its
 * accumulators are exact for the dataset, the FP4 tensor-core engine at 8 and 16 words per
 * stage, each with a pair tile of 32 SNPs j (one CTA) and of 64 (a cluster of two CTAs), and
 * the overlapped FP4 CTA-pair kernel at 4 and 8 words per stage (classes <= 65535 samples).
 * Caches the fastest per shape bucket (log2 of samples and SNPs); EPIK2_ENGINE_AUTO scans and
 * the batched form use the cached rates.  Reports the choice and the measured rates
 * (triplet*samples/s; 0 = not a candidate).  The k-strip (SNPs k per tile: 128 int8, 112
 * FP4) is fixed by the tensor-memory budget: both classes' accumulators and the scale
 * factors fill 480 of the 512 columns. */
typedef struct {
  int32_t engine;        /* EPIK2_ENGINE_INT, EPIK2_ENGINE_TC or EPIK2_ENGINE_TC_FP4 */
  int32_t stage_words;   /* tensor-core stage depth chosen (int8: 4 or 8, FP4: 8 or 16) */
  double rate_int;       /* measured rates on the slice */
  double rate_tc4;       /* int8, 4 words per stage, 32 j */
  double rate_tc8;       /* int8, 8 words, 32 j */
  double rate_fp4_8;     /* FP4, 8 words, 32 j */
  double rate_fp4_16;    /* FP4, 16 words, 64 j (CTA pairs) */
  double rate_fp4_8_pair;    /* FP4, 8 words, 64 j (CTA pairs) */
  double rate_fp4_16_single; /* FP4, 16 words, 32 j */
  int32_t pair_tile;     /* pair tile chosen: 32 or 64 SNPs j */
  int32_t overlap;       /* 1 = the overlapped kernel was chosen */
  double rate_fp4_4_overlap; /* overlapped FP4 CTA-pair kernel, 4 words per stage */
  double rate_fp4_8_overlap; /* the same, 8 words per stage */
} epik2_tune;
int epik2_autotune(epik2_ctx *ctx, int32_t dataset_id, epik2_tune *out);

/* --------------------------------------------------------------------------------
 * Serving form (no reference counterpart).  A request server owns a device context and
 * one worker thread.  Requests arrive at any time from any thread: either a set of
 * phenotype-permutation replicates against a genotype matrix kept resident in HBM, or a
 * fresh genotype matrix with its phenotype.  The worker batches continuously: before each
 * batched launch it admits queued replicate scans (oldest first) while free device memory
 * (above a reserve), a work target per launch and a slot limit allow, so scans of
 * different requests run in the same launch; memory and slots freed by a launch admit the
 * next scans.  A request completes when all its scans have; its latency is completion
 * time minus submission time.
 * ------------------------------------------------------------------------------ */
typedef struct epik2_server epik2_server;
typedef struct {
  int64_t hbm_reserve_bytes; /* device memory left unused by admission; 0 = 2 GiB */
  double batch_work;         /* triplet*samples to aim for per launch; 0 = 2e13 */
  int32_t max_active;        /* scans per launch at most; 0 = 256 */
  int32_t max_queued;        /* queued scans beyond which submissions are refused; 0 = 1 << 20 */
  int32_t rescore_fp64;      /* 1 = FP64 rescore of every scan's best triplet */
  int32_t stage_words;       /* tensor-core stage depth, 0 = autotuned */
} epik2_server_opts;
typedef struct {
  int64_t submitted, completed, rejected, cancelled; /* requests */
  int64_t scans_queued, scans_active, scans_done;    /* single scans (replicates) */
  int64_t launches;
  double triplet_samples; /* completed work */
  double busy_seconds;    /* worker time inside batched launches */
  int64_t max_active;     /* most scans admitted to one launch so far */
  double kernel_seconds;  /* device time of the search kernels inside those launches */
  int64_t replicate_scans;/* scans that ran in the replicate form (epik2_scan_replicates) */
} epik2_server_stats;
int epik2_server_create(epik2_server **out, int device, const epik2_server_opts *opts);
void epik2_server_destroy(epik2_server *srv);
/* Keep a genotype matrix (with a reference phenotype) resident for replicate requests. */
int epik2_server_add_matrix(epik2_server *srv, const uint8_t *geno, const uint8_t *pheno, int64_t n_samples,
                            int64_t n_snps, int32_t *matrix_id);
/* phenos: n_replicates x n_samples bytes, one phenotype per replicate. */
int epik2_server_submit_replicates(epik2_server *srv, int32_t matrix_id, const uint8_t *phenos,
                                   int32_t n_replicates, int64_t *request_id);
int epik2_server_submit_scan(epik2_server *srv, const uint8_t *geno, const uint8_t *pheno, int64_t n_samples,
                             int64_t n_snps, int64_t *request_id);
/* EPIK2_E_BUSY while the request runs; EPIK2_OK once done: out[r] = best triplet of scan r
 * (r < min(capacity, scans)), *latency_seconds set, and the request record released.
 * A refused or failed request reports its status here. */
int epik2_server_poll(epik2_server *srv, int64_t request_id, epik2_best *out, int32_t capacity, int32_t *n_out,
                      double *latency_seconds);
int epik2_server_cancel(epik2_server *srv, int64_t request_id);
int epik2_server_get_stats(epik2_server *srv, epik2_server_stats *out);

/* --------------------------------------------------------------------------------
 * Parity / inspection.  The reference keeps tables in registers (GPU/v4.cpp:317);
 * these expose the same counts and scores computed by the search kernel itself.
 * ------------------------------------------------------------------------------ */
/* Every triplet's 54 counts and FP32 score, at its lexicographic index
 * t(i,j,k) among the C(n_snps,3) triplets.  tables: C(M,3)*54 uint32 (may be NULL),
 * scores: C(M,3) float (may be NULL).  Limited to n_snps <= 512. */
int epik2_dump_tables(epik2_ctx *ctx, int32_t dataset_id, uint32_t *tables, float *scores);
/* Tables of an explicit list of triplets (n x 3 SNP indices). */
int epik2_tables(epik2_ctx *ctx, int32_t dataset_id, const uint32_t *triplets, int64_t n, uint32_t *tables);
/* The FP32 log-factorial lookup table used by the score, lut[0..n_max]. */
int epik2_k2_lut(int64_t n_max, float *lut);

/* --------------------------------------------------------------------------------
 * Allocation-free search.  No counterpart in the reference.
 * ------------------------------------------------------------------------------ */
#define EPIK2_NOALLOC_SCRATCH_BYTES (64u << 20)
/* Same result as epik2_scan_u8, for callers that cannot allocate device memory -- e.g.
 * code running inside a host application that owns the device heap, or under a device
 * memory budget fixed before this library is reached.  Creates no context and calls no
 * cudaMalloc/cudaFree or other allocating routine: every intermediate lives in one static
 * device array of EPIK2_NOALLOC_SCRATCH_BYTES (64 MiB) that each GPU loading this library
 * holds until the process exits.  Runs on the current device, on `cuda_stream` (NULL =
 * the default stream), and returns once the result is on the host.
 *   - Every call looks up the array's device address in the current context, so it stays
 *     valid across a device reset.  No call may be stream-captured: each one waits for its
 *     stream and copies through pageable host memory; a stream under capture is refused
 *     with EPIK2_E_INVALID before anything is enqueued.
 *   - A call that fails after enqueuing work waits for its stream before it returns.
 *   - All calls share the array, which keeps the last call's contents (each call clears
 *     what must start at zero).  Calls whose GPU work overlaps race on it.
 *   - Shapes whose buffers do not fit (about n_samples*n_snps + 16*n_snps^2 bytes plus
 *     n_samples*n_snps/4) or with more than 4096 SNPs return EPIK2_E_TOO_LARGE. */
int epik2_scan_u8_noalloc(const uint8_t *geno, const uint8_t *pheno, int64_t n_samples, int64_t n_snps,
                          void *cuda_stream, epik2_best *out);

#ifdef __cplusplus
}
#endif
#endif /* EPIK2_H */
