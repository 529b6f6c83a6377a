/*
 * cuapss.h -- C ABI of the B200-native hybrid all-pairs cosine similarity
 * search (APSS).
 *
 * Input : a CSR matrix of L2-normalised sparse vectors (n rows, d features,
 *         int64 row pointers, int32 feature ids sorted ascending in each row,
 *         float32 values) and a threshold t.
 * Output: every unordered pair (i, j), i < j, whose cosine similarity
 *         (= dot product of the normalised rows) is >= t, with its similarity.
 *
 * This replaces the single entry point of the reference,
 *   void similarity_join_device(int* dim_A, float* feature_A, int* tile_start_A,
 *                               ... x8 partitions ..., int* b_id_a,
 *                               int* apss_block_seg, int* apss_seg_start)
 * (similarity_search.h:3-14, defined similarity_search.cu:934-3014), which
 * takes a tile-ELL layout of 8 fixed partitions, allocates its own device
 * memory, returns void and only prints pair counts. The reference's
 * signature itself is kept as a compatibility shim, cuapss_compat.h.
 *
 * Conventions
 *  - Every call returns a cuapss_status. Nothing is printed.
 *  - A context owns one CUDA stream (its own or the caller's) and is used by
 *    one host thread at a time.
 *  - Pointers flagged on_device are CUDA device pointers on the context's
 *    device; otherwise they are host pointers (pinned or pageable).
 *  - Pair output is sorted by (i, j) ascending, i < j, in the caller's row
 *    numbering. If the caller's capacity is too small the call returns
 *    CUAPSS_EOVERFLOW with pairs->count set to the required capacity; the
 *    caller retries with a larger buffer (the search is deterministic).
 *  - Exactness contract: the emitted pair set equals the set of pairs whose
 *    similarity, accumulated in FP64 from the FP32 inputs in ascending
 *    feature-id order, is >= t. Each reported similarity is within 1e-6 of
 *    that FP64 value.
 */
#ifndef CUAPSS_H_
#define CUAPSS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CUAPSS_ABI_VERSION 2

typedef enum {
  CUAPSS_OK = 0,
  CUAPSS_EINVAL = 1,    /* malformed CSR, bad option, not normalised, bad t */
  CUAPSS_ENOMEM = 2,    /* device or host allocation failed */
  CUAPSS_EOVERFLOW = 3, /* output capacity too small; count = required */
  CUAPSS_ETIMEOUT = 4,  /* a bounded device or host wait gave up */
  CUAPSS_ECUDA = 5,     /* a CUDA runtime call failed */
  CUAPSS_EBUSY = 6      /* admission refused: HBM budget or queue full */
} cuapss_status;

typedef enum {
  CUAPSS_PREC_FP32 = 0,  /* plain FP32 hybrid: head on the forward-list dot */
  CUAPSS_PREC_MIXED = 1  /* BF16 head on tcgen05, FP32 tail, FP64 rescore  */
} cuapss_precision;

typedef struct {
  int device;          /* CUDA device ordinal */
  void* stream;        /* cudaStream_t to launch on; NULL: context creates one */
  int precision;       /* cuapss_precision */
  int head_width;      /* p, the number of most frequent features handled by
                          the pair-parallel head; 0 = autotuner picks */
  int remap;           /* 1 (default): frequency-ordered feature remap;
                          0: identity, head = feature ids < p (reference rule) */
  int validate;        /* 1 (default): check CSR structure and row norms */
  float norm_tol;      /* accepted | ||x||_2 - 1 | (default 1e-4) */
  int verbose;         /* reserved, 0 */
  int rare_max_count;  /* self-joins: features occurring in at most C rows
                          have their pairs enumerated instead of probed.
                          0 (default): C chosen with p by the cost model;
                          -1: none; C in {16, 32, ..., 2048}: that C */
} cuapss_opts;

typedef struct {
  int64_t n;              /* rows (vectors) */
  int64_t d;              /* features (dimension) */
  int64_t nnz;            /* non-zeros */
  const int64_t* rowptr;  /* [n+1] */
  const int32_t* col;     /* [nnz] feature ids, strictly ascending per row */
  const float* val;       /* [nnz] */
  int on_device;          /* 1: the three arrays are device pointers */
} cuapss_csr;

typedef struct {
  int32_t* i;        /* [capacity] first row id  (i < j) */
  int32_t* j;        /* [capacity] second row id */
  float* sim;        /* [capacity] similarity */
  int64_t capacity;  /* entries available in i, j, sim */
  int64_t count;     /* out: pairs found (required capacity on EOVERFLOW) */
  int on_device;     /* 1: i, j, sim are device pointers */
} cuapss_pairs;

typedef struct {
  int64_t pairs;          /* pairs emitted (sim >= t) */
  int64_t candidates;     /* pairs that left the tile epilogue */
  int64_t rescored;       /* candidates inside the error band, redone in FP64 */
  int64_t tiles;          /* 128x128 pair tiles evaluated */
  int64_t head_width;     /* p used */
  int64_t tail_entries;   /* non-zeros outside the head */
  int64_t tail_products;  /* sum over tail features of L(L-1)/2 */
  double max_band;        /* largest error margin used by the epilogue */
  double ms_preprocess;   /* validate + remap + row order + norms + layout */
  double ms_index;        /* inverted lists (block-local and global) */
  double ms_tiles;        /* head dot + tail scan + epilogue */
  double ms_finalize;     /* rescore, compensated re-score, sort, copy-out */
  double ms_total;
  int64_t launches;       /* CUDA kernels this call launched */
  int64_t explicit_pairs; /* rare-feature pairs enumerated instead of probed */
  int64_t rare_max_count; /* their features occur in at most this many rows
                             (0: every tail feature probed) */
} cuapss_stats;

typedef struct cuapss_ctx cuapss_ctx;

/* Defaults for cuapss_opts (device 0, own stream, FP32, autotuned p, remap,
 * validation on, norm_tol 1e-4). */
void cuapss_default_opts(cuapss_opts* opts);

/* Human-readable name of a status code. */
const char* cuapss_status_string(cuapss_status s);

/* Runtime ABI version (CUAPSS_ABI_VERSION of the built library). */
int cuapss_abi_version(void);

/* Create / destroy a context. Replaces the allocation prologue and the
 * (partial) frees of similarity_join_device (similarity_search.cu:946-1075,
 * 2996-3013). */
cuapss_status cuapss_create(cuapss_ctx** ctx, const cuapss_opts* opts);
cuapss_status cuapss_destroy(cuapss_ctx* ctx);

/* Self-join: all pairs i < j of `x` with sim >= t. Replaces the eight
 * intra-partition "apss" pipelines of similarity_join_device
 * (similarity_search.cu:2650-2993) and, since the whole input is one matrix,
 * also the 28 cross-partition joins (similarity_search.cu:1273-2632).
 * `stats` may be NULL. Synchronous: returns when `out` is filled. */
cuapss_status cuapss_run(cuapss_ctx* ctx, const cuapss_csr* x, float t,
                         cuapss_pairs* out, cuapss_stats* stats);

/* One shard of cuapss_run, for one process per GPU with no exchange between
 * them: the pairs (i, j), i < j, of the self-join whose row i lies in a
 * 128-row block b = i / 128 with b mod nshards == shard. The shards of
 * 0..nshards-1 are disjoint and their union is cuapss_run's output; every
 * shard prepares the whole matrix and evaluates about 1/nshards of the pair
 * tiles. The reference splits its input into 8 fixed partitions and joins
 * them one after another on one GPU (similarity_search.cu:1273-2993). */
cuapss_status cuapss_run_shard(cuapss_ctx* ctx, const cuapss_csr* x, float t,
                               int32_t shard, int32_t nshards, cuapss_pairs* out,
                               cuapss_stats* stats);

/* Row blocks owned by a shard of an n-row self-join (host only): writes up
 * to `capacity` block indices to blocks (may be NULL) and returns how many
 * there are, or -1 for bad arguments. */
int32_t cuapss_shard_blocks(int64_t n, int32_t shard, int32_t nshards, int32_t* blocks,
                            int64_t capacity);

/* Self-check of failure detection: every device wait of the tile kernels is
 * bounded by device time (mbarrier try-wait against a %globaltimer deadline
 * of 2 s) and reports CUAPSS_ETIMEOUT instead of hanging. This runs a kernel
 * that waits, with the same primitive and a deadline of limit_us
 * microseconds (1 .. 2,000,000), on a barrier that nothing completes; it
 * returns CUAPSS_ETIMEOUT when the wait gave up and reported it as designed
 * (any other status is a failure), and *waited_ns (may be NULL) the device
 * time from the first poll to the give-up. The context stays usable. No
 * counterpart in the reference, whose waits are blocking host syncs. */
cuapss_status cuapss_selftest_bounded_wait(cuapss_ctx* ctx, int32_t limit_us,
                                           int64_t* waited_ns);

/* Cross-join: all pairs (a, b), a row of `a`, b row of `b`, sim >= t.
 * out->i holds the row of `a`, out->j the row of `b`; sorted by (i, j).
 * This is the per-partition-pair join of the reference
 * (similarity_join1 / filter_pair / similarity_join_rest,
 * similarity_search.cu:370-531, launched at 1273-2632). */
cuapss_status cuapss_join(cuapss_ctx* ctx, const cuapss_csr* a,
                          const cuapss_csr* b, float t, cuapss_pairs* out,
                          cuapss_stats* stats);

/* ---- Resident index for serving ------------------------------------------
 * An index keeps a matrix resident in HBM, prepared for repeated query
 * batches: the frequency remap (fixed at creation), the dense head block and
 * the tail inverted lists of its rows, and a copy of its CSR for the exact
 * finalize. Appends add rows as a new immutable segment (its lists are built
 * for the new rows only); segments of similar size are merged, so an index of
 * N rows has O(log N) segments. A query batch (q rows, each with its own
 * threshold t[i]) returns every (query row i, index row j) with
 * sim >= t[i], sorted by (i, j), under the exactness contract above.
 *
 * Concurrency: one index may be queried from several contexts (host threads,
 * streams) at once and appended to from one of them; a query sees the
 * segments that existed when it started. The index's device and precision
 * are those of the context that created it; contexts used with it must be on
 * the same device.
 *
 * The reference has no resident index: similarity_join_device rebuilds every
 * partition's index on each call (similarity_search.cu:1075-1272). */
typedef struct cuapss_index cuapss_index;

/* Build an index over the rows of x (host or device CSR; copied). */
cuapss_status cuapss_index_create(cuapss_ctx* ctx, const cuapss_csr* x,
                                  cuapss_index** idx);

/* Append the rows of x (same d) as index rows [rows, rows + x->n). */
cuapss_status cuapss_index_append(cuapss_ctx* ctx, cuapss_index* idx,
                                  const cuapss_csr* x);

/* Query batch: q rows against the index, t[i] (host array of q->n floats,
 * each > 0) the threshold of query row i. out->i = query row, out->j = index
 * row. Synchronous on ctx's stream. */
cuapss_status cuapss_index_query(cuapss_ctx* ctx, const cuapss_index* idx,
                                 const cuapss_csr* q, const float* t,
                                 cuapss_pairs* out, cuapss_stats* stats);

/* Rows, segments, head width and device bytes held by the index (any
 * pointer may be NULL). */
cuapss_status cuapss_index_info(const cuapss_index* idx, int64_t* rows,
                                int32_t* segments, int32_t* head_width,
                                int64_t* device_bytes);

cuapss_status cuapss_index_destroy(cuapss_index* idx);

/* ---- Request server over a resident index (continuous batching) ----------
 * Requests (query batches with per-query thresholds, or appends) are queued
 * as they arrive. Each of `lanes` host threads owns a context (its own
 * stream and working memory); whenever a lane is free it merges the queued
 * query requests, in arrival order, into one batch (at most max_batch_rows
 * query rows, and admitted only while the estimated working memory of all
 * batches in flight stays within hbm_budget) and runs it, so requests that
 * arrive while others are on the GPU join the next batch and batches of
 * different lanes overlap on the device. Appends are applied in submission
 * order, one at a time; a query sees the rows appended before its batch
 * started (cuapss_request_info.index_rows). No counterpart in the reference,
 * which has no request path. */
typedef struct cuapss_server cuapss_server;

typedef struct {
  int32_t lanes;           /* batches in flight, default 3 */
  int64_t max_batch_rows;  /* query rows per batch, default 1024 (bounds the
                              time one batch holds the GPU) */
  int64_t hbm_budget;      /* working-memory bytes of batches in flight,
                              default 16 GiB */
} cuapss_server_opts;

typedef struct {
  cuapss_status status;  /* the request's own outcome */
  int64_t pairs;         /* pairs of this request */
  double queue_ms;       /* submit -> its batch started */
  double latency_ms;     /* submit -> results ready */
  int64_t batch_id;      /* batch it ran in (query requests) */
  int64_t batch_rows;    /* query rows of that batch */
  int64_t index_rows;    /* index rows it was matched against / after append */
} cuapss_request_info;

void cuapss_server_default_opts(cuapss_server_opts* o);

/* The server uses idx (which must outlive it) on `device`. */
cuapss_status cuapss_server_create(cuapss_server** s, cuapss_index* idx, int device,
                                   const cuapss_server_opts* o);

/* Queue a query request: q (host CSR, copied) with thresholds t[q->n]. */
cuapss_status cuapss_server_submit_query(cuapss_server* s, const cuapss_csr* q,
                                         const float* t, uint64_t* ticket);

/* Queue an append of the rows of x (host CSR, copied). */
cuapss_status cuapss_server_submit_append(cuapss_server* s, const cuapss_csr* x,
                                          uint64_t* ticket);

/* Wait up to timeout_ms (< 0: no limit) for a request. On success its pairs
 * (query rows numbered within the request) are copied to out (host arrays)
 * and the request is released; CUAPSS_EOVERFLOW sets out->count to the
 * required capacity and keeps the request; CUAPSS_ETIMEOUT if not done. */
cuapss_status cuapss_server_wait(cuapss_server* s, uint64_t ticket, int32_t timeout_ms,
                                 cuapss_pairs* out, cuapss_request_info* info);

/* Finishes the queued requests, stops the lanes, frees the server. */
cuapss_status cuapss_server_destroy(cuapss_server* s);

/* Size buckets of the batched self-join (instance rows n):
 * bucket 0: n <= 1024, bucket 1: n <= 8192, bucket 2: larger. */
#define CUAPSS_BATCH_BUCKETS 3

/* Batched self-joins of k independent instances: instance q is the row range
 * [inst_ptr[q], inst_ptr[q+1]) of `x` (inst_ptr[0] = 0, inst_ptr[k] = x->n,
 * non-decreasing; host array) with its own threshold t[q] (host array, each
 * > 0). Pairs never cross instances. Output as cuapss_run: (i, j, sim) in
 * x's row numbering, i < j, sorted by (i, j), so grouped by instance. All
 * instances share the feature remap; each size bucket gets its own head
 * width p (opts.head_width if set, else the context's autotuner, which times
 * candidate widths on a sample of the bucket the first time it meets a bucket
 * with those nnz statistics and keeps the winner). The tile launches of all
 * buckets run as one CUDA graph launch. bucket_p (may be NULL) receives the
 * width used per bucket (0: bucket empty). The reference runs its 8
 * partition self-joins one after another, two launches and host syncs each
 * (similarity_search.cu:2650-2993); it has no batched form. */
cuapss_status cuapss_batch_run(cuapss_ctx* ctx, const cuapss_csr* x, int32_t k,
                               const int64_t* inst_ptr, const float* t,
                               cuapss_pairs* out, cuapss_stats* stats,
                               int32_t* bucket_p);

/* Inverted index of the tail features, reference semantics: for every
 * feature f with f >= p (on the caller's ids, no remap), the rows that
 * contain f and their values, lists sorted by row. dim_ptr has d+1 entries
 * (exclusive scan of the per-feature counts; features < p have empty lists).
 * Replaces generate_index_ptr4 + the host scan + construct_Index2
 * (similarity_search.cu:105-191, 1168-1186, 221-274), whose list order is
 * nondeterministic; sorted by row the two are equal. All arrays are device
 * pointers if x->on_device, else host. idx_row/idx_val need capacity
 * >= number of tail non-zeros (returned in *tail_nnz; EOVERFLOW if short). */
cuapss_status cuapss_build_index(cuapss_ctx* ctx, const cuapss_csr* x,
                                 int32_t p, int32_t* dim_ptr, int32_t* idx_row,
                                 float* idx_val, int64_t capacity,
                                 int64_t* tail_nnz);

/* The plan cuapss_run makes for a self-join (default options, one shard),
 * from the posting counts alone, on the host, with no device: counts[f] =
 * the number of rows that contain feature f (d entries), n rows. Writes the
 * head width p, the rare-feature threshold C (0: none) and the number of
 * explicit pairs C implies (before the head's features are taken out).
 * max_pairs bounds the explicit pairs (<= 0: the library's bound; the run
 * also bounds them by free device memory). No reference counterpart. */
cuapss_status cuapss_plan_self_join(int32_t precision, int64_t n, int64_t d,
                                    const int32_t* counts, int64_t max_pairs,
                                    int32_t* head_width, int32_t* rare_max_count,
                                    int64_t* explicit_pairs);

/* Frequency-ordered feature remap: perm[f] = rank of feature f when features
 * are sorted by (posting count descending, id ascending); counts[f] = the
 * posting count. Device pointers if x->on_device. (No counterpart in the
 * reference, which fixes the head to ids < 4096.) */
cuapss_status cuapss_feature_remap(cuapss_ctx* ctx, const cuapss_csr* x,
                                   int32_t* perm, int32_t* counts);

/* The same remap as cuapss_feature_remap, with no device allocation: for
 * callers whose device memory belongs to another allocator or whose latency
 * path forbids cudaMalloc/cudaFree. x, perm and counts must be device
 * pointers on ctx's device (x->on_device = 1); all other memory is a fixed
 * ~1.6 MB file-scope device array, so d <= 65536 (larger d: CUAPSS_EINVAL).
 * Each call looks up that array's address on its device; the first call on a
 * device can load the module and should come before any stream capture. The
 * call returns once its work on ctx's stream is done (the host waits for it).
 * Calls that overlap on the GPU share the array and race: serialise them. If
 * the call returns CUAPSS_EINVAL for a bad column id or an unsorted row,
 * perm and counts are undefined. No counterpart in the reference. */
cuapss_status cuapss_feature_remap_noalloc(cuapss_ctx* ctx, const cuapss_csr* x,
                                           int32_t* perm, int32_t* counts);

#ifdef __cplusplus
}
#endif

#endif /* CUAPSS_H_ */
