/*
 * bm25_b200.h -- C ABI of the B200 BM25 Search engine (libbm25_b200.so).
 *
 * Plain pointers and sizes only; no CUDA or C++ types in the signatures, so the
 * library can be bound from C, C++ (AscendIndexBm25.h), Python ctypes or any FFI.
 *
 * Ranking contract (same as the reference): per query the K documents with the
 * highest FP32 score, ties broken by ascending document id; documents with
 * score zero tie with each other and fill the remaining ranks by ascending id.
 * Per-document scores are the FP32 sum of the query terms' posting scores added
 * in query-term order (duplicates added again, unknown word ids skipped), so
 * they are bit-identical to the reference's CPU search
 *   feature_retrieval/src/ascendfaiss/test/ascendhost/bm25/reference/cpu_index_search.h:170-190.
 *
 * Status codes mirror the IndexSDK APP_ERR mapping of
 *   feature_retrieval/src/ascendfaiss/ascendhost/include/impl/Bm25ErrorAdapter.h:11-45
 * (InvalidArgument -> INVALID_PARAM, InvalidState -> ILLEGAL_OPERATION,
 *  DeviceError/other -> INNER_ERROR).
 *
 * Threading: every call on one handle is serialised by a mutex inside the handle
 * (the reference serialises AscendIndexBm25 the same way, AscendIndexBm25.cpp:26).
 */
#ifndef BM25_B200_H
#define BM25_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BM25_OK 0
#define BM25_ERR_INVALID_PARAM 1     /* bad input; the handle stays usable */
#define BM25_ERR_ILLEGAL_OPERATION 2 /* closed, failed or uninitialised handle */
#define BM25_ERR_INNER_ERROR 3       /* device / runtime failure; the handle is poisoned */

typedef struct bm25_handle bm25_handle;

/* Session configuration (replaces Bm25Config, AscendIndexBm25.h:17-25). */
typedef struct bm25_options {
    int32_t device_id;       /* CUDA device ordinal (Bm25Config::deviceId) */
    int32_t max_k;           /* largest K a Search may ask for (Bm25Config::topK); 1..32, or up to 1024 with
                                the warp-tile and tile-group kernels */
    int64_t query_capacity;  /* largest query batch (Bm25Config::queryCount) */
    int64_t word_capacity;   /* largest total word count per batch (Bm25Config::maxQueryWords) */
    int32_t tile_docs;       /* documents per scoring tile; 0 = automatic (power of two, 2048..32768) */
    int32_t merge_fan_in;    /* lists merged per tree node; 0 = automatic (2..32) */
    int64_t directory_bytes; /* byte budget of the per-tile posting directory; 0 = automatic */
    void *stream;            /* borrowed cudaStream_t, or NULL for an engine-owned stream */
    int32_t kernel;          /* BM25_KERNEL_*: search kernel; bm25_default_options picks BM25_KERNEL_WARP_TILE */
    int32_t ring_stages;     /* posting-ring depth of the ring kernels (0 and 4), 2..8; 0 = automatic */
    int32_t ring_chunk;      /* postings per ring stage of the tile-group kernel, 512..4096, a multiple of 4;
                                0 = automatic */
    int32_t prune;           /* nonzero: build the 128-document block-max index and the term statistics of
                                the pruned and learned Searches (tile-group kernel only) */
    int64_t candidate_capacity; /* max_k > 32: candidates kept per query (0 = automatic, 512 K and at least
                                   2^18); a query that overflows it is searched again from its final bound.
                                   A Search whose K-th score is tied by more documents than this overflows
                                   every retry pass and fails with BM25_ERR_INNER_ERROR (device status 32) */
    float prune_route;       /* pruned Searches of 32 queries or more: a query keeping more than this share of
                                its 128-document blocks is streamed instead of block-scored (0 = the
                                kernel's default: never for the warp-tile kernel, whose block scorer reads
                                each word's run of kept blocks at the streaming rate; 0.3 for the others;
                                negative or >= 1 = never) */
    int64_t wait_budget_cycles; /* SM clock cycles a bounded wait of the ring kernels (0 and 4) spends
                                   before it gives up and the Search reports a device error
                                   (0 = 4e9, about 2 s) */
    float dense_density;     /* warp-tile kernel: a term whose postings cover at least this share of the
                                documents is also kept as a dense FP32 row of per-document scores (zero
                                where absent), read with 128-bit loads instead of scattered
                                (0 = 0.25: such a row is at most twice the bytes of the postings it
                                replaces and a quarter of the instructions; negative = none) */
} bm25_options;

/* Search kernels (bm25_options.kernel):
 *   BM25_KERNEL_STREAM     persistent kernel, 2048-8192-document tiles, one posting ring per CTA
 *   BM25_KERNEL_PER_TILE   one CTA per (query, tile) and an in-launch merge tree
 *   BM25_KERNEL_TILE_GROUP persistent kernel, 1024-document tiles, one warp per tile of an
 *                          8-tile group fed by one bulk copy per query word
 *   BM25_KERNEL_WARP_TILE  persistent kernel, 1024-document tiles, every warp takes its own claims
 *                          (a query and 4 consecutive tiles) and loads its postings itself, the
 *                          claim's posting runs prefetched into L2 (the default) -- for plain
 *                          Searches with one K <= 32; pruned Searches, batches with a K per query
 *                          and K > 32 run the tile-group kernel */
#define BM25_KERNEL_STREAM 0
#define BM25_KERNEL_PER_TILE 1
#define BM25_KERNEL_TILE_GROUP 4
#define BM25_KERNEL_WARP_TILE 5

/* Fills defaults: device 0, max_k 10, 8 queries, 24 words (the reference's Bm25Config defaults),
 * the warp-tile kernel. */
void bm25_default_options(bm25_options *options);

/*
 * Creates a resident index from an eager CSC matrix (the bm25s layout,
 * reference_only/bm25s_original/bm25s/scoring.py:371-410):
 *   indptr  int64 [vocab + 1], indptr[0] = 0, non-decreasing, indptr[vocab] = M
 *   indices int32 [M], doc ids in [0, num_docs), strictly ascending within a term
 *   data    float [M], finite and >= 0 (precomputed per-posting BM25 scores)
 * The arrays are validated and copied to the device; the caller keeps ownership.
 * Replaces Init's index upload (AscendIndexBm25.cpp:33-48, large_search.cpp:107-188).
 */
int bm25_create(const int64_t *indptr, const int32_t *indices, const float *data, int64_t vocab, int64_t num_docs,
                const bm25_options *options, bm25_handle **out);

/*
 * Creates a resident index from the reference's lazy index
 * (common/bm25/index_data.h:9-42; files of standalone/resident_index.py:12-18):
 *   term_offsets int64 [vocab + 1], posting_doc_ids int32 [M], posting_tf float [M],
 *   doc_norm float [num_docs], idf float [vocab]
 * validated with the reference's rules, then turned into eager FP32 posting scores
 * on the GPU with the reference's expression (idf * (tf * f32(k1 + 1))) / (tf + norm)
 * (ops/ascendc/bm25/fused/op_kernel/bm25_fused_score_top_k.cpp:738-739); k1 = 1.2
 * reproduces the reference's 2.2F literal.
 */
int bm25_create_lazy(const int64_t *term_offsets, const int32_t *posting_doc_ids, const float *posting_tf,
                     const float *doc_norm, const float *idf, int64_t vocab, int64_t num_docs, float k1,
                     const bm25_options *options, bm25_handle **out);

/*
 * Search with host buffers (replaces Session::Search, large_search.cpp:190-212):
 *   qoffsets int64 [q + 1] (qoffsets[0] = 0, non-decreasing), words int32 [qoffsets[q]]
 *   (the packed layout of common/bm25/search_inputs.h:23-42), 1 <= q <= query_capacity,
 *   qoffsets[q] <= word_capacity, at most 64 words per query, every word in [0, INT32_MAX - 1];
 *   1 <= k <= min(max_k, num_docs).
 * Writes out_scores[q * k] and out_ids[q * k] only on success.  One CUDA-graph
 * replay: query H2D, scoring + selection + merge tree, result D2H; then the
 * result is validated on the host (large_search.cpp:64-85).
 */
int bm25_search(bm25_handle *handle, const int64_t *qoffsets, const int32_t *words, int64_t q, int32_t k,
                float *out_scores, int32_t *out_ids);

/*
 * Device-resident variant for callers that keep queries and results in HBM:
 * all four arrays are device pointers; work is enqueued on `stream` (a
 * cudaStream_t, NULL = the handle's stream) and the call returns without
 * synchronising.  No host validation of the device inputs: words outside the
 * vocabulary are skipped, negative words set the device status that
 * bm25_device_status reports.
 */
int bm25_search_device(bm25_handle *handle, const int64_t *qoffsets, const int32_t *words, int64_t q, int32_t k,
                       float *out_scores, int32_t *out_ids, void *stream);

/*
 * Pruned device-resident Search (no counterpart in the reference; the learned
 * part of the engine).  As bm25_search_device, plus tau float [q]: a starting
 * lower bound guess for each query's K-th score (e.g. the threshold MLP's
 * prediction).  Tiles whose FP32 upper bound (the query words' per-tile maxima
 * added in query-word order) is below a query's running bound -- which starts
 * at tau -- are skipped.  out_exact int32 [q]: 1 where K documents reached tau,
 * which proves the pruned top-K exact; 0 where the guess was too high, and a
 * retry pass in the same call searched the query again on the plain path.
 * Every output row is the exact top-K.  Needs a session created with
 * options.prune = 1 and the tile-group kernel.
 */
int bm25_search_pruned_device(bm25_handle *handle, const int64_t *qoffsets, const int32_t *words, const float *tau,
                              int64_t q, int32_t k, float *out_scores, int32_t *out_ids, int32_t *out_exact,
                              void *stream);

/* Pruned Search on host buffers (as bm25_search, plus tau [q] and out_exact [q]; one graph replay). */
int bm25_search_pruned(bm25_handle *handle, const int64_t *qoffsets, const int32_t *words, const float *tau,
                       int64_t q, int32_t k, float *out_scores, int32_t *out_ids, int32_t *out_exact);

/*
 * A batch with a K per query (no counterpart in the reference; the tile-group
 * kernel): ks int32 [q], each in [1, min(max_k, N)].  Results are packed by
 * query: query i's ks[i] (score, id) pairs start at ks[0] + ... + ks[i-1].
 * One graph replay covers the whole batch.
 */
int bm25_search_batch(bm25_handle *handle, const int64_t *qoffsets, const int32_t *words, const int32_t *ks,
                      int64_t q, float *out_scores, int32_t *out_ids);

/*
 * A batch runs in the CUDA graph of its capacity bucket: the query count rounded up to
 * a power of two (at most query_capacity) and the largest K rounded up to 32, 128 or
 * 1024 (at most max_k); the extra queries are empty.  Graphs are instantiated on first
 * use and at most 64 are kept (the least recently used is dropped).
 * bm25_prepare_batch_graphs instantiates every bucket's graph for batches of up to
 * max_batch queries (learned: the learned variant), so that a serving loop never
 * instantiates one on its request path; bm25_server_create calls it.
 */
int bm25_prepare_batch_graphs(bm25_handle *handle, int32_t max_batch, int32_t learned);

/* bm25_search_batch with the learned bounds; out_exact int32 [q] as bm25_search_pruned. */
int bm25_search_batch_learned(bm25_handle *handle, const int64_t *qoffsets, const int32_t *words, const int32_t *ks,
                              int64_t q, float *out_scores, int32_t *out_ids, int32_t *out_exact);

/*
 * Device-resident batch with a K per query: ks int32 [q] and kout int64 [q] (query
 * i's first output slot) on the device; kmax (host) at least every ks[i]; the
 * output buffers hold kout[i] + ks[i] entries for every i.  learned != 0: learned
 * bounds and out_exact int32 [q].  Asynchronous on stream.
 */
int bm25_search_batch_device(bm25_handle *handle, const int64_t *qoffsets, const int32_t *words, const int32_t *ks,
                             const int64_t *kout, int64_t q, int32_t kmax, int32_t learned, float *out_scores,
                             int32_t *out_ids, int32_t *out_exact, void *stream);

/*
 * Exact merge of per-shard top-K lists on device buffers (replaces the reference's
 * MergePrepare / bm25_top_k_merge, ascendhost/src/bm25/fused_runtime.h:33-34,
 * ops/ascendc/bm25/merge/op_kernel/bm25_top_k_merge.cpp:10-86): scores/ids
 * [q][shards][k] ([shards][q][k] when shard_major, an all-gather's layout), each
 * list sorted by (score desc, id asc) over a disjoint document range; bases int32
 * [shards] (device) is added to each list's ids, or NULL when the ids are already
 * global; out [q][k].  A list that is not a valid
 * strict ranking makes that query's output row -1.  Asynchronous on stream;
 * errors are read with bm25_last_error(NULL, ...).
 */
int bm25_merge_topk(const float *scores, const int32_t *ids, const int32_t *bases, int64_t q, int32_t shards,
                    int32_t k, int64_t num_docs, int32_t shard_major, float *out_scores, int32_t *out_ids,
                    void *stream);

/*
 * Learned starting bounds.  A prune session keeps, per term, its 32 largest
 * posting scores and its mean posting score (computed on the device at
 * creation).  From them each query gets 32 features and a safe bound (the
 * largest K-th posting score among its words, which K documents always reach);
 * the threshold model (an MLP 32 -> 64 -> 64 -> 1 predicting the log of the
 * K-th score; see bm25_mlp_*) turns the features into tau = max(exp(prediction
 * - margin), safe bound).  Without a model (params = NULL) tau is the safe bound.
 */
int bm25_set_threshold_model(bm25_handle *handle, const float *params, float margin);

/* features float [q][32] and safe float [q] (may be NULL) on device buffers; asynchronous on stream. */
int bm25_query_features_device(bm25_handle *handle, const int64_t *qoffsets, const int32_t *words, int64_t q,
                               int32_t k, float *features, float *safe, void *stream);

/* bm25_search_pruned with the learned bounds (host buffers). */
int bm25_search_learned(bm25_handle *handle, const int64_t *qoffsets, const int32_t *words, int64_t q, int32_t k,
                        float *out_scores, int32_t *out_ids, int32_t *out_exact);

/* bm25_search_pruned_device with the learned bounds. */
int bm25_search_learned_device(bm25_handle *handle, const int64_t *qoffsets, const int32_t *words, int64_t q,
                               int32_t k, float *out_scores, int32_t *out_ids, int32_t *out_exact, void *stream);

/*
 * Search counters summed over Searches since the last reset (waits for the
 * handle's work), out[7]: tile-group kernel -- [0] claims (query x 8-tile
 * groups), [1] tiles scanned, [2] postings copied from HBM into the staging
 * rings; block-max pruned pass -- [3] tiles scored, [4] 128-document blocks
 * kept, [5] postings read, [6] queries streamed instead (prune_route).
 */
int bm25_search_stats(bm25_handle *handle, uint64_t *out, int32_t reset);

/* Waits for the handle's device-resident Searches and returns their accumulated device status word
 * (0 = clean), then clears it.  Device-resident Searches only OR into this word. */
int bm25_device_status(bm25_handle *handle, uint32_t *status);

/* Releases device and pinned resources; idempotent; a failed close can be retried (planned_search.cpp:22-56). */
int bm25_close(bm25_handle *handle);

/* Closes (if needed) and frees the handle itself. */
void bm25_destroy(bm25_handle *handle);

/*
 * Test hook, no counterpart in the reference: arms a one-shot failure of the next
 * bm25_search on `handle` so the error contract can be tested without faulting a GPU
 * (the reference tests it with a mocked session whose Search throws,
 * ut/cases/bm25/sdk_facade_tests.cpp:47-56).
 *   BM25_INJECT_HOST_FAILURE: the Search runs, then is reported as a device failure
 *     (BM25_ERR_INNER_ERROR, the session poisoned); handle NULL arms it for the next
 *     bm25_search of any handle in the process.
 *   BM25_INJECT_STALL: the tile-group kernel's producer issues no ring stage, so its
 *     consumers' bounded waits run out (options.wait_budget_cycles) and the kernel
 *     reports a timeout in the device status: BM25_ERR_INNER_ERROR, session poisoned.
 *     Needs a handle; other kernels have no wait to stall and ignore it.
 */
#define BM25_INJECT_HOST_FAILURE 1
#define BM25_INJECT_STALL 2
int bm25_test_inject(bm25_handle *handle, int32_t what);

/* Last error message of the handle (ErrorInfo, common/bm25/error_info.h:8-20); code = CUDA error or 0. */
int bm25_last_error(const bm25_handle *handle, char *buffer, size_t length, int64_t *code);

/*
 * Search without any device allocation, for callers that cannot call
 * cudaMalloc (a framework that owns all device memory through its own pool, a
 * serving loop that forbids allocation after start-up): the caller holds the
 * eager CSC index (same rules as bm25_create) and the query packet in device
 * memory and passes device pointers for the outputs.  No counterpart in the
 * reference.
 *   - indices and data must be 16-byte aligned and readable up to the next
 *     multiple of 4 elements past indptr[vocab];
 *   - num_words = qoffsets[q] (at most 64 words per query); 1 <= k <= min(32, num_docs);
 *   - all scratch comes from one fixed 16 MiB device array inside this library
 *     (held by every GPU that loads it until exit); a Search needing more is
 *     rejected with BM25_ERR_INVALID_PARAM before any device work.  The need,
 *     in bytes, with a16(x) = x rounded up to a multiple of 16:
 *       tile  = the smallest of 2048, 4096, 8192 with tile * SMs >= num_docs
 *               (8192 when none is), tiles = ceil(num_docs / tile),
 *       need  = 256 + 2 a16(4 q) + 128 q + 64 q tiles k + 16 max(1, num_words) tiles;
 *   - work runs on `stream` (a cudaStream_t) on device `device_id`; the call
 *     waits for it and returns the device status; the caller's current device
 *     is the same after the call as before it;
 *   - the first call on a device looks up the array's device address, sets
 *     kernel attributes and page-locks a static host word for the status
 *     (nothing is allocated): make it before any stream capture;
 *   - every call shares the array, so calls that overlap on the GPU (other
 *     streams, other host threads) race: serialise them;
 *   - error details: bm25_last_error(NULL, ...) on the calling thread.
 */
int bm25_search_csc_static(const int64_t *indptr, const int32_t *indices, const float *data, int64_t vocab,
                           int64_t num_docs, const int64_t *qoffsets, const int32_t *words, int64_t q,
                           int64_t num_words, int32_t k, float *out_scores, int32_t *out_ids, void *stream,
                           int32_t device_id);

/*
 * Measurement hook, no counterpart in the reference: with timing enabled,
 * every bm25_search_device records a CUDA event pair on its stream around the
 * main search kernel (the streaming kernel, or the per-tile kernel).
 * bm25_kernel_times waits for them and returns the durations in ms of the
 * Searches issued since the last read (at most the 4096 most recent), then
 * starts a new count.  Graph-replayed bm25_search calls are not timed.
 */
int bm25_kernel_timing(bm25_handle *h, int32_t enable);
int bm25_kernel_times(bm25_handle *h, float *ms, int64_t capacity, int64_t *count);

/*
 * Threshold MLP of the learned-pruning path (no counterpart in the reference).
 * A 32 -> 64 -> 64 -> 1 ReLU network in FP32 whose parameters are one flat array
 * of bm25_mlp_param_count() floats: W1[64][32] | b1[64] | W2[64][64] | b2[64] |
 * w3[64] | b3.  It predicts a query's log K-th score from 32 features; all
 * pointers are device pointers, work is enqueued on `stream` (a cudaStream_t).
 *   bm25_mlp_forward:  out[i] = f(features[i][0..31]) for i < batch.
 *   bm25_mlp_gradient: grad = d/dparams of mean_i w_i * (f(x_i) - t_i)^2, w_i =
 *     over_weight when f(x_i) > t_i else 1 (an over-estimate costs a plain re-run),
 *     and *loss = that mean; deterministic (fixed summation order).  `scratch`
 *     holds bm25_mlp_scratch_floats(batch) floats.  `loss` may be NULL.
 *   bm25_mlp_adam: one Adam step (beta1 0.9, beta2 0.999, eps 1e-8), step >= 1.
 * Error details: bm25_mlp_last_error.
 */
int64_t bm25_mlp_param_count(void);
int64_t bm25_mlp_scratch_floats(int64_t batch);
int bm25_mlp_forward(const float *params, const float *features, int64_t batch, float *out, void *stream);
int bm25_mlp_gradient(const float *params, const float *features, const float *targets, int64_t batch,
                      float over_weight, float *scratch, float *grad, float *loss, void *stream);
int bm25_mlp_adam(float *params, float *m, float *v, const float *grad, float lr, int32_t step, void *stream);
int bm25_mlp_last_error(char *buffer, size_t length);

/*
 * Continuous-batching server over one session (no counterpart in the reference):
 * queries are submitted one at a time from any thread; a worker thread runs the
 * waiting queries as one Search with a K per query (bm25_search_batch, or the
 * learned variant) whenever the previous batch returns.  Admission: arrival
 * order, at most max_batch queries (<= the session's query_capacity), the
 * session's word capacity, and a candidate budget (sum of the batch's K; 0 = no
 * limit).  max_wait_us > 0 lets a partial batch wait that long for more
 * arrivals.  Needs a tile-group session (prune = 1 for learned).
 */
typedef struct bm25_server bm25_server;
typedef struct bm25_server_options {
    int32_t max_batch;
    int32_t learned;
    int32_t max_wait_us;
    int32_t reserved;
    int64_t candidate_budget;
} bm25_server_options;
void bm25_default_server_options(bm25_server_options *options);
int bm25_server_create(bm25_handle *handle, const bm25_server_options *options, bm25_server **out);
/* words int32 [n] (n <= 64), K in [1, max_k]; *ticket identifies the query for bm25_server_wait. */
int bm25_server_submit(bm25_server *server, const int32_t *words, int32_t n, int32_t k, uint64_t *ticket);
/* Blocks until the query's batch returns: scores/ids [k] (may be NULL), exact (learned; may be NULL),
 * latency_us from submission to the batch's return. */
int bm25_server_wait(bm25_server *server, uint64_t ticket, float *scores, int32_t *ids, int32_t *exact,
                     double *latency_us);
int bm25_server_stats(bm25_server *server, int64_t *batches, int64_t *served);
/* Stops after the queued queries are served. */
int bm25_server_destroy(bm25_server *server);
int bm25_server_last_error(char *buffer, size_t length);
/*
 * Open-loop Poisson load on a server made with `options`: `total` arrivals at
 * rate_qps (exponential gaps, seeded), query i taken from the pool (qoffsets
 * [pool + 1], words, ks [pool]) at i % pool; latency_us [total] from each
 * scheduled arrival to its batch's return; elapsed_s from the start to the last
 * return; *batches Searches run.
 */
int bm25_serve_poisson(bm25_handle *handle, const bm25_server_options *options, const int64_t *qoffsets,
                       const int32_t *words, const int32_t *ks, int64_t pool, double rate_qps, int64_t total,
                       uint64_t seed, double *latency_us, double *elapsed_s, int64_t *batches);

/*
 * Index builder on the GPU (replaces the reference's Python builder,
 * standalone/large_corpus.py:95-297): documents as token ids (doc_offsets int64
 * [num_docs + 1], tokens int32, each in [0, vocab)) -> the lazy index of
 * standalone/resident_index.py:12-18 in host buffers: term_offsets [vocab + 1],
 * posting_doc_ids and posting_tf (room for doc_offsets[num_docs] postings; term
 * frequencies as FP32), doc_norm [num_docs] = f32(k1 (1 - b + b len / avgdl))
 * and idf [vocab] = f32(log1p((N - df + 0.5) / (df + 0.5))), both evaluated in
 * double as the reference's Python does (it uses k1 = 1.2, b = 0.75);
 * *postings receives the posting count.  The postings of a term are in
 * ascending document order.  Feed the result to bm25_create_lazy.  Error
 * details: bm25_build_last_error.
 */
int bm25_build_index(const int64_t *doc_offsets, const int32_t *tokens, int64_t num_docs, int64_t vocab, double k1,
                     double b, int32_t device_id, int64_t *term_offsets, int32_t *posting_doc_ids, float *posting_tf,
                     float *doc_norm, float *idf, int64_t *postings);
int bm25_build_last_error(char *buffer, size_t length);

/*
 * Runtime tuning of a session (no counterpart in the reference): knobs that change speed,
 * never results, settable on a live session without re-uploading the index (the
 * autotuner, bm25-npu_b200/autotune.py, times them on a sample batch and keeps the
 * fastest).  Setting them drops the session's instantiated graphs.
 *   claim_tiles      warp-tile kernel: tiles per claim, 2, 4 or 8
 *   tail_claims      warp-tile kernel: single-tile claims per warp at the end, 0..8
 *   ring_stages      tile-group kernel: ring depth, 2..8
 *   ring_chunk       tile-group kernel: postings per ring stage, a multiple of 4 in 512..4096
 *                    (stages and chunk must fit one SM's shared memory)
 *   candidate_cap    max_k > 32: candidates kept per query in a Search of one K > 32, from
 *                    max(2048, 8 max_k) up to the session's candidate_capacity (0 = all of
 *                    it); rounded up to a multiple of 4; a query that overflows it is
 *                    searched again (ties beyond it are reported as with candidate_capacity)
 *   prune_route      as bm25_options.prune_route
 */
typedef struct bm25_tuning {
    int32_t claim_tiles;
    int32_t tail_claims;
    int32_t ring_stages;
    int32_t ring_chunk;
    int64_t candidate_cap;
    float prune_route;
    int32_t reserved;
} bm25_tuning;
int bm25_get_tuning(bm25_handle *handle, bm25_tuning *tuning);
int bm25_set_tuning(bm25_handle *handle, const bm25_tuning *tuning);

/* Engine facts for reports and tests. */
typedef struct bm25_info {
    int64_t num_docs, vocab, postings;
    int32_t tile_docs, tiles, merge_fan_in, merge_levels;
    int64_t directory_rows, directory_min_df;
    int64_t index_bytes, device_bytes;
    int64_t graph_replays, searches;
    int32_t kernel, ring_stages, grid, smem_bytes, ring_chunk;
    int32_t query_capacity, word_capacity, max_k, prune;
    int64_t graph_instantiations; /* CUDA graphs instantiated since create */
    int64_t graphs_cached;        /* instantiated graphs held now */
    int64_t dense_rows;           /* terms kept as dense rows (dense_density) */
} bm25_info;
int bm25_get_info(const bm25_handle *handle, bm25_info *info);

#ifdef __cplusplus
}
#endif
#endif /* BM25_B200_H */
