/*
 * CPU oracle for the BM25 Search hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker the parity tests, smoke() and bench.py's cpu_baseline
 * leg compare the CUDA engine against.  It is never linked into, loaded by or
 * called from the product library; the product fails loudly when its CUDA
 * extension is missing instead of falling back to anything here.
 *
 * It restates, in plain C, the reference's CPU search:
 *   - term-order FP32 scatter-add per document
 *       feature_retrieval/src/ascendfaiss/test/ascendhost/bm25/reference/cpu_index_search.h:170-190
 *     with the per-posting contribution either read from an eager CSC `data`
 *     array (the bm25s layout, reference_only/bm25s_original/bm25s/scoring.py:361-366)
 *     or computed lazily with the reference's FP32 expression
 *       cpu_index_search.h:185-186, ops/.../bm25_fused_score_top_k.cpp:738-739
 *   - strict top-K over every document (score desc, doc id asc; documents whose
 *     score is zero tie and fill by ascending id)
 *       feature_retrieval/src/ascendfaiss/common/bm25/topk_document_shards.h:13-47,
 *       common/bm25/topk_heap.h:11-28
 *   - input rules: words < 0 or == INT32_MAX rejected, words >= V skipped
 *       cpu_index_search.h:159-178
 *
 * Parity is pinned against (a) the reference's own CpuSearchSession compiled from
 * its sources (oracle/_ref, k1 = 1.2, K <= 32), (b) goldens produced by the
 * reference's Python corpus generator standalone/large_corpus.py, and (c) goldens
 * produced by the vendored bm25s query path; see tests/golden/.
 *
 * Build: gcc -O2 -std=c11 -fopenmp -ffp-contract=off -fno-fast-math -shared -fPIC
 * (FLT_EVAL_METHOD 0 on x86-64 SSE: every float operation rounds to binary32).
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_OK 0
#define ORACLE_INVALID (-1)
#define ORACLE_NOMEM (-2)

typedef struct {
    float score;
    int32_t id;
} cand_t;

/* score desc, id asc (topk_heap.h:11-16) */
static inline int better(cand_t a, cand_t b)
{
    return a.score > b.score || (a.score == b.score && a.id < b.id);
}

/* Bounded heap whose root is the worst kept candidate. */
static void heap_sift_down(cand_t *h, int64_t n, int64_t i)
{
    for (;;) {
        int64_t l = 2 * i + 1, r = l + 1, w = i;
        if (l < n && better(h[w], h[l]))
            w = l;
        if (r < n && better(h[w], h[r]))
            w = r;
        if (w == i)
            return;
        cand_t t = h[i];
        h[i] = h[w];
        h[w] = t;
        i = w;
    }
}

static void heap_sift_up(cand_t *h, int64_t i)
{
    while (i > 0) {
        int64_t p = (i - 1) / 2;
        if (!better(h[p], h[i]))
            return;
        cand_t t = h[i];
        h[i] = h[p];
        h[p] = t;
        i = p;
    }
}

static void keep(cand_t *h, int64_t *size, int64_t k, cand_t item)
{
    if (*size < k) {
        h[*size] = item;
        heap_sift_up(h, *size);
        ++*size;
    } else if (better(item, h[0])) {
        h[0] = item;
        heap_sift_down(h, *size, 0);
    }
}

static int cmp_better(const void *a, const void *b)
{
    const cand_t x = *(const cand_t *)a, y = *(const cand_t *)b;
    if (better(x, y))
        return -1;
    if (better(y, x))
        return 1;
    return 0;
}

static inline int is_zero_bits(float v)
{
    uint32_t u;
    memcpy(&u, &v, 4);
    return (u & 0x7fffffffu) == 0;
}

/* One posting's contribution with the reference's FP32 expression (k1p1 = f32(k1 + 1)). */
static inline float lazy_contribution(float idf, float tf, float norm, float k1p1)
{
    const float numerator = tf * k1p1;
    return (idf * numerator) / (tf + norm);
}

/*
 * Eager contributions for a lazy (tf, norm, idf) index, in posting order.
 * Follows cpu_index_search.h:185-186 with 2.2F generalised to f32(k1 + 1).
 */
int oracle_contributions(const int64_t *offsets, int64_t vocab, const int32_t *docs, const float *tf,
                         const float *norm, int64_t num_docs, const float *idf, float k1p1, float *data)
{
    if (!offsets || !docs || !tf || !norm || !idf || !data || vocab < 1 || num_docs < 1)
        return ORACLE_INVALID;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t t = 0; t < vocab; ++t)
        for (int64_t p = offsets[t]; p < offsets[t + 1]; ++p)
            data[p] = lazy_contribution(idf[t], tf[p], norm[docs[p]], k1p1);
    return ORACLE_OK;
}

/*
 * Full per-document scores of query rows [0, Q) into full[Q * N] (the
 * reference's DebugScores, cpu_index_search.h:218-222).  If data is NULL the
 * contribution is computed lazily from tf/norm/idf/k1p1.
 */
static void score_row(const int64_t *indptr, int64_t vocab, const int32_t *indices, const float *data,
                      const float *tf, const float *norm, const float *idf, float k1p1, const int32_t *words,
                      int64_t nwords, float *row, int64_t num_docs)
{
    memset(row, 0, (size_t)num_docs * sizeof(float));
    for (int64_t w = 0; w < nwords; ++w) {
        const int32_t term = words[w];
        if ((int64_t)term >= vocab)
            continue; /* unknown word: skipped, cpu_index_search.h:177-178 */
        for (int64_t p = indptr[term]; p < indptr[term + 1]; ++p) {
            const int32_t doc = indices[p];
            const float c = data ? data[p] : lazy_contribution(idf[term], tf[p], norm[doc], k1p1);
            row[doc] += c;
        }
    }
}

static int validate_queries(const int64_t *qoffsets, const int32_t *words, int64_t q)
{
    if (!qoffsets || q < 1 || qoffsets[0] != 0)
        return 0;
    for (int64_t i = 0; i < q; ++i)
        if (qoffsets[i + 1] < qoffsets[i])
            return 0;
    for (int64_t w = 0; w < qoffsets[q]; ++w)
        if (!words || words[w] < 0 || words[w] == INT32_MAX)
            return 0;
    return 1;
}

/* Strict top-K of one full score row (topk_document_shards.h semantics, unbounded K). */
static void select_row(const float *row, int64_t num_docs, int64_t k, cand_t *heap, float *out_scores,
                       int32_t *out_ids)
{
    int64_t size = 0;
    for (int64_t d = 0; d < num_docs; ++d)
        if (!is_zero_bits(row[d]))
            keep(heap, &size, k, (cand_t){row[d], (int32_t)d});
    qsort(heap, (size_t)size, sizeof(cand_t), cmp_better);
    int64_t r = 0;
    for (; r < size; ++r) {
        out_scores[r] = heap[r].score;
        out_ids[r] = heap[r].id;
    }
    /* Zero-score documents tie; the smallest ids fill the remaining ranks. */
    for (int64_t d = 0; r < k && d < num_docs; ++d)
        if (is_zero_bits(row[d])) {
            out_scores[r] = 0.0f;
            out_ids[r] = (int32_t)d;
            ++r;
        }
}

/*
 * Search: queries given as offsets[Q + 1] (int64) and words (int32), the packed
 * layout of common/bm25/search_inputs.h:23-42.  Outputs [Q * K].
 * Either data (eager) or tf/norm/idf/k1p1 (lazy) supplies contributions.
 * full (optional, [Q * N]) receives the per-document scores.
 */
int oracle_search(const int64_t *indptr, int64_t vocab, const int32_t *indices, const float *data,
                  const float *tf, const float *norm, const float *idf, float k1p1, int64_t num_docs,
                  const int64_t *qoffsets, const int32_t *words, int64_t q, int64_t k, float *out_scores,
                  int32_t *out_ids, float *full, int threads)
{
    if (!indptr || !indices || vocab < 1 || num_docs < 1 || k < 1 || k > num_docs || !out_scores || !out_ids)
        return ORACLE_INVALID;
    if (!data && (!tf || !norm || !idf))
        return ORACLE_INVALID;
    if (!validate_queries(qoffsets, words, q))
        return ORACLE_INVALID;
    if (threads < 1)
        threads = omp_get_max_threads();
    int failed = 0;
#pragma omp parallel num_threads(threads)
    {
        float *row = full ? NULL : (float *)malloc((size_t)num_docs * sizeof(float));
        cand_t *heap = (cand_t *)malloc((size_t)k * sizeof(cand_t));
        if ((!full && !row) || !heap) {
#pragma omp atomic write
            failed = 1;
        }
#pragma omp barrier
        if (!failed) {
#pragma omp for schedule(dynamic, 1)
            for (int64_t i = 0; i < q; ++i) {
                float *r = full ? full + i * num_docs : row;
                score_row(indptr, vocab, indices, data, tf, norm, idf, k1p1, words + qoffsets[i],
                          qoffsets[i + 1] - qoffsets[i], r, num_docs);
                select_row(r, num_docs, k, heap, out_scores + i * k, out_ids + i * k);
            }
        }
        free(row);
        free(heap);
    }
    return failed ? ORACLE_NOMEM : ORACLE_OK;
}

/*
 * Exact merge of per-shard top-K lists (the document-partition argument of
 * topk_document_shards.h:4): lists[S][K] with -1 ids as empty slots, already
 * holding global doc ids.  Writes the strict global top-K.  Zero-score entries
 * participate like any other (they carry their ids), so shards must report
 * their zero fill too.
 */
int oracle_merge(const float *scores, const int32_t *ids, int64_t shards, int64_t k, float *out_scores,
                 int32_t *out_ids)
{
    if (!scores || !ids || shards < 1 || k < 1)
        return ORACLE_INVALID;
    cand_t *heap = (cand_t *)malloc((size_t)k * sizeof(cand_t));
    if (!heap)
        return ORACLE_NOMEM;
    int64_t size = 0;
    for (int64_t i = 0; i < shards * k; ++i)
        if (ids[i] >= 0)
            keep(heap, &size, k, (cand_t){scores[i], ids[i]});
    qsort(heap, (size_t)size, sizeof(cand_t), cmp_better);
    for (int64_t r = 0; r < k; ++r) {
        out_scores[r] = r < size ? heap[r].score : -1.0f;
        out_ids[r] = r < size ? heap[r].id : -1;
    }
    free(heap);
    return ORACLE_OK;
}

int oracle_max_threads(void) { return omp_get_max_threads(); }
