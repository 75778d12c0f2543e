/*
 * Seeded synthetic corpus -> resident-index arrays, on the host (C + OpenMP).
 *
 * This is the engine's counterpart of the reference's corpus/index generator
 * standalone/large_corpus.py:95-297: two passes over a replayable document
 * stream (pass 1 counts document frequencies, pass 2 writes postings), producing
 * the reference's lazy index layout
 *     term_offsets int64 [V+1], posting_doc_ids int32 [M] (ascending per term),
 *     posting_tf float [M], doc_norm float [N], idf float [V]
 * (standalone/resident_index.py:12-18) with the reference's formulas
 *     idf  = f32(log1p((N - df + 0.5) / (df + 0.5)))      large_corpus.py:148
 *     norm = f32(k1 * (1 - b + b * len / avgdl))           large_corpus.py:174
 * evaluated in double and rounded once, as the reference does.
 *
 * The document stream: token ranks follow Zipf(s) over V terms (term id =
 * rank - 1; s = 0 draws every term alike, the reference's uniform stream of
 * large_corpus.py:58-62) and lengths follow round(lognormal(ln(mean) -
 * sigma^2/2, sigma)), at least 1 -- or, for sigma < 0, a uniform integer in
 * [mean - |sigma|, mean + |sigma|] (mean 32, sigma -16: the reference's 16..48).  Every random draw
 * is a counter-based hash of (seed, document, position), so the corpus does not
 * depend on the thread count and pass 2 replays pass 1 exactly.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SYNTH_MAX_LEN 65536

static inline uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

static inline uint64_t draw(uint64_t seed, uint64_t a, uint64_t b)
{
    return splitmix64(splitmix64(seed ^ (a * 0xD1342543DE82EF95ull)) ^ (b * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull));
}

static inline double unit53(uint64_t x) { return (double)(x >> 11) * (1.0 / 9007199254740992.0); }

typedef struct {
    int64_t docs, vocab, postings, tokens;
    double zipf_s, len_mean, len_sigma;
    uint64_t seed;
    int chunks;
    double *prob;     /* alias table */
    int32_t *alias;
    int32_t *doc_len; /* [N] */
    int32_t *chunk_df; /* [chunks][V]: df per chunk, later relative cursors */
    int64_t *df;       /* [V] */
} synth_t;

static int32_t doc_length(const synth_t *s, int64_t d)
{
    if (s->len_sigma < 0) {  /* uniform integer lengths in [mean - |sigma|, mean + |sigma|] */
        const int64_t lo = (int64_t)floor(s->len_mean + s->len_sigma + 0.5);
        const int64_t hi = (int64_t)floor(s->len_mean - s->len_sigma + 0.5);
        const uint64_t x = draw(s->seed, (uint64_t)d, 0xFFFFFFFF00000001ull);
        const int64_t len = lo + (int64_t)(x % (uint64_t)(hi - lo + 1));
        return (int32_t)(len < 1 ? 1 : (len > SYNTH_MAX_LEN ? SYNTH_MAX_LEN : len));
    }
    const double mu = log(s->len_mean) - 0.5 * s->len_sigma * s->len_sigma;
    const double u1 = unit53(draw(s->seed, (uint64_t)d, 0xFFFFFFFF00000001ull));
    const double u2 = unit53(draw(s->seed, (uint64_t)d, 0xFFFFFFFF00000002ull));
    const double z = sqrt(-2.0 * log(1.0 - u1)) * cos(6.283185307179586 * u2);
    double len = floor(exp(mu + s->len_sigma * z) + 0.5);
    if (len < 1)
        len = 1;
    if (len > SYNTH_MAX_LEN)
        len = SYNTH_MAX_LEN;
    return (int32_t)len;
}

static inline int32_t token(const synth_t *s, int64_t d, int32_t pos)
{
    const uint64_t x = draw(s->seed, (uint64_t)d, (uint64_t)pos);
    const uint64_t column = ((x >> 32) * (uint64_t)s->vocab) >> 32;
    const double frac = (double)(uint32_t)x * (1.0 / 4294967296.0);
    return frac < s->prob[column] ? (int32_t)column : s->alias[column];
}

static void sort_small(int32_t *a, int32_t n)
{
    if (n <= 48) {
        for (int32_t i = 1; i < n; ++i) {
            int32_t v = a[i], j = i - 1;
            while (j >= 0 && a[j] > v) {
                a[j + 1] = a[j];
                --j;
            }
            a[j + 1] = v;
        }
        return;
    }
    /* heapsort for the long tail of document lengths */
    for (int32_t start = n / 2 - 1; start >= 0; --start) {
        int32_t i = start;
        for (;;) {
            int32_t l = 2 * i + 1, m = i;
            if (l < n && a[l] > a[m])
                m = l;
            if (l + 1 < n && a[l + 1] > a[m])
                m = l + 1;
            if (m == i)
                break;
            int32_t t = a[i];
            a[i] = a[m];
            a[m] = t;
            i = m;
        }
    }
    for (int32_t end = n - 1; end > 0; --end) {
        int32_t t = a[0];
        a[0] = a[end];
        a[end] = t;
        int32_t i = 0;
        for (;;) {
            int32_t l = 2 * i + 1, m = i;
            if (l < end && a[l] > a[m])
                m = l;
            if (l + 1 < end && a[l + 1] > a[m])
                m = l + 1;
            if (m == i)
                break;
            int32_t u = a[i];
            a[i] = a[m];
            a[m] = u;
            i = m;
        }
    }
}

/* Walker alias table for p_r proportional to r^-s, r = 1..V. */
static int build_alias(synth_t *s)
{
    const int64_t v = s->vocab;
    double *p = (double *)malloc((size_t)v * sizeof(double));
    int32_t *small = (int32_t *)malloc((size_t)v * sizeof(int32_t));
    int32_t *large = (int32_t *)malloc((size_t)v * sizeof(int32_t));
    s->prob = (double *)malloc((size_t)v * sizeof(double));
    s->alias = (int32_t *)malloc((size_t)v * sizeof(int32_t));
    if (!p || !small || !large || !s->prob || !s->alias) {
        free(p);
        free(small);
        free(large);
        return -1;
    }
    double total = 0;
    for (int64_t r = 0; r < v; ++r) {
        p[r] = pow((double)(r + 1), -s->zipf_s);
        total += p[r];
    }
    int64_t ns = 0, nl = 0;
    for (int64_t r = 0; r < v; ++r) {
        p[r] = p[r] * (double)v / total;
        if (p[r] < 1.0)
            small[ns++] = (int32_t)r;
        else
            large[nl++] = (int32_t)r;
    }
    while (ns && nl) {
        const int32_t a = small[--ns], g = large[nl - 1];
        s->prob[a] = p[a];
        s->alias[a] = g;
        p[g] = (p[g] + p[a]) - 1.0;
        if (p[g] < 1.0) {
            --nl;
            small[ns++] = g;
        }
    }
    while (nl) {
        const int32_t g = large[--nl];
        s->prob[g] = 1.0;
        s->alias[g] = g;
    }
    while (ns) {
        const int32_t a = small[--ns];
        s->prob[a] = 1.0;
        s->alias[a] = a;
    }
    free(p);
    free(small);
    free(large);
    return 0;
}

void synth_destroy(void *handle)
{
    synth_t *s = (synth_t *)handle;
    if (!s)
        return;
    free(s->prob);
    free(s->alias);
    free(s->doc_len);
    free(s->chunk_df);
    free(s->df);
    free(s);
}

/*
 * Pass 1: document lengths and per-term document frequencies.
 * Returns NULL on invalid sizes or allocation failure.
 */
void *synth_create(int64_t docs, int64_t vocab, double zipf_s, double len_mean, double len_sigma, uint64_t seed,
                   int threads)
{
    if (docs < 1 || docs > INT32_MAX || vocab < 1 || vocab >= INT32_MAX || len_mean <= 0 ||
        (len_sigma < 0 && len_mean + len_sigma < 1))
        return NULL;
    synth_t *s = (synth_t *)calloc(1, sizeof(synth_t));
    if (!s)
        return NULL;
    s->docs = docs;
    s->vocab = vocab;
    s->zipf_s = zipf_s;
    s->len_mean = len_mean;
    s->len_sigma = len_sigma;
    s->seed = seed;
    if (threads < 1)
        threads = omp_get_max_threads();
    s->chunks = threads < 32 ? threads : 32;
    if ((int64_t)s->chunks > docs)
        s->chunks = (int)docs;
    s->doc_len = (int32_t *)malloc((size_t)docs * sizeof(int32_t));
    s->chunk_df = (int32_t *)calloc((size_t)s->chunks * (size_t)vocab, sizeof(int32_t));
    s->df = (int64_t *)calloc((size_t)vocab, sizeof(int64_t));
    if (!s->doc_len || !s->chunk_df || !s->df || build_alias(s)) {
        synth_destroy(s);
        return NULL;
    }
    int64_t tokens = 0;
    int failed = 0;
#pragma omp parallel for num_threads(s->chunks) schedule(static, 1) reduction(+ : tokens)
    for (int c = 0; c < s->chunks; ++c) {
        int32_t *buf = (int32_t *)malloc(SYNTH_MAX_LEN * sizeof(int32_t));
        if (!buf) {
#pragma omp atomic write
            failed = 1;
            continue;
        }
        int32_t *mydf = s->chunk_df + (size_t)c * (size_t)vocab;
        const int64_t begin = docs * c / s->chunks, end = docs * (c + 1) / s->chunks;
        for (int64_t d = begin; d < end; ++d) {
            const int32_t len = doc_length(s, d);
            s->doc_len[d] = len;
            tokens += len;
            for (int32_t i = 0; i < len; ++i)
                buf[i] = token(s, d, i);
            sort_small(buf, len);
            for (int32_t i = 0; i < len; ++i)
                if (i == 0 || buf[i] != buf[i - 1])
                    mydf[buf[i]]++;
        }
        free(buf);
    }
    if (failed) {
        synth_destroy(s);
        return NULL;
    }
    s->tokens = tokens;
    int64_t m = 0;
#pragma omp parallel for reduction(+ : m)
    for (int64_t t = 0; t < vocab; ++t) {
        int64_t acc = 0;
        for (int c = 0; c < s->chunks; ++c) {
            int32_t *cell = s->chunk_df + (size_t)c * (size_t)vocab + t;
            const int32_t here = *cell;
            *cell = (int32_t)acc; /* becomes the chunk's relative write cursor */
            acc += here;
        }
        s->df[t] = acc;
        m += acc;
    }
    s->postings = m;
    return s;
}

int64_t synth_postings(void *handle) { return ((synth_t *)handle)->postings; }
int64_t synth_tokens(void *handle) { return ((synth_t *)handle)->tokens; }

/*
 * Pass 2: fill the lazy index.  Caller buffers: offsets[V+1], docs[M], tf[M],
 * norm[N], idf[V], doc_len[N] (doc_len may be NULL).  Single use per handle.
 */
int synth_fill(void *handle, double k1, double b, int64_t *offsets, int32_t *docs, float *tf, float *norm,
               float *idf, int32_t *doc_len)
{
    synth_t *s = (synth_t *)handle;
    if (!s || !offsets || !docs || !tf || !norm || !idf)
        return -1;
    const int64_t v = s->vocab, n = s->docs;
    offsets[0] = 0;
    for (int64_t t = 0; t < v; ++t)
        offsets[t + 1] = offsets[t] + s->df[t];
    const double avg = (double)s->tokens / (double)n;
#pragma omp parallel for
    for (int64_t t = 0; t < v; ++t) {
        const double df = (double)s->df[t];
        idf[t] = (float)log1p(((double)n - df + 0.5) / (df + 0.5));
    }
#pragma omp parallel for
    for (int64_t d = 0; d < n; ++d) {
        norm[d] = (float)(k1 * (1.0 - b + b * (double)s->doc_len[d] / avg));
        if (doc_len)
            doc_len[d] = s->doc_len[d];
    }
    int failed = 0;
#pragma omp parallel for num_threads(s->chunks) schedule(static, 1)
    for (int c = 0; c < s->chunks; ++c) {
        int32_t *buf = (int32_t *)malloc(SYNTH_MAX_LEN * sizeof(int32_t));
        if (!buf) {
#pragma omp atomic write
            failed = 1;
            continue;
        }
        int32_t *cursor = s->chunk_df + (size_t)c * (size_t)v;
        const int64_t begin = n * c / s->chunks, end = n * (c + 1) / s->chunks;
        for (int64_t d = begin; d < end; ++d) {
            const int32_t len = s->doc_len[d];
            for (int32_t i = 0; i < len; ++i)
                buf[i] = token(s, d, i);
            sort_small(buf, len);
            for (int32_t i = 0; i < len;) {
                int32_t j = i + 1;
                while (j < len && buf[j] == buf[i])
                    ++j;
                const int32_t term = buf[i];
                const int64_t pos = offsets[term] + cursor[term]++;
                docs[pos] = (int32_t)d;
                tf[pos] = (float)(j - i);
                i = j;
            }
        }
        free(buf);
    }
    return failed ? -2 : 0;
}

/*
 * Seeded query batch: Q queries whose term counts are uniform in [lo, hi];
 * terms drawn with probability df(t) / M (a posting drawn uniformly, its term
 * taken), distinct within a query when `distinct` is set.  Writes
 * qoffsets[Q+1] and words[<= Q*hi]; returns the word count or -1.
 */
int64_t synth_queries(const int64_t *offsets, int64_t vocab, int64_t q, int32_t lo, int32_t hi, int distinct,
                      uint64_t seed, int64_t *qoffsets, int32_t *words)
{
    if (!offsets || vocab < 1 || q < 1 || lo < 0 || hi < lo || hi > 4096 || offsets[vocab] < 1)
        return -1;
    const int64_t m = offsets[vocab];
    int64_t n = 0;
    qoffsets[0] = 0;
    for (int64_t i = 0; i < q; ++i) {
        const uint64_t span = (uint64_t)(hi - lo + 1);
        const int32_t count = lo + (int32_t)(draw(seed, (uint64_t)i, 0xFFFFFFFF00000003ull) % span);
        uint64_t attempt = 0;
        for (int32_t j = 0; j < count; ++j) {
            for (;;) {
                const uint64_t x = draw(seed ^ 0x5DEECE66Dull, (uint64_t)i, attempt++);
                const int64_t posting = (int64_t)(x % (uint64_t)m);
                int64_t lo_t = 0, hi_t = vocab; /* largest t with offsets[t] <= posting */
                while (hi_t - lo_t > 1) {
                    const int64_t mid = lo_t + (hi_t - lo_t) / 2;
                    if (offsets[mid] <= posting)
                        lo_t = mid;
                    else
                        hi_t = mid;
                }
                int dup = 0;
                if (distinct)
                    for (int64_t w = qoffsets[i]; w < n; ++w)
                        dup |= words[w] == (int32_t)lo_t;
                if (!dup || attempt > 1000000) {
                    words[n++] = (int32_t)lo_t;
                    break;
                }
            }
        }
        qoffsets[i + 1] = n;
    }
    return n;
}
