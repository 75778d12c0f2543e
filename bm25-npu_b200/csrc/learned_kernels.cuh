// Learned starting bounds of the pruned Search (no counterpart in the reference).
//
// TermStatsKernel -- at session creation (prune = 1), one warp per term keeps
//   the term's kTermTop largest posting scores (descending, 0 past its
//   document frequency) and its mean posting score.
// QueryFeatures -- 32 features of one query from those statistics (the
//   query's four strongest words by top score, sums and extremes over all its
//   words, K), plus the query's safe bound: the largest, over its words, of the
//   word's K-th largest posting score.  K documents each hold that word with at
//   least that score, and every FP32 sum of non-negative contributions is at
//   least each of its terms (rounded addition is monotone), so K documents
//   reach the safe bound: it never makes a query fall back.
// LearnedBoundKernel -- features -> threshold MLP (log of the K-th score) ->
//   tau = max(exp(prediction - margin), safe bound); without a model tau is the
//   safe bound.  A query whose safe bound is 0 (no word with K postings) gets
//   tau = 0 and is not pruned.
#pragma once
#include "mlp.cuh"
#include "tile_kernels.cuh"

namespace bm25k {

constexpr int kTermTop = 32;  // largest posting scores kept per term (K <= 32)
constexpr int kFeatures = bm25mlp::kIn;
static_assert(kFeatures == 32, "feature layout below fills 32 slots");

__global__ void TermStatsKernel(const long long *indptr, const float *data, long long vocab, float *top, float *mean)
{
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * blockDim.x / 32;
    for (long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32; t < vocab; t += warps) {
        const long long s = indptr[t], e = indptr[t + 1];
        float ls = -1.0f, sum = 0.0f;
        int li = kNoId;
        for (long long b = s; b < e; b += 32) {
            const long long i = b + lane;
            const bool has = i < e;
            const float v = has ? data[i] : 0.0f;
            sum += v;
            WarpOffer(v, (int)(i - s), has, ls, li, kTermTop, lane);
        }
#pragma unroll
        for (int o = 16; o; o >>= 1)
            sum += __shfl_xor_sync(kFull, sum, o);
        top[t * kTermTop + lane] = li == kNoId ? 0.0f : fmaxf(ls, 0.0f);
        if (lane == 0)
            mean[t] = e > s ? sum / (float)(e - s) : 0.0f;
    }
}

struct LearnedArgs {
    const long long *indptr;
    const float *top;   // [vocab][kTermTop]
    const float *mean;  // [vocab]
    int vocab;
    const long long *qoffsets;
    const int *words;
    int q, k;
    long long word_cap;
    const float *params;  // threshold MLP, or nullptr: safe bounds only
    float margin;
    float *features;  // [q][kFeatures] (QueryFeaturesKernel)
    float *safe;      // [q] (QueryFeaturesKernel; may be nullptr)
    float *tau;       // [q] (LearnedBoundKernel)
};

__device__ __forceinline__ float LogScore(float x) { return log1pf(fmaxf(x, 0.0f)); }

// Features of query q (layout: 4 strongest words x [log1p top, log1p K-th, log1p mean,
// log1p(df) / 16], then valid words / 8, log1p of the sums of tops, K-ths and means, log1p
// of the largest K-th, log(K) / 4, summed and least log1p(df), log1p of the largest and of the
// summed (K+1)/2-th scores, out-of-vocabulary words / 8, a constant 1, four zeros).
__device__ __forceinline__ float QueryFeatures(const LearnedArgs &a, int q, float *f)
{
    const long long qb = a.qoffsets[q], qe = a.qoffsets[q + 1];
    long long n = qe - qb;
    if (n < 0 || n > kMaxTerms || qb < 0 || qb + n > a.word_cap)
        n = 0;  // the Search reports the malformed query
    const int k = a.k, h = (k - 1) / 2;
    float sum_top = 0.0f, sum_kth = 0.0f, max_kth = 0.0f, sum_mean = 0.0f, sum_ldf = 0.0f, min_ldf = 0.0f;
    float max_half = 0.0f, sum_half = 0.0f;
    int valid = 0, oov = 0;
    int best[4] = {-1, -1, -1, -1};
    float best_top[4] = {-1.0f, -1.0f, -1.0f, -1.0f};
    for (long long i = 0; i < n; ++i) {
        const int w = a.words[qb + i];
        if (w < 0 || w >= a.vocab) {
            ++oov;
            continue;
        }
        const float *t = a.top + (long long)w * kTermTop;
        const float mx = t[0], kth = t[k - 1], half = t[h];
        const float ldf = log1pf((float)(a.indptr[w + 1] - a.indptr[w]));
        sum_top += mx;
        sum_kth += kth;
        max_kth = fmaxf(max_kth, kth);
        sum_mean += a.mean[w];
        sum_ldf += ldf;
        min_ldf = valid ? fminf(min_ldf, ldf) : ldf;
        max_half = fmaxf(max_half, half);
        sum_half += half;
        ++valid;
        int pos = 4;  // strongest words first; an earlier word stays ahead of an equal one
        while (pos > 0 && mx > best_top[pos - 1])
            --pos;
        if (pos < 4) {
            for (int j = 3; j > pos; --j) {
                best_top[j] = best_top[j - 1];
                best[j] = best[j - 1];
            }
            best_top[pos] = mx;
            best[pos] = w;
        }
    }
    for (int j = 0; j < 4; ++j) {
        const int w = best[j];
        if (w < 0) {
            f[4 * j] = f[4 * j + 1] = f[4 * j + 2] = f[4 * j + 3] = 0.0f;
            continue;
        }
        const float *t = a.top + (long long)w * kTermTop;
        f[4 * j] = LogScore(t[0]);
        f[4 * j + 1] = LogScore(t[k - 1]);
        f[4 * j + 2] = LogScore(a.mean[w]);
        f[4 * j + 3] = log1pf((float)(a.indptr[w + 1] - a.indptr[w])) / 16.0f;
    }
    f[16] = valid / 8.0f;
    f[17] = LogScore(sum_top);
    f[18] = LogScore(sum_kth);
    f[19] = LogScore(max_kth);
    f[20] = LogScore(sum_mean);
    f[21] = logf((float)k) / 4.0f;
    f[22] = sum_ldf / 64.0f;
    f[23] = min_ldf / 16.0f;
    f[24] = LogScore(max_half);
    f[25] = LogScore(sum_half);
    f[26] = oov / 8.0f;
    f[27] = 1.0f;
    f[28] = f[29] = f[30] = f[31] = 0.0f;
    return max_kth;
}

__global__ void QueryFeaturesKernel(const LearnedArgs a)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < a.q; q += gridDim.x * blockDim.x) {
        float f[kFeatures];
        const float safe = QueryFeatures(a, q, f);
        for (int i = 0; i < kFeatures; ++i)
            a.features[(long long)q * kFeatures + i] = f[i];
        if (a.safe)
            a.safe[q] = safe;
    }
}

constexpr int kLearnedThreads = 64;

__global__ void __launch_bounds__(kLearnedThreads) LearnedBoundKernel(const LearnedArgs a)
{
    __shared__ float p[bm25mlp::kParams];
    if (a.params) {
        for (int i = threadIdx.x; i < bm25mlp::kParams; i += kLearnedThreads)
            p[i] = a.params[i];
    }
    __syncthreads();
    const int q = blockIdx.x * kLearnedThreads + threadIdx.x;
    if (q >= a.q)
        return;
    float f[kFeatures];
    const float safe = QueryFeatures(a, q, f);
    float tau = safe;
    if (a.params && safe > 0.0f) {
        float h1[bm25mlp::kH], h2[bm25mlp::kH];
        const float y = bm25mlp::Forward(p, f, h1, h2);
        tau = fmaxf(expf(y - a.margin), safe);  // a NaN prediction leaves the safe bound
    }
    a.tau[q] = tau;
}

} // namespace bm25k
