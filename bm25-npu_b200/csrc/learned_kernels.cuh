// Learned starting bounds of the pruned Search (no counterpart in the reference).
//
// TermStatsKernel -- at session creation (prune = 1), one warp per term keeps
//   the term's kTermTop largest posting scores (descending, 0 past its
//   document frequency) and its mean posting score.
// QueryFeatures -- 32 features of one query from those statistics (the
//   query's four strongest words by top score, sums and extremes over all its
//   words, K), plus the query's safe bound: for K <= 32 the largest, over its
//   words, of the word's K-th largest posting score (K documents each hold that
//   word with at least that score, and every FP32 sum of non-negative
//   contributions is at least each of its terms -- rounded addition is
//   monotone -- so K documents reach it and it never makes a query fall back);
//   for K in 33..1024 the same with the word's score at the smallest rank 64,
//   128, ..., 1024 not below K (term ranks, warp-tile sessions; else 0); -1
//   when the query's words hold fewer than K postings in all
//   (fewer than K documents can match: such a query is not pruned).
// LearnedBoundKernel -- features -> threshold MLP (log of the K-th score) ->
//   tau = max(exp(prediction - margin), safe bound); without a model tau is the
//   safe bound; tau = 0 where the safe bound is -1.
#pragma once
#include "mlp.cuh"
#include <cfloat>
#include <climits>
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
    const float *rank;  // [vocab][5] scores at ranks 64 .. 1024 (safe bounds for K above 32), or nullptr
    const float *mean;  // [vocab]
    int vocab;
    const long long *qoffsets;
    const int *words;
    int q, k;
    const int *kq;  // [q] K per query, or nullptr: every query takes k
    long long word_cap;
    const float *params;  // threshold MLP, or nullptr: safe bounds only
    float margin;
    float *features;  // [q][kFeatures] (QueryFeaturesKernel)
    float *safe;      // [q] (QueryFeaturesKernel; may be nullptr)
    float *tau;       // [q] (LearnedBoundKernel)
};

__device__ __forceinline__ float LogScore(float x) { return log1pf(fmaxf(x, 0.0f)); }

// Features of query q, computed by one warp (lane l takes the query's words l and l + 32; sums
// and extremes are warp reductions in a fixed order, so the result is deterministic).  Layout:
// 4 strongest words by top score (an earlier word ahead of an equal one) x [log1p top, log1p
// K-th, log1p mean, log1p(df) / 16], then valid words / 8, log1p of the sums of tops, K-ths and
// means, log1p of the largest K-th, log(K) / 4, summed and least log1p(df), log1p of the largest
// and of the summed (K+1)/2-th scores, out-of-vocabulary words / 8, a constant 1, four zeros;
// the K-th and (K+1)/2-th scores are taken at min(K, 32).  Lane 0 writes f and returns the safe
// bound (every lane returns it).
__device__ __forceinline__ float QueryFeaturesWarp(const LearnedArgs &a, int q, float *f, int lane)
{
    const long long qb = a.qoffsets[q], qe = a.qoffsets[q + 1];
    long long nl = qe - qb;
    if (nl < 0 || nl > kMaxTerms || qb < 0 || qb + nl > a.word_cap)
        nl = 0;  // the Search reports the malformed query
    const int n = (int)nl;
    const int k = a.kq ? min(max(a.kq[q], 1), a.k) : a.k, kk = min(k, kTermTop), h = (kk - 1) / 2;
    long long postings = 0;
    float max_rank = 0.0f;  // K > 32: the largest, over the words, score at the smallest rank >= K
    float sum_top = 0.0f, sum_kth = 0.0f, max_kth = 0.0f, sum_mean = 0.0f, sum_ldf = 0.0f;
    float min_ldf = FLT_MAX, max_half = 0.0f, sum_half = 0.0f;
    int valid = 0, oov = 0;
    float top_of[2] = {-1.0f, -1.0f};  // this lane's words (position lane, lane + 32)
    int word_of[2] = {-1, -1};
    float feat_of[2][4] = {};  // their four per-word features
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const int i = lane + 32 * u;
        if (i >= n)
            continue;
        const int w = a.words[qb + i];
        if (w < 0 || w >= a.vocab) {
            ++oov;
            continue;
        }
        const float *t = a.top + (long long)w * kTermTop;
        const float mx = t[0], kth = t[kk - 1], half = t[h];
        if (a.rank && k > kTermTop && k <= 1024)
            max_rank = fmaxf(max_rank, a.rank[(long long)w * 5 + (31 - __clz(k - 1)) - 5]);
        const long long df = a.indptr[w + 1] - a.indptr[w];
        postings += df;
        const float ldf = log1pf((float)df);
        sum_top += mx;
        sum_kth += kth;
        max_kth = fmaxf(max_kth, kth);
        sum_mean += a.mean[w];
        sum_ldf += ldf;
        min_ldf = fminf(min_ldf, ldf);
        max_half = fmaxf(max_half, half);
        sum_half += half;
        ++valid;
        top_of[u] = mx;
        word_of[u] = w;
        feat_of[u][0] = LogScore(mx);
        feat_of[u][1] = LogScore(kth);
        feat_of[u][2] = LogScore(a.mean[w]);
        feat_of[u][3] = ldf / 16.0f;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        postings += __shfl_xor_sync(kFull, postings, o);
        sum_top += __shfl_xor_sync(kFull, sum_top, o);
        sum_kth += __shfl_xor_sync(kFull, sum_kth, o);
        max_kth = fmaxf(max_kth, __shfl_xor_sync(kFull, max_kth, o));
        max_rank = fmaxf(max_rank, __shfl_xor_sync(kFull, max_rank, o));
        sum_mean += __shfl_xor_sync(kFull, sum_mean, o);
        sum_ldf += __shfl_xor_sync(kFull, sum_ldf, o);
        min_ldf = fminf(min_ldf, __shfl_xor_sync(kFull, min_ldf, o));
        max_half = fmaxf(max_half, __shfl_xor_sync(kFull, max_half, o));
        sum_half += __shfl_xor_sync(kFull, sum_half, o);
        valid += __shfl_xor_sync(kFull, valid, o);
        oov += __shfl_xor_sync(kFull, oov, o);
    }
    // the four strongest words: four rounds of a warp arg-max on (top desc, position asc)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int u = top_of[1] > top_of[0] ? 1 : 0;  // position lane + 32u; ties keep the earlier
        float bt = top_of[u];
        int bp = word_of[u] >= 0 ? lane + 32 * u : INT_MAX;
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const float ot = __shfl_xor_sync(kFull, bt, o);
            const int op = __shfl_xor_sync(kFull, bp, o);
            if (ot > bt || (ot == bt && op < bp)) {
                bt = ot;
                bp = op;
            }
        }
        const bool found = bp != INT_MAX && bt >= 0.0f;
        float g[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        if (found && (bp & 31) == lane) {  // the owner hands over its winner's features and drops it
            const int slot = bp >> 5;
#pragma unroll
            for (int c = 0; c < 4; ++c)
                g[c] = slot ? feat_of[1][c] : feat_of[0][c];
            top_of[slot] = -1.0f;
            word_of[slot] = -1;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c)
            g[c] = __shfl_sync(kFull, g[c], found ? (bp & 31) : 0);
        if (lane == 0)
#pragma unroll
            for (int c = 0; c < 4; ++c)
                f[4 * j + c] = found ? g[c] : 0.0f;
    }
    if (lane == 0) {
        f[16] = valid / 8.0f;
        f[17] = LogScore(sum_top);
        f[18] = LogScore(sum_kth);
        f[19] = LogScore(max_kth);
        f[20] = LogScore(sum_mean);
        f[21] = logf((float)k) / 4.0f;
        f[22] = sum_ldf / 64.0f;
        f[23] = valid ? min_ldf / 16.0f : 0.0f;
        f[24] = LogScore(max_half);
        f[25] = LogScore(sum_half);
        f[26] = oov / 8.0f;
        f[27] = 1.0f;
        f[28] = f[29] = f[30] = f[31] = 0.0f;
    }
    __syncwarp();
    if (postings < k)
        return -1.0f;
    return k <= kTermTop ? max_kth : max_rank;
}

// One warp per query.
__global__ void QueryFeaturesKernel(const LearnedArgs a)
{
    __shared__ float fs[8][kFeatures];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = blockIdx.x * (blockDim.x >> 5) + warp; q < a.q; q += gridDim.x * (blockDim.x >> 5)) {
        float *f = fs[warp];
        const float safe = QueryFeaturesWarp(a, q, f, lane);
        a.features[(long long)q * kFeatures + lane] = f[lane];
        if (a.safe && lane == 0)
            a.safe[q] = safe;
        __syncwarp();
    }
}

constexpr int kLearnedQueries = 4;                            // queries per CTA
constexpr int kLearnedThreads = kLearnedQueries * bm25mlp::kH;  // a hidden unit per thread and query

// kLearnedQueries queries per CTA.  The parameters are staged in shared memory with both weight
// matrices transposed (unit i's weight j at [j][i]: consecutive threads read consecutive words);
// warp j builds query j's features; thread i of a query's group computes hidden unit i of each
// layer with the same fmaf chain, in the same order, as bm25mlp::Forward, so the prediction is
// bit-identical to the training kernels' forward pass; the group's first thread the output.
__global__ void __launch_bounds__(kLearnedThreads) LearnedBoundKernel(const LearnedArgs a)
{
    using namespace bm25mlp;
    // rows padded by one word: the transposing stores and the per-unit reads are both free of
    // bank conflicts
    __shared__ float w1t[kIn][kH + 1], w2t[kH][kH + 1], b1[kH], b2[kH], w3[kH];
    __shared__ float b3;
    __shared__ float f[kLearnedQueries][kFeatures], h1[kLearnedQueries][kH], h2[kLearnedQueries][kH];
    __shared__ float safe_s[kLearnedQueries];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = tid / kH, i = tid % kH;  // query slot in the CTA, hidden unit
    const int q0 = blockIdx.x * kLearnedQueries;
    AllowDependents();  // the plan kernel is built meanwhile (it reads none of this kernel's output)
    if (a.params) {
        const float *p = a.params;
        for (int x = tid; x < kH * kIn; x += kLearnedThreads)
            w1t[x % kIn][x / kIn] = __ldg(p + kOffW1 + x);
        for (int x = tid; x < kH * kH; x += kLearnedThreads)
            w2t[x % kH][x / kH] = __ldg(p + kOffW2 + x);
        for (int x = tid; x < kH; x += kLearnedThreads) {
            b1[x] = __ldg(p + kOffB1 + x);
            b2[x] = __ldg(p + kOffB2 + x);
            w3[x] = __ldg(p + kOffW3 + x);
        }
        if (tid == 0)
            b3 = __ldg(p + kOffB3);
    }
    if (warp < kLearnedQueries && q0 + warp < a.q) {
        const float safe = QueryFeaturesWarp(a, q0 + warp, f[warp], lane);
        if (lane == 0)
            safe_s[warp] = safe;
    }
    __syncthreads();
    const int q = q0 + g;
    const bool live = q < a.q;
    const float safe = live ? safe_s[g] : -1.0f;
    const bool run = a.params && safe >= 0.0f;  // uniform within a query's group
    if (run) {
        float acc = b1[i];
        for (int j = 0; j < kIn; ++j)
            acc = fmaf(w1t[j][i], f[g][j], acc);
        h1[g][i] = fmaxf(acc, 0.0f);
    }
    __syncthreads();
    if (run) {
        float acc = b2[i];
        for (int j = 0; j < kH; ++j)
            acc = fmaf(w2t[j][i], h1[g][j], acc);
        h2[g][i] = fmaxf(acc, 0.0f);
    }
    __syncthreads();
    if (live && i == 0) {
        float tau = fmaxf(safe, 0.0f);
        if (run) {
            float y = b3;
            for (int j = 0; j < kH; ++j)
                y = fmaf(w3[j], h2[g][j], y);
            tau = fmaxf(expf(y - a.margin), safe);  // a NaN prediction leaves the safe bound
        }
        a.tau[q] = tau;
        if (a.safe)
            a.safe[q] = safe;
    }
}

} // namespace bm25k
