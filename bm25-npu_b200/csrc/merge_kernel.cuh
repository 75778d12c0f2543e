// Exact merge of per-shard top-K lists (the role of the reference's
// bm25_top_k_merge, ops/ascendc/bm25/merge/op_kernel/bm25_top_k_merge.cpp:10-86):
// input [Q][S][K] (score, id) lists, each sorted by (score desc, id asc) over a
// disjoint document range; output [Q][K].  A list that is not a valid strict
// ranking (negative or non-finite score, id outside [0, num_docs), order broken)
// makes the query's whole output row -1, as in the reference.
//
// Rank merge instead of the reference's K rounds of warp arg-max: every entry's
// output rank is its position in its own list plus, in every other list, the
// number of entries ranked before it (a binary search of a sorted list); ids are
// distinct across disjoint shards, so the ranks are a permutation and an entry
// with rank < K is written straight to its slot.  One CTA per query; S lists of
// K entries each, S * K * log2(K) compares in all, no serial rounds.
#pragma once
#include "tile_kernels.cuh"

namespace bm25k {

constexpr int kMergeThreads = 256;

struct MergeArgs {
    const float *scores;  // [Q][S][K], or [S][Q][K] when shard_major (an all-gather's layout)
    const int *ids;       // same layout (local ids when bases is set)
    const int *bases;     // [S] first document of each shard, or nullptr: ids are global
    int q, shards, k;
    long long num_docs;   // global document count
    float *out_scores;    // [Q][K]
    int *out_ids;
    int shard_major;
};

// Position of entry r of shard s's list for query q.
__device__ __forceinline__ long long MergeAt(const MergeArgs &a, int q, int s, int r)
{
    return a.shard_major ? ((long long)s * a.q + q) * a.k + r : ((long long)q * a.shards + s) * a.k + r;
}

__device__ __forceinline__ int MergeId(const MergeArgs &a, int s, int id) { return a.bases ? id + a.bases[s] : id; }

__global__ void __launch_bounds__(kMergeThreads) MergeShardsKernel(const MergeArgs a)
{
    __shared__ int bad;
    const int q = blockIdx.x, tid = threadIdx.x;
    const int S = a.shards, K = a.k;
    if (tid == 0)
        bad = 0;
    __syncthreads();
    for (int e = tid; e < S * K; e += kMergeThreads) {
        const int s = e / K, r = e % K;
        const long long at = MergeAt(a, q, s, r);
        const float sc = a.scores[at];
        const long long id = (long long)MergeId(a, s, a.ids[at]);
        bool ok = sc >= 0.0f && sc <= FLT_MAX && a.ids[at] >= 0 && id >= 0 && id < a.num_docs;
        if (ok && r > 0) {
            const float ps = a.scores[at - 1];
            const int pi = MergeId(a, s, a.ids[at - 1]);
            ok = ps > sc || (ps == sc && (long long)pi < id);
        }
        if (!ok)
            bad = 1;
    }
    __syncthreads();
    float *os = a.out_scores + (long long)q * K;
    int *oi = a.out_ids + (long long)q * K;
    if (bad) {
        for (int r = tid; r < K; r += kMergeThreads) {
            os[r] = -1.0f;
            oi[r] = -1;
        }
        return;
    }
    for (int e = tid; e < S * K; e += kMergeThreads) {
        const int s = e / K, r = e % K;
        const long long at = MergeAt(a, q, s, r);
        const float sc = a.scores[at];
        const int id = MergeId(a, s, a.ids[at]);
        int rank = r;
        for (int o = 0; o < S && rank < K; ++o) {
            if (o == s)
                continue;
            // entries of list o ranked before (sc, id): the first position that is not Better
            int lo = 0, hi = K;
            const long long lb = MergeAt(a, q, o, 0);
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (Better(a.scores[lb + mid], MergeId(a, o, a.ids[lb + mid]), sc, id))
                    lo = mid + 1;
                else
                    hi = mid;
            }
            rank += lo;
        }
        if (rank < K) {
            os[rank] = sc;
            oi[rank] = id;
        }
    }
}

} // namespace bm25k
