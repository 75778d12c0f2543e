// Plan kernel for Searches over a caller-held CSC index without a per-tile
// directory (the directory is built by a session; a caller that owns only the
// CSC arrays has none).  Same output as PlanKernel: plan[w][tile] = absolute
// posting range of query word w inside tile, by lower_bound over the word's
// sorted doc ids (in shared memory when the list is short).
#pragma once
#include "stream_kernel.cuh"

namespace bm25k {

__global__ void __launch_bounds__(kPlanThreads) PlanNoDirectoryKernel(const StreamArgs a)
{
    __shared__ int ids[kPlanSmemIds];
    long long total = a.qoffsets[a.q];
    if (total < 0 || total > a.word_cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0)
            atomicOr(a.status, kStatusBadQuery);
        total = total < 0 ? 0 : a.word_cap;
    }
    for (long long w = blockIdx.x; w < total; w += gridDim.x) {
        const int term = a.words[w];
        PlanEntry *out = a.plan + w * a.tiles;
        if (term < 0 || term >= a.vocab) {
            if (term < 0 && threadIdx.x == 0)
                atomicOr(a.status, kStatusBadWord);
            for (int t = threadIdx.x; t < a.tiles; t += kPlanThreads)
                out[t] = PlanEntry{0, 0};
            continue;
        }
        const long long s = a.indptr[term], e = a.indptr[term + 1];
        if (e - s <= kPlanSmemIds) {
            const int n = (int)(e - s);
            __syncthreads();  // the previous word's readers are done with ids[]
            for (int p = threadIdx.x; p < n; p += kPlanThreads)
                ids[p] = __ldg(a.indices + s + p);
            __syncthreads();
            for (int t = threadIdx.x; t < a.tiles; t += kPlanThreads) {
                const long long lo = (long long)t * a.tile_docs;
                out[t] = PlanEntry{s + LowerBoundSmem(ids, n, lo), s + LowerBoundSmem(ids, n, lo + a.tile_docs)};
            }
        } else {
            for (int t = threadIdx.x; t < a.tiles; t += kPlanThreads) {
                const long long lo = (long long)t * a.tile_docs;
                out[t] = PlanEntry{LowerBoundGlobal(a.indices, s, e, lo),
                                   LowerBoundGlobal(a.indices, s, e, lo + a.tile_docs)};
            }
        }
    }
}

} // namespace bm25k
