// Block-max pruned scoring in the warp-tile style (warp-tile sessions' pruned passes).
//
// The work list is BlockBoundKernel's: one item per (query, 1024-document tile) with a
// kept block, its kept-block mask and its query's words.  A warp claims items from the
// pass's counter (the atomic for the next item is in flight while the current one runs)
// and scores each like a warp-tile tile:
//   * lane s resolves query word s's posting range in the tile: the plan entry [b, e) and,
//     for a word with a directory row, the block offsets, from which the range narrows to
//     [first posting of the first kept block, end of the last kept block) -- the postings
//     of dropped blocks between two kept ones are read as well (one contiguous run per
//     word, no per-block bookkeeping);
//   * the words go in groups of kWtLead: the first window (128 postings) of every word of a
//     group is loaded at once straight into registers, the rest two windows at a time, and
//     the group's words are added one by one (query-word order, a __syncwarp between words)
//     into the warp's private FP32 row, so an item waits for memory about once per group;
//   * the kept blocks are selected against the query's running bound (TileSelectAppend
//     with the mask) and the row is cleared.
// A document of a dropped block holds at most a partial sum, below its block's bound and so
// below tau, which the running bound never falls under: it is never selected, and its row
// entries are cleared with the block.  The result is the same as BlockScoreKernel's, which
// stages only the kept blocks' postings in shared memory with 4-byte asynchronous copies
// and pays one exposed memory latency per item on top of its metadata; here an item waits
// for its ranges, then for its postings about once per group of words, and a long run reads
// its first window with the rest of its group.
#pragma once
#include "block_kernels.cuh"
#include "warp_tile_kernel.cuh"

namespace bm25k {

// Posting range of query word w of an item in tile t with kept-block mask `mask` (nonzero):
// [lo, hi).  A word outside the vocabulary has an empty plan entry.
__device__ __forceinline__ void BtWordRange(const StreamArgs &a, long long w, int t, unsigned mask, int &lo, int &hi)
{
    int r;  // -1 short list, -2 not a term
    if (a.rows_plan) {  // written by PlanRowsKernel
        const int *row = a.plan_rows + w * a.dir_stride + t;
        lo = __ldcg(row);
        hi = __ldcg(row + 1);
        r = __ldcg(&a.word_rec[w].z);
    } else {  // written by PlanKernel
        const PlanEntry pe = a.plan[w * a.tiles + t];
        lo = (int)pe.b;
        hi = (int)pe.e;
        r = __ldcg(a.wrow + w);
    }
    if (r >= 0 && lo < hi) {
        const uint4 o = __ldg(reinterpret_cast<const uint4 *>(a.boff + ((long long)r * a.tiles + t) * 8));
        const unsigned off[4] = {o.x, o.y, o.z, o.w};
        const int first = __ffs((int)mask) - 1, last = 31 - __clz((int)mask);
        int ofirst = 0, oend = hi - lo;
#pragma unroll
        for (int j = 0; j < 8; ++j) {  // register-indexed: no local memory
            const int oj = (int)((off[j >> 1] >> ((j & 1) * 16)) & 0xffffu);
            if (j == first)
                ofirst = oj;
            if (j == last + 1)
                oend = oj;
        }
        hi = lo + oend;
        lo += ofirst;
    } else if (r == -2) {
        hi = lo;
    }
}

__global__ void __launch_bounds__(kWtThreads, 3) BlockTileKernel(const StreamArgs a)
{
    extern __shared__ __align__(128) unsigned char wt_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float *row = reinterpret_cast<float *>(wt_smem) + (size_t)warp * kWtTile;
    float4 *row4 = reinterpret_cast<float4 *>(row);
    WtShared &sh = *reinterpret_cast<WtShared *>(wt_smem + (size_t)kWtWarps * kWtTile * sizeof(float));
    WarpSel &ws = sh.wsel[warp];
#pragma unroll
    for (int j = 0; j < kWtTile / 128; ++j)
        row4[lane + 32 * j] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncwarp();
    AllowDependents();
    WaitPrerequisites();  // the work list of the block bound kernel
    const unsigned count = (unsigned)min((long long)__ldcg(a.item_count), a.item_cap);
    if (count == 0)
        return;  // no item (an empty retry list), the same for every warp: the counter is left untouched
    unsigned bad = 0;
    unsigned long long read = 0;

    unsigned nxt = 0;
    if (lane == 0)
        nxt = atomicAdd(&a.ctrl->next, 1u);
    for (;;) {
        const unsigned c = __shfl_sync(kFull, nxt, 0);
        if (c >= count)
            break;
        if (lane == 0)
            nxt = atomicAdd(&a.ctrl->next, 1u);  // the next item, in flight meanwhile
        const uint4 item = __ldcg(a.items + c);
        const int q = (int)(item.x & 0xffffu), t = (int)item.y;
        unsigned mask = (item.x >> 16) & 0xffu;
        const long long qb = (long long)item.z;
        // a routed query is streamed by the warp-tile kernel: its items are skipped
        const int n = a.route_limit && __ldcg(a.qkept + q) > a.route_limit ? 0 : (int)item.w;
        if (n == 0 || mask == 0u)
            continue;  // uniform
        const int k = QueryK(a, q);
        const unsigned thr_bits = lane == 0 ? __ldcg(a.threshold + q) : 0u;
        const unsigned slot_bits = lane < min(k, 32) ? __ldcg(a.tslots + (long long)q * 32 + lane) : 0xffffffffu;
        const int base_doc = t * kWtTile;
        float rmax = 0.0f;
        bool any = false;
        for (int s0 = 0; s0 < n; s0 += 32) {  // uniform; more than 32 words is rare
            const int nw = min(32, n - s0);
            int lo = 0, hi = 0;
            if (lane < nw)
                BtWordRange(a, qb + s0 + lane, t, mask, lo, hi);
            any |= hi > lo;
            read += (unsigned long long)max(0, hi - lo);
            // words in groups of kWtLead: the first window of every word of a group is loaded at once,
            // then the group's words are added in query order
            for (int g = 0; g < nw; g += kWtLead) {  // uniform
                int lid[kWtLead][4];
                float lval[kWtLead][4];
#pragma unroll
                for (int u = 0; u < kWtLead; ++u) {
                    const int b = __shfl_sync(kFull, lo, g + u), e = __shfl_sync(kFull, hi, g + u);
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        const int p = b + lane + 32 * v;
                        lid[u][v] = -1;
                        lval[u][v] = 0.0f;
                        if (g + u < nw && p < e) {
                            lid[u][v] = LdStreamI32(a.indices + p);
                            lval[u][v] = LdStreamF32(a.data + p);
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < kWtLead; ++u) {
                    if (g + u >= nw)
                        break;  // uniform
                    __syncwarp();  // the previous word's adds are in the row before this word's
                    const int b = __shfl_sync(kFull, lo, g + u), e = __shfl_sync(kFull, hi, g + u);
                    WtScatter(lid[u], lval[u], base_doc, row, rmax, bad);
                    WtWordWindows(a, b + kWtWindow, e, base_doc, row, lane, rmax, bad);
                }
            }
        }
        __syncwarp();
        if (!__any_sync(kFull, any))
            continue;  // nothing was added: the row is clear
        const float thr = fmaxf(__uint_as_float(__shfl_sync(kFull, thr_bits, 0)),
                                __uint_as_float(__reduce_min_sync(kFull, slot_bits)));
        if (__any_sync(kFull, rmax >= fmaxf(thr, kLeastPositive)))
            bad |= TileSelectAppend<kWtTile>(a, ws, row4, thr, q, t, lane, mask);  // clears the kept blocks
        else
            mask = 0u;
        // the rest of the row (dropped blocks inside a word's run; every block when nothing was selected)
#pragma unroll
        for (int j = 0; j < kWtTile / 128; ++j)
            if (!((mask >> j) & 1u))
                row4[lane + 32 * j] = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncwarp();
    }

    bad = __reduce_or_sync(kFull, bad);
    read = __reduce_add_sync(kFull, (unsigned)read);
    if (lane == 0) {
        if (bad)
            atomicOr(a.status, bad);
        sh.counters[warp][0] = sh.counters[warp][1] = 0u;
        sh.counters[warp][2] = (unsigned)read;
    }
    WtRetire(a, sh, kStatPostingsRead);
}

} // namespace bm25k
