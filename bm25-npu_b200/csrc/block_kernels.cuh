// Block-max pruned Search (no counterpart in the reference; the learned part of
// the engine).
//
// Index (prune sessions): for every directory row (a long posting list) and every
// tile, the posting offset of each 128-document block from the tile's start
// (uint16: a tile holds at most one posting per document) and the block's largest
// posting score.  Short lists are bounded from their few postings on the fly.
//
// Search, after PlanKernel has resolved every query word's posting range per tile:
// BlockBoundKernel -- one thread per (query, tile): adds, per 128-document block,
//   the query words' block maxima in query-word order.  Rounded addition is
//   monotone in both operands, so the FP32 sum bounds every document's FP32 sum
//   in the block (which adds the document's own contributions, each at most the
//   word's block maximum, in the same order).  Blocks whose bound is below the
//   query's starting bound tau (or zero) are dropped; tiles with a kept block go
//   to a compact work list with their kept-block mask.  The query's running
//   bound starts at tau.
// BlockScoreKernel -- persistent warps over the work list: a warp fetches the
//   item's word metadata lane-parallel (plan range, directory row, block
//   offsets), stages the kept blocks' postings of all its words in shared memory
//   with asynchronous 4-byte copies (cp.async, all in flight at once), adds them
//   word by word into its private shared-memory row (FP32, query-word order),
//   then selects and appends like the tile-group consumers (TileSelectAppend).
// A dropped block holds no document at or above tau, so whenever K documents
// reach tau the top K all lie in kept blocks and are appended; FinalSelect
// reports per query whether K did (else the retry pass answers the query).
#pragma once
#include "tile_group_kernel.cuh"

namespace bm25k {

constexpr int kBlockDocs = 128;
constexpr int kBsWarps = 8;
constexpr int kBsThreads = kBsWarps * 32;
constexpr int kBbThreads = 128;

// Block offsets and maxima of directory row r in tile t (thread per (row, tile)).  A maximum is
// stored rounded up to FP16 (never below the FP32 value: still a bound, half the bytes the block
// bound kernel reads per (word, tile)); a maximum past FP16's range becomes +inf, which keeps the
// block.
__global__ void BuildBlockIndexKernel(const long long *indptr, const int *indices, const float *data,
                                      const int *dir_terms, const int *dir, long long rows, int tiles, long long stride,
                                      int tile_docs, unsigned short *boff, __half *bmax)
{
    const int nb = tile_docs / kBlockDocs;
    const long long total = rows * (long long)tiles;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / tiles;
        const int t = (int)(i % tiles);
        const long long s = indptr[dir_terms[r]];
        const int *d = dir + r * stride;
        const long long b = s + d[t], e = s + d[t + 1];
        unsigned short *o = boff + i * nb;
        __half *m = bmax + i * nb;
        int blk = 0;
        float mx = 0.0f;
        o[0] = 0;
        for (long long p = b; p < e; ++p) {
            const int bi = min(nb - 1, max(0, (indices[p] - t * tile_docs) / kBlockDocs));
            while (blk < bi) {
                m[blk] = __float2half_ru(mx);
                mx = 0.0f;
                ++blk;
                o[blk] = (unsigned short)(p - b);
            }
            mx = fmaxf(mx, data[p]);  // fmaxf(0, negative) = 0: a negative score is bounded by 0
        }
        m[blk] = __float2half_ru(mx);
        for (int j = blk + 1; j < nb; ++j) {
            o[j] = (unsigned short)(e - b);
            m[j] = __float2half(0.0f);
        }
    }
}

// grid (ceil(tiles / kBbThreads), Q): thread = (query blockIdx.y, tile).
template <int kTile>
__global__ void __launch_bounds__(kBbThreads) BlockBoundKernel(const StreamArgs a)
{
    constexpr int kNb = kTile / kBlockDocs;
    const int t = blockIdx.x * kBbThreads + threadIdx.x, lane = threadIdx.x & 31;
    AllowDependents();    // the block scorer may be placed meanwhile
    WaitPrerequisites();  // the plan, or the fail list of the final select before a retry
    int q = blockIdx.y;
    float tau;
    if (a.retry) {
        // a query whose first pass fell short: its bound is now a proven one, the larger of its
        // group slots' least (real documents' scores) and its safe bound from term statistics
        if ((unsigned)q >= __ldcg(a.fail_in_count))
            return;
        q = __ldcg(a.fail_in + q);
        const int k = QueryK(a, q), ns = min(k, 32);
        const unsigned slot = lane < ns ? __ldcg(a.tslots + (long long)q * 32 + lane) : 0xffffffffu;
        tau = __uint_as_float(__reduce_min_sync(kFull, slot));
        if (a.safe)
            tau = fmaxf(tau, a.safe[q]);
    } else {
        tau = a.tau[q];
    }
    tau = tau > 0.0f ? tau : 0.0f;  // NaN or negative: no bound
    if (t == 0)
        a.threshold[q] = __float_as_uint(tau);
    const long long qb = a.qoffsets[q], qe = a.qoffsets[q + 1];
    long long n = qe - qb;
    if (n < 0 || n > kMaxTerms || qb < 0 || qb + n > a.word_cap)
        n = 0;  // PlanKernel reports the malformed query
    unsigned keep = 0;
    if (t < a.tiles) {
        float bound[kNb];
#pragma unroll
        for (int j = 0; j < kNb; ++j)
            bound[j] = 0.0f;
        // kPf words at a time: their rows and plan ranges, then the directory words' block maxima,
        // all loaded before the sums, which run in query-word order
        constexpr int kPf = kTile == 1024 ? 4 : 2;
        for (long long s0 = 0; s0 < n; s0 += kPf) {
            int r[kPf];
            PlanEntry pe[kPf];
#pragma unroll
            for (int u = 0; u < kPf; ++u) {
                r[u] = -2;
                pe[u] = PlanEntry{0, 0};
                if (s0 + u < n) {
                    const long long w = qb + s0 + u;
                    if (a.rows_plan) {  // written by PlanRowsKernel
                        const int *row = a.plan_rows + w * a.dir_stride + t;
                        r[u] = __ldcg(&a.word_rec[w].z);
                        pe[u] = PlanEntry{__ldcg(row), __ldcg(row + 1)};
                    } else {  // written by PlanKernel
                        r[u] = __ldcg(a.wrow + w);
                        pe[u] = a.plan[w * a.tiles + t];
                    }
                }
            }
            float m[kPf][kNb];
#pragma unroll
            for (int u = 0; u < kPf; ++u) {
#pragma unroll
                for (int j = 0; j < kNb; ++j)
                    m[u][j] = 0.0f;
                if (r[u] >= 0 && pe[u].b < pe[u].e) {  // 8 FP16 maxima per 16-byte load
                    const uint4 *src =
                        reinterpret_cast<const uint4 *>(a.bmax + ((long long)r[u] * a.tiles + t) * kNb);
#pragma unroll
                    for (int j = 0; j < kNb / 8; ++j) {
                        const uint4 v = __ldg(src + j);
                        const unsigned h[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                        for (int x = 0; x < 4; ++x) {  // the lower half of each word is the earlier block
                            m[u][8 * j + 2 * x] = __half2float(__ushort_as_half((unsigned short)(h[x] & 0xffffu)));
                            m[u][8 * j + 2 * x + 1] = __half2float(__ushort_as_half((unsigned short)(h[x] >> 16)));
                        }
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kPf; ++u) {
                if (r[u] == -2 || pe[u].b >= pe[u].e)
                    continue;  // not a valid term, or no posting in the tile: adds 0
                if (r[u] == -1) {  // a short list: the maxima from its few postings in the tile
                    for (long long p = pe[u].b; p < pe[u].e; ++p) {
                        const int bi = (__ldg(a.indices + p) - t * kTile) / kBlockDocs;
                        const float v = fmaxf(__ldg(a.data + p), 0.0f);
#pragma unroll
                        for (int j = 0; j < kNb; ++j)
                            m[u][j] = bi == j ? fmaxf(m[u][j], v) : m[u][j];
                    }
                }
#pragma unroll
                for (int j = 0; j < kNb; ++j)
                    bound[j] = __fadd_rn(bound[j], m[u][j]);
            }
        }
#pragma unroll
        for (int j = 0; j < kNb; ++j)
            if (bound[j] > 0.0f && bound[j] >= tau)
                keep |= 1u << j;
    }
    if (a.qkept) {  // this CTA's kept blocks, one atomic per warp
        const unsigned kept = __reduce_add_sync(kFull, (unsigned)__popc(keep));
        if (lane == 0 && kept)
            atomicAdd(a.qkept + q, kept);
    }
    // warp-aggregated append of the tiles with a kept block
    const unsigned has = __ballot_sync(kFull, keep != 0);
    if (!has)
        return;
    unsigned base = 0;
    if (lane == 0)
        base = atomicAdd(a.item_count, (unsigned)__popc(has));
    base = __shfl_sync(kFull, base, 0);
    if (keep) {
        const unsigned at = base + __popc(has & ((1u << lane) - 1u));
        if ((long long)at < a.item_cap)
            a.items[at] = make_uint4((unsigned)q | (keep << 16), (unsigned)t, (unsigned)qb, (unsigned)n);
        else
            atomicOr(a.status, kStatusCandOverflow);  // cannot happen: item_cap covers every (query, tile)
    }
    if (a.stats) {
        const unsigned kept = __reduce_add_sync(kFull, (unsigned)__popc(keep));
        if (lane == 0) {
            atomicAdd(a.stats + kStatItems, (unsigned long long)__popc(has));
            atomicAdd(a.stats + kStatBlocksKept, (unsigned long long)kept);
        }
    }
}

constexpr int kBsStage = 512;  // postings a warp stages in shared memory between flushes

inline size_t BlockScoreSmem(int tile_docs)
{
    return (size_t)kBsWarps * tile_docs * sizeof(float) + (size_t)kBsWarps * kBsStage * 2 * sizeof(int) +
           (size_t)kBsWarps * sizeof(WarpSel);
}

// 4-byte asynchronous copy global -> shared (cp.async, no multicast).
__device__ __forceinline__ void CpAsync4(void *smem, const void *gmem)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}

__device__ __forceinline__ void CpAsyncWaitAll()
{
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

template <int kTile>
__global__ void __launch_bounds__(kBsThreads, kTile == 1024 ? 3 : 2) BlockScoreKernel(const StreamArgs a)
{
    constexpr int kNb = kTile / kBlockDocs;
    extern __shared__ __align__(16) unsigned char bs_smem[];
    float *rows = reinterpret_cast<float *>(bs_smem);
    int *stage_ids = reinterpret_cast<int *>(rows + (size_t)kBsWarps * kTile);
    float *stage_vals = reinterpret_cast<float *>(stage_ids + (size_t)kBsWarps * kBsStage);
    WarpSel *wsel = reinterpret_cast<WarpSel *>(stage_vals + (size_t)kBsWarps * kBsStage);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    AllowDependents();
    WaitPrerequisites();  // the work list of the block bound kernel
    const unsigned count = (unsigned)min((long long)__ldcg(a.item_count), a.item_cap);
    if (blockIdx.x * kBsWarps >= count)
        return;  // no item for any warp of this CTA (an empty retry list among them)
    for (int i = tid; i < kBsWarps * kTile / 4; i += kBsThreads)
        reinterpret_cast<float4 *>(rows)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    float *row = rows + (size_t)warp * kTile;
    float4 *row4 = reinterpret_cast<float4 *>(row);
    int *sid = stage_ids + (size_t)warp * kBsStage;
    float *sval = stage_vals + (size_t)warp * kBsStage;
    unsigned bad = 0;
    unsigned long long read = 0;
    // Word metadata of one item, lane l holding word s0 + l: plan range, directory row (-2: not a
    // valid term) and block offsets.  fetch_rows issues the first loads, fetch_offsets the
    // dependent block offsets; items are software-pipelined: while item i's postings are in
    // flight, item i + 1's metadata loads are, and item i + 2's record.
    struct Meta {
        int pb, pe, r;
        unsigned o[kNb / 2];
        unsigned slot, thr;
    };
    auto fetch_rows = [&](const uint4 item, int s0, Meta &m) {
        const int n = (int)item.w, q = (int)(item.x & 0xffffu), t = (int)item.y;
        const long long qb = (long long)item.z;
        const int s = s0 + lane;
        m.pb = m.pe = 0;
        m.r = -2;
#pragma unroll
        for (int j = 0; j < kNb / 2; ++j)
            m.o[j] = 0u;
        if (s < n) {
            m.r = __ldcg(a.wrow + qb + s);
            const PlanEntry e = a.plan[(qb + s) * a.tiles + t];
            m.pb = (int)e.b;
            m.pe = (int)e.e;
        }
        m.slot = lane < QueryK(a, q) ? __ldcg(a.tslots + (long long)q * 32 + lane) : 0xffffffffu;
        m.thr = __ldcg(a.threshold + q);
    };
    auto fetch_offsets = [&](const uint4 item, Meta &m) {
        if (m.r >= 0 && m.pb < m.pe) {
            const uint4 *src = reinterpret_cast<const uint4 *>(a.boff + ((long long)m.r * a.tiles + item.y) * kNb);
#pragma unroll
            for (int j = 0; j < kNb / 8; ++j) {
                const uint4 v = __ldg(src + j);
                m.o[4 * j] = v.x;
                m.o[4 * j + 1] = v.y;
                m.o[4 * j + 2] = v.z;
                m.o[4 * j + 3] = v.w;
            }
        }
    };
    const unsigned stride = gridDim.x * kBsWarps;
    unsigned it = blockIdx.x * kBsWarps + warp;
    const uint4 none = make_uint4(0u, 0u, 0u, 0u);
    uint4 item = it < count ? __ldcg(a.items + it) : none;
    Meta cur;
    fetch_rows(item, 0, cur);
    fetch_offsets(item, cur);
    uint4 next = it + stride < count ? __ldcg(a.items + it + stride) : none;
    for (; it < count; it += stride) {
        const bool more = it + stride < count;
        Meta nxt;
        fetch_rows(next, 0, nxt);  // loads in flight while this item is scored
        const uint4 after = it + 2 * stride < count ? __ldcg(a.items + it + 2 * stride) : none;
        const int q = (int)(item.x & 0xffffu), t = (int)item.y;
        // a routed query is streamed by the tile-group kernel: its items are skipped
        const int n = a.route_limit && __ldcg(a.qkept + q) > a.route_limit ? 0 : (int)item.w;
        const unsigned mask = item.x >> 16;
        // running bound: the threshold (seeded with tau) or the least group slot when higher
        const float thr = fmaxf(__uint_as_float(cur.thr), __uint_as_float(__reduce_min_sync(kFull, cur.slot)));
        const int base = t * kTile;
        bool shortw = false;  // a short list (no block offsets) added postings of every block
        for (int s0 = 0; s0 < n; s0 += 32) {
            Meta m = cur;
            if (s0 > 0) {  // more than 32 words: the next ones' metadata, fetched here
                fetch_rows(item, s0, m);
                fetch_offsets(item, m);
            }
            // Stage the words' kept postings in query-word order with asynchronous copies, all in
            // flight at once; a flush waits for them and adds them word by word (lane i holds the
            // staged range of the i-th staged word), before the stage would overflow and at the end.
            int fill = 0, staged = 0, my_lo = 0, my_hi = 0;
            auto flush = [&]() {
                CpAsyncWaitAll();
                __syncwarp();
                for (int i = 0; i < staged; ++i) {
                    const int lo = __shfl_sync(kFull, my_lo, i), hi = __shfl_sync(kFull, my_hi, i);
                    for (int x = lo + lane; x < hi; x += 32) {
                        const int d = sid[x] - base;
                        if ((unsigned)d < (unsigned)kTile)
                            row[d] += sval[x];
                        else
                            bad |= kStatusBadPosting;
                    }
                    __syncwarp();  // this word's adds land before the next word's
                }
                fill = 0;
                staged = 0;
            };
            const int words = min(32, n - s0);
            // 1024-document tiles: the words' block offsets go to a table in the warp's selection
            // scratch (unused until the select), one 16-byte row per word
            unsigned short *otab = reinterpret_cast<unsigned short *>(&wsel[warp]);
            if (kNb == 8) {
                static_assert(sizeof(WarpSel) >= 32 * 16, "offset table fits the selection scratch");
                __syncwarp();  // the previous chunk's reads are done
                reinterpret_cast<uint4 *>(otab)[lane] = make_uint4(m.o[0], m.o[1 % (kNb / 2)], m.o[2 % (kNb / 2)],
                                                                   m.o[3 % (kNb / 2)]);
                __syncwarp();
            }
            for (int w = 0; w < words; ++w) {  // query-word order
                const int b = __shfl_sync(kFull, m.pb, w), e = __shfl_sync(kFull, m.pe, w);
                const int rw = __shfl_sync(kFull, m.r, w);
                if (b >= e || rw == -2)
                    continue;
                unsigned off[kNb / 2];
                if (kNb != 8) {
#pragma unroll
                    for (int j = 0; j < kNb / 2; ++j)
                        off[j] = __shfl_sync(kFull, m.o[j], w);
                }
                shortw |= rw < 0;
                int start = fill;
                for (unsigned mk = rw >= 0 ? mask : 1u; mk; mk &= mk - 1) {
                    int lo = b, hi = e;  // a short list: all its postings in the tile, filtered when added
                    if (rw >= 0) {
                        const int j = __ffs(mk) - 1;
                        if (kNb == 8) {
                            lo = b + otab[w * 8 + j];
                            if (j + 1 < kNb)
                                hi = b + otab[w * 8 + j + 1];
                        } else {
#pragma unroll
                            for (int u = 0; u < kNb; ++u) {  // register-indexed: no local memory
                                const int ou = (int)((off[u >> 1] >> ((u & 1) * 16)) & 0xffffu);
                                if (u == j)
                                    lo = b + ou;
                                if (u == j + 1)
                                    hi = b + ou;
                            }
                        }
                    }
                    for (int c = lo; c < hi;) {
                        if (fill == kBsStage) {  // close this word's part and flush
                            if (lane == staged) {
                                my_lo = start;
                                my_hi = fill;
                            }
                            ++staged;
                            flush();
                            start = 0;
                        }
                        const int len = min(hi - c, kBsStage - fill);
                        for (int x = lane; x < len; x += 32) {
                            CpAsync4(sid + fill + x, a.indices + c + x);
                            CpAsync4(sval + fill + x, a.data + c + x);
                        }
                        if (lane == 0)
                            read += (unsigned long long)len;
                        fill += len;
                        c += len;
                    }
                }
                if (fill > start) {
                    if (lane == staged) {
                        my_lo = start;
                        my_hi = fill;
                    }
                    ++staged;
                }
                if (staged == 32)
                    flush();
            }
            if (s0 == 0 && more)
                fetch_offsets(next, nxt);  // its rows have arrived by now; its offsets fly with our postings
            if (staged)
                flush();
        }
        if (n == 0 && more)
            fetch_offsets(next, nxt);
        // a short list's postings outside the kept blocks were staged too: clear them (the select
        // reads the kept blocks only, and every block must be zero for the next item)
        if (shortw && mask != (1u << kNb) - 1u) {
#pragma unroll
            for (int j = 0; j < kNb; ++j)
                if (!((mask >> j) & 1u))
                    row4[lane + 32 * j] = make_float4(0.f, 0.f, 0.f, 0.f);
            __syncwarp();
        }
        bad |= TileSelectAppend<kTile>(a, wsel[warp], row4, thr, q, t, lane, mask);
        __syncwarp();
        item = next;
        cur = nxt;
        next = after;
    }
    bad = __reduce_or_sync(kFull, bad);
    if (lane == 0) {
        if (bad)
            atomicOr(a.status, bad);
        if (a.stats && read)
            atomicAdd(a.stats + kStatPostingsRead, read);
    }
}

// One CTA: the queries that keep more than route_limit blocks, for the tile-group kernel.
__global__ void RouteKernel(const StreamArgs a)
{
    unsigned routed = 0;
    for (int q = threadIdx.x; q < a.q; q += blockDim.x)
        if (__ldcg(a.qkept + q) > a.route_limit) {
            a.route_list[atomicAdd(a.route_count, 1u)] = q;
            ++routed;
        }
    if (a.stats && routed)
        atomicAdd(a.stats + kStatRouted, (unsigned long long)routed);
}

inline const void *BlockScoreKernelFor(int tile_docs)
{
    return tile_docs == 2048 ? reinterpret_cast<const void *>(&BlockScoreKernel<2048>)
                             : reinterpret_cast<const void *>(&BlockScoreKernel<1024>);
}

} // namespace bm25k
