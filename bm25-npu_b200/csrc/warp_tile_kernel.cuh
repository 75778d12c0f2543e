// Warp-tile BM25 Search kernel for sm_100a (kernel 5, the default plain path).
//
// The reference scores one (query, 8192-document leaf) per task, streaming each
// query term's postings through the unified buffer
//   feature_retrieval/src/ascendfaiss/ops/ascendc/bm25/fused/op_kernel/bm25_fused_score_top_k.cpp:637-793
// This kernel gives every warp its own work and its own data path:
//   * a claim is one query and kC consecutive 1024-document tiles; warps take
//     claims from one global counter (the atomic for the next claim is in
//     flight while the current one runs), in tile-major order, so every query
//     gets tiles early and its running bound rises at once; the last tiles
//     (about two claims per warp) are claimed one at a time, so the launch does
//     not end waiting on a few warps with long claims of a dense query;
//   * the warp resolves the claim itself: lane s holds query word s's posting
//     position at each of the claim's kC + 1 tile bounds, read from the word's
//     plan row (PlanRowsKernel: the directory row made absolute for a long list,
//     built from the postings for a short one) with its word record (seed, dense
//     row) in one round of loads, and issues one L2 prefetch per word for the
//     postings of all kC tiles (cp.async.bulk.prefetch.L2: no shared memory, no
//     registers held while the bytes are in flight);
//   * per tile the warp loads its postings straight from global memory into
//     registers -- the first window (128 postings) of each of the query's first
//     kWtLead words at once, so a typical tile waits for memory once, the rest
//     of a long word two windows at a time (lane l takes postings l, l + 32,
//     l + 64, l + 96 of a window, so consecutive lanes add consecutive
//     documents of a dense list into distinct shared-memory banks) -- and adds
//     them into its private 4 KB FP32 row in query-word order (a __syncwarp
//     between words orders the lanes: each document's sum is
//     ((0 + s_1) + s_2) + ... as in cpu_index_search.h:176-188).  A word kept as
//     a dense row (df >= dense_density * N) is added from that row instead:
//     1024 scores with 128-bit loads, zero where the word is absent (adding +0
//     leaves a sum unchanged);
//   * then it selects the tile's top-K at or above the query's running bound
//     (TileSelectAppend, shared with the tile-group kernel) and clears the row.
//     The lanes keep the largest sum they wrote, which is the tile's largest
//     score (contributions are non-negative, so a document's final sum is the
//     largest it takes); a tile whose largest score is below the bound only
//     clears its row.
// A query's running bound starts at the largest, over its words, of the word's
// K-th largest posting score (K <= 32; for K up to 1024, its score at the
// smallest rank 64, 128, ..., 1024 not below K) from term statistics kept at
// create: that many documents hold the word with at least that score, and a
// non-negative FP32 sum is at least each of its terms, so K documents reach it.  Without it the
// first wave of claims (every warp's first tiles) would run with no bound and
// select and append in full.
// No producer warp, no mbarrier, no wait on another warp: the only latencies
// are the warp's own loads.  FinalSelectKernel finishes every query.
//
// A retry pass (a.retry) covers only the queries of the fail list, as in the
// tile-group kernel.
#pragma once
#include "tile_group_kernel.cuh"

namespace bm25k {

constexpr int kWtTile = 1024;        // documents per tile (one warp's row)
constexpr int kWtWarps = 8;
constexpr int kWtThreads = kWtWarps * 32;
constexpr int kWtWindow = 128;       // postings per window (4 per lane)
constexpr int kWtLead = 3;           // words whose first window is loaded before any add
constexpr int kPlanRowChunk = 1024;  // plan row entries per PlanRowsKernel CTA (grid.y; 2048: +1.2 us per Search at 10M)
constexpr int kTermTopK = 32;        // largest posting scores kept per term

constexpr int kWtMaxC = 8;           // largest kC: claim bounds kept per word

struct WtShared {
    WarpSel wsel[kWtWarps];
    // words 32..63 of a claim's query (rare: at most 64 words per query): their posting positions at
    // the claim's tile bounds and their dense rows, per warp; words 0..31 are held in registers
    int offB[kWtWarps][32][kWtMaxC + 1];
    int drowB[kWtWarps][32];
    unsigned counters[kWtWarps][3];  // claims, tiles, postings of the warp
};

inline size_t WarpTileSmem() { return (size_t)kWtWarps * kWtTile * sizeof(float) + sizeof(WtShared); }

// Streaming loads of postings: read once, so they do not displace the query and directory lines
// in L1.
__device__ __forceinline__ int LdStreamI32(const int *p)
{
    int v;
    asm("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ float LdStreamF32(const float *p)
{
    float v;
    asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ float4 LdStreamF32x4(const float4 *p)
{
    float4 v;
    asm("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(p));
    return v;
}

// Prefetch of [p, p + bytes) into L2 (p 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void PrefetchL2(const void *p, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Posting positions of query word w at the bounds of the claim's tiles t0 .. t0 + nt (j > nt
// repeats the last bound): off[j] = first posting of the word's list in tile t0 + j, from the word's
// plan row; seed raised to the word's starting-bound seed, drow = its dense row or -1 (both from
// its word record).  Both are written by PlanRowsKernel before this kernel reads them, so a claim
// resolves its words with one round of independent loads.
template <int kC>
__device__ __forceinline__ void WtWordRow(const StreamArgs &a, long long w, int t0, int nt, int *off, float &seed,
                                          int &drow)
{
    const int *row = a.plan_rows + w * a.dir_stride + t0;
#pragma unroll
    for (int j = 0; j <= kC; ++j)
        off[j] = __ldcg(row + min(j, nt));
    const int4 r = __ldcg(a.word_rec + w);
    seed = fmaxf(seed, __int_as_float(r.x));
    drow = r.y;
}

// L2 prefetch of postings [lo, hi) of both arrays, widened to 16-byte boundaries (the arrays are
// padded past their end).
__device__ __forceinline__ void PrefetchRun(const StreamArgs &a, int lo, int hi, int drow, int t0, int nt)
{
    if (lo >= hi)
        return;
    if (drow >= 0) {  // the dense row's scores of the claim's tiles
        PrefetchL2(a.dense + (long long)drow * a.dense_stride + (long long)t0 * kWtTile,
                   (unsigned)nt * kWtTile * (unsigned)sizeof(float));
        return;
    }
    const int p0 = lo & ~3, p1 = (hi + 3) & ~3;
    const unsigned bytes = (unsigned)(p1 - p0) * 4u;
    PrefetchL2(a.indices + p0, bytes);
    PrefetchL2(a.data + p0, bytes);
}

// Adds one window set of a word: lane l's postings l, l + 32, l + 64, l + 96 of the window (ids -1:
// none) into the warp's row.  A word's postings are distinct documents, so the lanes never collide.
__device__ __forceinline__ void WtScatter(const int (&id)[4], const float (&val)[4], int base_doc, float *row,
                                          float &rmax, unsigned &bad)
{
    int d[4];
    float r[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        d[v] = id[v] - base_doc;
        if (id[v] >= 0 && (unsigned)d[v] >= (unsigned)kWtTile)
            bad |= kStatusBadPosting;
    }
#pragma unroll
    for (int v = 0; v < 4; ++v)
        if ((unsigned)d[v] < (unsigned)kWtTile)
            r[v] = row[d[v]];
#pragma unroll
    for (int v = 0; v < 4; ++v)
        if ((unsigned)d[v] < (unsigned)kWtTile) {
            const float x = r[v] + val[v];
            row[d[v]] = x;
            rmax = fmaxf(rmax, x);
        }
}

// Postings [b, e) of one word in the tile, two windows (256 postings) per round.
__device__ __forceinline__ void WtWordWindows(const StreamArgs &a, int b, int e, int base_doc, float *row, int lane,
                                              float &rmax, unsigned &bad)
{
    for (int p0 = b; p0 < e; p0 += 2 * kWtWindow) {  // uniform
        int id[2][4];
        float val[2][4];
#pragma unroll
        for (int w = 0; w < 2; ++w)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int p = p0 + w * kWtWindow + lane + 32 * v;
                id[w][v] = -1;
                val[w][v] = 0.0f;
                if (p < e) {
                    id[w][v] = LdStreamI32(a.indices + p);
                    val[w][v] = LdStreamF32(a.data + p);
                }
            }
        WtScatter(id[0], val[0], base_doc, row, rmax, bad);
        WtScatter(id[1], val[1], base_doc, row, rmax, bad);
    }
}

// A word kept as a dense row: the tile's 1024 scores, 8 x 128 bits per lane, added in place.
__device__ __forceinline__ void WtDenseAdd(const StreamArgs &a, int drow, int base_doc, float4 *row4, int lane,
                                           float &rmax)
{
    const float4 *src = reinterpret_cast<const float4 *>(a.dense + (long long)drow * a.dense_stride + base_doc);
    float4 v[kWtTile / 128];
#pragma unroll
    for (int z = 0; z < kWtTile / 128; ++z)
        v[z] = LdStreamF32x4(src + lane + 32 * z);
#pragma unroll
    for (int z = 0; z < kWtTile / 128; ++z) {
        float4 r = row4[lane + 32 * z];
        r.x += v[z].x;
        r.y += v[z].y;
        r.z += v[z].z;
        r.w += v[z].w;
        row4[lane + 32 * z] = r;
        rmax = fmaxf(rmax, fmaxf(fmaxf(r.x, r.y), fmaxf(r.z, r.w)));
    }
}

// End of a warp-tile style kernel: the CTA's counters (claims, tiles, postings: statistic stat2)
// go to the Search's statistics and the CTA counts itself done, one thread for the CTA (the warps
// all finish at about the same time, and per-warp atomics on these few addresses would queue up
// behind one another at the launch's end); the last CTA to finish resets the work counter for the
// next pass.
__device__ __forceinline__ void WtRetire(const StreamArgs &a, WtShared &sh, int stat2 = kStatPostingsCopied)
{
    __syncthreads();  // every warp has taken its last claim and written its counters
    if (threadIdx.x != 0)
        return;
    unsigned long long c[3] = {0ull, 0ull, 0ull};
#pragma unroll
    for (int w = 0; w < kWtWarps; ++w)
#pragma unroll
        for (int x = 0; x < 3; ++x)
            c[x] += sh.counters[w][x];
    if (a.stats) {
        if (c[0])
            atomicAdd(a.stats + kStatClaims, c[0]);
        if (c[1])
            atomicAdd(a.stats + kStatTilesScanned, c[1]);
        if (c[2])
            atomicAdd(a.stats + stat2, c[2]);
    }
    const unsigned d = atomicAdd(&a.ctrl->done, 1u);
    if (d == gridDim.x - 1) {
        a.ctrl->next = 0u;
        a.ctrl->done = 0u;
    }
}

// kC: tiles per claim.  kLean: the plain first pass with one K <= 32 for every query.
template <int kC, bool kLean>
__global__ void __launch_bounds__(kWtThreads, 3) WarpTileKernel(const StreamArgs a)
{
    static_assert(kC <= kWtMaxC, "claim bounds of words 32..63 are kept for kWtMaxC tiles");
    extern __shared__ __align__(128) unsigned char wt_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float *row = reinterpret_cast<float *>(wt_smem) + (size_t)warp * kWtTile;
    float4 *row4 = reinterpret_cast<float4 *>(row);
    WtShared &sh = *reinterpret_cast<WtShared *>(wt_smem + (size_t)kWtWarps * kWtTile * sizeof(float));
    int *offB = &sh.offB[warp][0][0];  // [32][kWtMaxC + 1]
    WarpSel &ws = sh.wsel[warp];
#pragma unroll
    for (int j = 0; j < kWtTile / 128; ++j)
        row4[lane + 32 * j] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncwarp();
    AllowDependents();    // the final select may be placed as this kernel's CTAs retire
    WaitPrerequisites();  // plan rows (and a retry pass's fail list) of the kernels before this one
    const unsigned nq = !kLean && a.retry ? __ldcg(a.fail_in_count) : (unsigned)a.q;
    if (nq == 0)
        return;  // an empty retry list, the same for every warp: the work counter is left untouched
    const unsigned bulk = (unsigned)min(a.wt_bulk, a.tiles / kC);
    const unsigned claims_bulk = nq * bulk;
    const unsigned claims = claims_bulk + nq * (unsigned)(a.tiles - (int)bulk * kC);
    unsigned bad = 0;
    if (lane == 0)
        sh.counters[warp][0] = sh.counters[warp][1] = sh.counters[warp][2] = 0u;

    unsigned nxt = 0;
    if (lane == 0)
        nxt = atomicAdd(&a.ctrl->next, 1u);
    for (;;) {
        const unsigned c = __shfl_sync(kFull, nxt, 0);
        if (c >= claims)
            break;
        if (lane == 0)
            nxt = atomicAdd(&a.ctrl->next, 1u);  // the next claim, in flight meanwhile

        // ---- the claim: query, tiles, and each word's posting positions at the tile bounds ----
        const bool single = c >= claims_bulk;
        const unsigned cc = single ? c - claims_bulk : c;
        const unsigned qi = cc % nq;
        const int q = !kLean && a.retry ? __ldcg(a.fail_in + qi) : (int)qi;
        const int t0 = single ? (int)(bulk * kC + cc / nq) : (int)(cc / nq) * kC;
        const int nt = single ? 1 : kC;
        const long long qb = __ldg(a.qoffsets + q), qe = __ldg(a.qoffsets + q + 1);
        int nw = (int)(qe - qb);
        if (qe - qb < 0 || qe - qb > kMaxTerms || qb < 0 || qe > a.word_cap) {
            bad |= kStatusBadQuery;
            nw = 0;
        }
        const int k = kLean ? a.k : QueryK(a, q);
        int offA[kC + 1];  // word `lane`'s posting positions at the claim's tile bounds
#pragma unroll
        for (int j = 0; j <= kC; ++j)
            offA[j] = 0;
        float seed = 0.0f;
        int drowA = -1;
        if (lane < nw)
            WtWordRow<kC>(a, qb + lane, t0, nt, offA, seed, drowA);
        if (a.prefetch)
            PrefetchRun(a, offA[0], offA[kC], drowA, t0, nt);
        const unsigned denseA = __ballot_sync(kFull, drowA >= 0);
        unsigned denseB = 0;
        if (nw > 32) {  // uniform: words 32..63 go to shared memory
            int offR[kC + 1];
#pragma unroll
            for (int j = 0; j <= kC; ++j)
                offR[j] = 0;
            int drowB = -1;
            if (lane + 32 < nw)
                WtWordRow<kC>(a, qb + lane + 32, t0, nt, offR, seed, drowB);
            if (a.prefetch)
                PrefetchRun(a, offR[0], offR[kC], drowB, t0, nt);
#pragma unroll
            for (int j = 0; j <= kC; ++j)
                offB[lane * (kWtMaxC + 1) + j] = offR[j];
            sh.drowB[warp][lane] = drowB;
            denseB = __ballot_sync(kFull, drowB >= 0);
            __syncwarp();
        }
        // the largest starting-bound seed of the query's words (0 without term statistics)
        seed = __uint_as_float(__reduce_max_sync(kFull, __float_as_uint(seed)));  // non-negative: bit order
        {
            unsigned posts = (unsigned)(offA[kC] - offA[0]);
            if (nw > 32)
                posts += (unsigned)(offB[lane * (kWtMaxC + 1) + kC] - offB[lane * (kWtMaxC + 1)]);
            posts = __reduce_add_sync(kFull, posts);
            if (lane == 0) {
                sh.counters[warp][0] += 1u;
                sh.counters[warp][1] += (unsigned)nt;
                sh.counters[warp][2] += posts;
            }
        }

        // ---- the claim's tiles ----
        for (int j = 0; j < nt; ++j) {
            const int tile = t0 + j;
            const int base_doc = tile * kWtTile;
            // the query's running bound, read now and used after the adds (other warps raise it)
            const unsigned thr_bits = lane == 0 ? __ldcg(a.threshold + q) : 0u;
            const unsigned slot_bits = lane < k ? __ldcg(a.tslots + (long long)q * 32 + lane) : 0xffffffffu;
            float rmax = 0.0f;  // the largest sum this lane wrote
            // First window (128 postings) of each of the first kWtLead sparse words: loaded at once,
            // so a typical tile waits for memory once.
            int lid[kWtLead][4];
            float lval[kWtLead][4];
#pragma unroll
            for (int s = 0; s < kWtLead; ++s) {
                const int b = __shfl_sync(kFull, offA[0], s), e = __shfl_sync(kFull, offA[1], s);
                const bool sparse = s < nw && !((denseA >> s) & 1u);  // uniform
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int p = b + lane + 32 * v;
                    lid[s][v] = -1;
                    lval[s][v] = 0.0f;
                    if (sparse && p < e) {
                        lid[s][v] = LdStreamI32(a.indices + p);
                        lval[s][v] = LdStreamF32(a.data + p);
                    }
                }
            }
            // the words in query order
#pragma unroll
            for (int s = 0; s < kWtLead; ++s) {
                if (s >= nw)
                    break;  // uniform
                if (s > 0)
                    __syncwarp();  // the previous word's adds are in the row before this word's
                const int b = __shfl_sync(kFull, offA[0], s), e = __shfl_sync(kFull, offA[1], s);
                if ((denseA >> s) & 1u) {
                    if (e > b)
                        WtDenseAdd(a, __shfl_sync(kFull, drowA, s), base_doc, row4, lane, rmax);
                } else {
                    WtScatter(lid[s], lval[s], base_doc, row, rmax, bad);
                    WtWordWindows(a, b + kWtWindow, e, base_doc, row, lane, rmax, bad);
                }
            }
            for (int s = kWtLead; s < nw; ++s) {
                __syncwarp();
                int b, e, drow;
                bool dense;
                if (s < 32) {
                    b = __shfl_sync(kFull, offA[0], s);
                    e = __shfl_sync(kFull, offA[1], s);
                    drow = __shfl_sync(kFull, drowA, s);
                    dense = (denseA >> s) & 1u;
                } else {
                    b = offB[(s - 32) * (kWtMaxC + 1) + j];
                    e = offB[(s - 32) * (kWtMaxC + 1) + j + 1];
                    drow = sh.drowB[warp][s - 32];
                    dense = (denseB >> (s - 32)) & 1u;
                }
                if (dense) {
                    if (e > b)
                        WtDenseAdd(a, drow, base_doc, row4, lane, rmax);
                } else {
                    WtWordWindows(a, b, e, base_doc, row, lane, rmax, bad);
                }
            }
            bool any = lane < nw && offA[1] > offA[0];
            if (nw > 32)
                any |= lane + 32 < nw && offB[lane * (kWtMaxC + 1) + j + 1] > offB[lane * (kWtMaxC + 1) + j];
            const bool W = __any_sync(kFull, any);
            __syncwarp();
            const float thr = fmaxf(fmaxf(seed, __uint_as_float(__shfl_sync(kFull, thr_bits, 0))),
                                    __uint_as_float(__reduce_min_sync(kFull, slot_bits)));
            if (__any_sync(kFull, rmax >= fmaxf(thr, kLeastPositive))) {
                bad |= TileSelectAppend<kWtTile, kLean>(a, ws, row4, thr, q, tile, lane);
                __syncwarp();
            } else if (W > 0) {  // nothing reaches the bound: clear the row (a tile without postings is clear)
#pragma unroll
                for (int z = 0; z < kWtTile / 128; ++z)
                    row4[lane + 32 * z] = make_float4(0.f, 0.f, 0.f, 0.f);
                __syncwarp();
            }
#pragma unroll
            for (int x = 0; x < kC; ++x)
                offA[x] = offA[x + 1];
        }
    }

    bad = __reduce_or_sync(kFull, bad);
    if (lane == 0 && bad)
        atomicOr(a.status, bad);
    WtRetire(a, sh);
}

template <int kC>
inline const void *WarpTileKernelFor(bool lean)
{
    return lean ? reinterpret_cast<const void *>(&WarpTileKernel<kC, true>)
                : reinterpret_cast<const void *>(&WarpTileKernel<kC, false>);
}

// ---- plan rows and word records of a Search's query words ---------------------------------------
//
// rows[w][t] = position of the first posting of word w's list with document >= t * tile_docs, for
// t in [0, tiles] (indptr[term] plus the directory row's entry where the term has one); a word
// outside the vocabulary gets an empty row (all 0), and a negative one is flagged.  CTA (x, y)
// covers row entries [y * kPlanRowChunk, (y + 1) * kPlanRowChunk) of words x, x + gridDim.x, ...
// A word with a directory row copies it; for the others two warps find the chunk's first and last
// posting (32-way searches), the chunk's postings mark the entry of their tile when they are the
// first there, and a suffix minimum fills the entries of the tiles without postings with the next
// marked one: O(postings + tiles) per word.
// The CTAs of chunk 0 also write each word's record: its seed -- the word's posting score at rank
// K of its query (term_top for K <= 32, else the smallest stored rank 64, 128, ..., 1024 not
// below K), which K documents reach (0 without term statistics) --, its dense row, and its
// directory row (-1: a short list; -2: not a term).  One CTA also empties the block path's work
// lists of the Search (when it has them), as PlanKernel does where it runs.
__global__ void __launch_bounds__(kPlanThreads) PlanRowsKernel(const StreamArgs a)
{
    __shared__ int ent[kPlanRowChunk];
    __shared__ int lim[2];
    __shared__ int wmin[kPlanThreads / 32];
    constexpr int kPer = kPlanRowChunk / kPlanThreads;
    static_assert(kPlanRowChunk % kPlanThreads == 0, "whole entries per thread");
    AllowDependents();  // the search kernel sets up its shared memory meanwhile
    if (a.rows_plan && a.item_count && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x < 4)
        a.item_count[threadIdx.x] = 0u;
    long long total = __ldg(a.qoffsets + a.q);
    if (total < 0 || total > a.word_cap) {
        if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0)
            atomicOr(a.status, kStatusBadQuery);
        total = total < 0 ? 0 : a.word_cap;
    }
    const int n_ent = a.tiles + 1;
    const int e0 = (int)blockIdx.y * kPlanRowChunk, e1 = min(n_ent, e0 + kPlanRowChunk);
    if (e0 >= e1) {
        WaitPrerequisites();
        return;
    }
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (long long w = blockIdx.x; w < total; w += gridDim.x) {
        const int term = __ldg(a.words + w);
        int *out = a.plan_rows + w * a.dir_stride;
        const bool known = term >= 0 && term < a.vocab;
        // a K per query: the word's query is the number of q in [1, Q] with qoffsets[q] <= w (the last
        // query starting at or before w), counted by the whole CTA at once (a malformed batch is
        // flagged by the search kernel and fails as a whole)
        int wq = 0;
        if (a.kq && blockIdx.y == 0) {  // uniform
            for (int base = 1; base <= a.q; base += kPlanThreads)
                wq += __syncthreads_count(base + tid <= a.q && __ldg(a.qoffsets + base + tid) <= w);
            wq = min(wq, a.q - 1);
        }
        if (blockIdx.y == 0 && tid == 0) {
            float seed = 0.0f;
            int drow = -1, dr = -2;
            if (known) {
                dr = a.dir_row ? __ldg(a.dir_row + term) : -1;
                const int k = a.kq ? QueryK(a, wq) : a.k;
                if (a.term_top && k <= kTermTopK)
                    seed = __ldg(a.term_top + (long long)term * kTermTopK + (k - 1));
                else if (a.term_rank && k <= 1024)
                    seed = __ldg(a.term_rank + (long long)term * 5 + (31 - __clz(k - 1)) - 5);
                if (a.dense_row)
                    drow = __ldg(a.dense_row + term);
            } else if (term < 0) {
                atomicOr(a.status, kStatusBadWord);
            }
            a.word_rec[w] = make_int4(__float_as_int(seed), drow, dr, 0);
        }
        if (!known) {  // no postings
            for (int t = e0 + tid; t < e1; t += kPlanThreads)
                out[t] = 0;
            continue;
        }
        const long long s = __ldg(a.indptr + term), e = __ldg(a.indptr + term + 1);
        const int r = a.dir_row ? __ldg(a.dir_row + term) : -1;
        if (r >= 0) {  // the directory row, made absolute
            const int *src = a.dir + (long long)r * a.dir_stride;
            for (int t = e0 + tid; t < e1; t += kPlanThreads)
                out[t] = (int)s + __ldg(src + t);
            continue;
        }
        if (warp < 2) {
            const long long target = (long long)(warp == 0 ? e0 : e1) * a.tile_docs;
            const long long p = WarpLowerBoundGlobal(a.indices, s, e, target, lane);
            if (lane == 0)
                lim[warp] = (int)(p - s);
        }
        for (int i = tid; i < kPlanRowChunk; i += kPlanThreads)
            ent[i] = INT_MAX;
        __syncthreads();
        const int b = lim[0], en = lim[1];
        for (int i = b + tid; i < en; i += kPlanThreads) {
            const int t = __ldg(a.indices + s + i) / a.tile_docs;
            const int tp = i > 0 ? __ldg(a.indices + s + i - 1) / a.tile_docs : -1;
            if (tp != t)
                ent[t - e0] = i;  // the tile's first posting; t is in [e0, e1)
        }
        __syncthreads();
        // suffix minimum over the chunk, ending in en
        int v[kPer];
        int m = INT_MAX;
#pragma unroll
        for (int u = kPer - 1; u >= 0; --u) {
            m = min(m, ent[tid * kPer + u]);
            v[u] = m;
        }
        int x = m;  // suffix minimum of the thread aggregates within the warp
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_down_sync(kFull, x, o);
            if (lane + o < 32)
                x = min(x, y);
        }
        if (lane == 0)
            wmin[warp] = x;
        __syncthreads();
        int carry = en;
        for (int j = warp + 1; j < kPlanThreads / 32; ++j)
            carry = min(carry, wmin[j]);
        const int after = __shfl_down_sync(kFull, x, 1);
        if (lane < 31)
            carry = min(carry, after);
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            const int t = e0 + tid * kPer + u;
            if (t < e1)
                out[t] = (int)s + min(v[u], carry);
        }
        __syncthreads();  // ent, lim and wmin are rewritten for the next word
    }
    // launched overlapped after the plan kernel (a pruned or batched Search): complete only after it,
    // so that every later kernel sees that plan too
    WaitPrerequisites();
}

// Grid of PlanRowsKernel for a batch capacity of `words` query words.
inline dim3 PlanRowsGrid(long long words, int tiles, int sms)
{
    const int chunks = (tiles + 1 + kPlanRowChunk - 1) / kPlanRowChunk;
    const long long x = std::max<long long>(1, std::min<long long>(words, std::max(1, sms * 4 / chunks)));
    return dim3((unsigned)x, (unsigned)chunks);
}

} // namespace bm25k
