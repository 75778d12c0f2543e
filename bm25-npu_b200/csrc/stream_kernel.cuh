// Persistent, warp-specialised BM25 Search kernels for sm_100a (the default path).
//
// Contract of the reference's fused scoring + merge operators
//   feature_retrieval/src/ascendfaiss/ops/ascendc/bm25/fused/op_kernel/bm25_fused_score_top_k.cpp:637-936
//   feature_retrieval/src/ascendfaiss/ops/ascendc/bm25/merge/op_kernel/bm25_top_k_merge.cpp:10-98
// (exact per-query top-K, score desc / id asc, zero-score fill by id), organised
// for a B200 as three launches:
//
// PlanKernel -- resolves every query word's posting sub-range in every tile
//   (per-tile directory rows for long lists; one pass over the postings for
//   short lists), written as absolute [b, e) pairs to plan[word][tile].
//
// StreamSearchKernel -- persistent: each CTA has one producer warp and eight
//   consumer warps.  Tasks are (query, tile) pairs in tile-major order, so every
//   query has tiles in the first wave and gets a score threshold early.
//   * The producer takes kTaskBatch tasks per work-counter atomic, reads their
//     plan entries and the queries' running thresholds lane-parallel, skips
//     tasks without postings, and streams the postings of the others -- doc ids
//     and FP32 scores -- as chunks of up to kChunk postings into a shared-memory
//     ring with 1-D bulk async copies (cp.async.bulk ... mbarrier::complete_tx,
//     no multicast), up to `stages` chunks ahead, across task boundaries.
//   * Consumer warp w owns documents [w * R, (w + 1) * R) of the tile
//     (R = tile_docs / 8).  It waits on each ring stage itself, finds its slice
//     of the chunk (one term's postings, sorted by document) with a
//     warp-parallel lower_bound, adds it into its own part of the shared-memory
//     tile row and releases the stage.  Only warp w touches a document of its
//     region and it consumes the ring in order, so each document's FP32 sum is
//     built in query-term order with no CTA barrier at all.
//   * At the end of a task each warp keeps its region's top-K among scores at
//     or above max(query threshold, a lower bound on the region's K-th score
//     from its lanes' maxima), appends them to the query's candidate buffer,
//     publishes its region's K-th score as the query's new threshold (K region
//     documents reach it, so the global K-th does too) and clears its region.
//     A global top-K document is in the top-K of every subset that contains
//     it, so every filter keeps it.
//
// FinalSelectKernel -- one CTA per query ranks the query's candidates exactly,
//   adds the zero-score fill, writes the K results and resets the query's
//   buffer and threshold for the next Search.
//
// Every wait in the streaming kernel is on an mbarrier and bounded by a clock
// budget; on expiry the kernel records kStatusTimeout, drains its own copies
// (bounded) and returns.
#pragma once
#include "tile_kernels.cuh"

#include <algorithm>
#include <climits>
#include <cuda_fp16.h>

namespace bm25k {

constexpr int kConsumerWarps = 8;
constexpr int kConsumerThreads = kConsumerWarps * 32;
constexpr int kStreamThreads = kConsumerThreads + 32;  // + one producer warp
constexpr int kChunk = 2048;                           // postings per ring stage
constexpr int kMaxStages = 8;
constexpr int kTaskBatch = 8;                          // tasks per work-counter atomic
constexpr int kPlanCache = 4;                          // plan entries a producer lane keeps in registers
constexpr int kWarpSurvCap = 64;                       // region candidates ranked exactly per warp
constexpr int kFinalThreads = 256;
constexpr int kSurvCap = 512;                          // candidates ranked exactly per query
constexpr long long kWaitBudget = 4000000000LL;        // cycles (~2 s) before a wait gives up
constexpr int kPlanThreads = 256;

enum : uint32_t {
    kStatusTimeout = 16u,       // a bounded wait gave up
    kStatusCandOverflow = 32u,  // a query's candidate buffer was too small
};

// Search counters (StreamArgs::stats): tile-group claims, tiles and postings copied into the
// rings; block path: tiles scored, 128-document blocks kept, postings read.
enum : int {
    kStatClaims = 0,
    kStatTilesScanned = 1,
    kStatPostingsCopied = 2,
    kStatItems = 3,
    kStatBlocksKept = 4,
    kStatPostingsRead = 5,
    kStatRouted = 6,
    kStats = 7,
};

enum : int {
    kFirstOfTask = 1,
    kLastOfTask = 4,
    kStop = 8,
};

struct StreamCtrl {
    unsigned next;  // next task to hand out
    unsigned done;  // producers that found no more tasks
};

struct PlanEntry {
    long long b, e;
};

struct StreamArgs {
    const long long *indptr;
    const int *indices;
    const float *data;
    const int *dir_row;
    const int *dir;
    long long dir_stride;
    const long long *qoffsets;
    const int *words;
    int vocab, num_docs, tile_docs, tiles, k, q;
    long long word_cap;     // rows of `plan`; query words beyond it are rejected
    PlanEntry *plan;        // [word][tile]
    unsigned *threshold;    // [Q] running K-th score bits (0 = none yet)
    unsigned *tslots;       // [Q][32] slot g: best tile maximum among tiles with tile % k == g
    unsigned *cand_count;   // [Q] candidates appended
    float *cand_scores;     // [Q][cand_cap]
    int *cand_ids;          // [Q][cand_cap]
    long long cand_cap;
    StreamCtrl *ctrl;
    int stages;
    int chunk;              // postings per ring stage (tile-group kernel)
    float *out_scores;
    int *out_ids;
    unsigned *status;
    // pruned Search (block kernels): nullptr on the plain path
    const unsigned short *boff;  // [dir row][tile][block] posting offset of the block from the tile's start
    // [dir row][tile][block] largest posting score of the row's term in the block, rounded up to FP16
    // (a larger value is still a bound: rounded FP32 addition is monotone)
    const __half *bmax;
    const float *tau;            // [Q] starting bound guesses
    const float *safe;           // [Q] safe bounds (learned Searches; a retry's bound), or nullptr
    int *exact;                  // [Q] 1 where K candidates reached tau
    uint4 *items;                // (query | kept-block mask << 16, tile, first word, words) per tile to score
    int *wrow;                   // [word] directory row of the word's term, -1 none, -2 not a valid term
    unsigned *item_count;        // items listed (first pass at [0], retry pass at [2]; reset by PlanKernel)
    long long item_cap;
    // routing: a query keeping more than route_limit blocks is streamed by the tile-group kernel
    // instead (route_limit 0: never); qkept [Q] counts its kept blocks, route_list its queries
    unsigned *qkept;
    unsigned route_limit;
    int *route_list;
    unsigned *route_count;
    // retry passes: a pass appends to fail_out the queries it could not answer (a pruned pass that
    // fell short of K, a K > 32 candidate buffer that overflowed); a retry pass (retry != 0)
    // searches the queries of fail_in on the plain path.  Counts are reset before the Search.
    const int *fail_in;
    const unsigned *fail_in_count;
    int *fail_out;
    unsigned *fail_out_count;
    int retry;
    unsigned long long *stats;   // [kStats] counters, accumulated (nullptr: not kept)
    // a batch with a K per query (tile-group kernel): nullptr when every query takes a.k
    const int *kq;               // [Q] K of each query (a.k is their maximum)
    const long long *kout;       // [Q] first output slot of each query (packed rows)
    // warp-tile kernel, both written by PlanRowsKernel for every query word w of the Search:
    // plan_rows [word][tiles + 1] the position in the posting arrays of the word's first posting in
    // each tile (tiles + 1: the list's end), so a claim reads its bounds with one load per tile bound;
    // word_rec [word] (starting-bound seed as float bits, dense row or -1, directory row: -1 a
    // short list, -2 not a term, 0).  prefetch != 0: each claim's posting runs are prefetched into
    // L2 when the claim is taken.  rows_plan != 0: the block path (BlockBoundKernel, BlockTileKernel)
    // takes a word's range in a tile from its plan row and its directory row from its record, and
    // PlanKernel does not run (a warp-tile session's pruned Search)
    int *plan_rows;
    int4 *word_rec;
    int rows_plan;
    int prefetch;
    // [vocab][32] each term's 32 largest posting scores (descending, 0 past its document
    // frequency): the warp-tile kernel starts a K <= 32 query's running bound at the largest K-th
    // score of its words, which K documents reach (nullptr: start at 0)
    const float *term_top;
    const float *term_rank;  // [vocab][5] scores at ranks 64 .. 1024: starting bounds for K in 33 .. 1024
    // [dense row][dense_stride] per-document scores of the terms kept dense (0 where absent);
    // dense_row [vocab]: a term's dense row or -1
    const float *dense;
    const int *dense_row;
    long long dense_stride;
    // warp-tile kernel: claims of kC tiles cover tile blocks [0, wt_bulk); the tiles after them
    // are claimed one at a time, so the last claims of the launch are short
    int wt_bulk;
    // cycles a bounded wait spends before it gives up (0: kWaitBudget)
    long long wait_budget;
    // test hook: a nonzero word makes the tile-group kernel's producer issue no ring stage, so its
    // consumers' bounded waits run out (nullptr: none)
    const unsigned *inject;
};

// The wait budget of a launch.
__device__ __forceinline__ long long WaitBudget(const StreamArgs &a)
{
    return a.wait_budget > 0 ? a.wait_budget : kWaitBudget;
}

// K of query q, and the first output slot of its row.
__device__ __forceinline__ int QueryK(const StreamArgs &a, int q)
{
    return a.kq ? min(max(__ldg(a.kq + q), 1), a.k) : a.k;
}
__device__ __forceinline__ long long OutRow(const StreamArgs &a, int q)
{
    return a.kout ? __ldg(a.kout + q) : (long long)q * a.k;
}

struct __align__(16) StageMeta {
    long long base;  // posting position of ring element 0
    int lo, hi;      // valid ring elements [lo, hi) of the current term
    int count;       // elements copied (multiple of 4)
    int flags;
    int q, tile;
    float thr;       // the query's running threshold when the task was fetched
};

struct StreamShared {
    unsigned long long full[kMaxStages];
    unsigned long long empty[kMaxStages];
    StageMeta meta[kMaxStages];
    float wbuf_s[kConsumerWarps][kWarpSurvCap];
    int wbuf_i[kConsumerWarps][kWarpSurvCap];
    float wsel_s[kConsumerWarps][32];
    int wsel_i[kConsumerWarps][32];
    unsigned bad;
    int abort;
};

// ---- PTX wrappers ----------------------------------------------------------

__device__ __forceinline__ unsigned SmemAddr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void MbarInit(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void MbarArriveExpectTx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(SmemAddr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void MbarArrive(unsigned long long *bar)
{
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(SmemAddr(bar)) : "memory");
}

__device__ __forceinline__ bool MbarTryWait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(SmemAddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// try_wait that may suspend the thread (up to ~20 us) until the phase completes,
// so a waiting warp does not spin through issue slots.
__device__ __forceinline__ bool MbarTryWaitSuspend(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2, %3;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(SmemAddr(bar)), "r"(parity), "r"(20000u)
        : "memory");
    return ok != 0;
}

// Bounded wait; false when the budget ran out or another role aborted.
__device__ __forceinline__ bool MbarWait(unsigned long long *bar, unsigned parity, volatile int *abort,
                                         long long budget = kWaitBudget)
{
    if (MbarTryWait(bar, parity))
        return true;
    const long long t0 = clock64();
    for (;;) {
        if (MbarTryWaitSuspend(bar, parity))
            return true;
        if (*abort)
            return false;
        if (clock64() - t0 > budget) {
            *abort = 1;
            return false;
        }
    }
}

// Whole-warp bounded wait: lane 0 waits, then every lane acquires the completed phase.
__device__ __forceinline__ bool WarpWait(unsigned long long *bar, unsigned parity, volatile int *abort, int lane,
                                         long long budget = kWaitBudget)
{
    int ok = 1;
    if (lane == 0)
        ok = MbarWait(bar, parity, abort, budget) ? 1 : 0;
    ok = __shfl_sync(kFull, ok, 0);
    if (ok)
        (void)MbarTryWait(bar, parity);  // complete already: returns at once, acquiring for this lane
    return ok != 0;
}

// Whole-warp bounded wait with every lane on the barrier (no divergent branch);
// the outcome is agreed by vote, so all lanes return the same.
__device__ __forceinline__ bool WarpWaitAll(unsigned long long *bar, unsigned parity, volatile int *abort,
                                            long long budget = kWaitBudget)
{
    bool ok = MbarTryWait(bar, parity);
    if (!__all_sync(kFull, ok)) {
        const long long t0 = clock64();
        while (!ok) {
            ok = MbarTryWaitSuspend(bar, parity);
            if (!ok && (*abort || clock64() - t0 > budget)) {
                *abort = 1;
                break;
            }
        }
        ok = __all_sync(kFull, ok);
    }
    return ok;
}

// 1-D bulk copy global -> shared, completion counted on `bar` (no multicast).
__device__ __forceinline__ void BulkLoad(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     SmemAddr(dst)),
                 "l"(src), "r"(bytes), "r"(SmemAddr(bar))
                 : "memory");
}

// ---- warp top-K with the K-th entry cached in registers (tie fallbacks) --------

// Lane l holds the l-th best (score, id) seen by the warp (l < k <= 32), best
// first; empty slots hold (-1, kNoId).  (ts, ti) caches lane k-1's entry so an
// offer that inserts nothing costs one compare and one ballot.
struct WarpTopK {
    float ls, ts;
    int li, ti;
    __device__ __forceinline__ void Reset()
    {
        ls = ts = -1.0f;
        li = ti = kNoId;
    }
    __device__ __forceinline__ void Offer(float cs, int ci, bool has, int k, int lane)
    {
        unsigned pending = __ballot_sync(kFull, has && Better(cs, ci, ts, ti));
        while (pending) {
            const int src = __ffs(pending) - 1;
            pending &= pending - 1;
            const float s = __shfl_sync(kFull, cs, src);
            const int id = __shfl_sync(kFull, ci, src);
            if (Better(s, id, ts, ti)) {  // uniform
                const bool above = lane < k && Better(ls, li, s, id);
                const int pos = __popc(__ballot_sync(kFull, above));
                const float us = __shfl_up_sync(kFull, ls, 1);
                const int ui = __shfl_up_sync(kFull, li, 1);
                if (lane < k && lane > pos) {
                    ls = us;
                    li = ui;
                }
                if (lane == pos) {
                    ls = s;
                    li = id;
                }
                ts = __shfl_sync(kFull, ls, k - 1);
                ti = __shfl_sync(kFull, li, k - 1);
            }
        }
    }
};

// ---- per-warp region selection ---------------------------------------------------

// Descending bitonic sort across the warp; returns this lane's element.
__device__ __forceinline__ float WarpSortDesc(float v, int lane)
{
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const float o = __shfl_xor_sync(kFull, v, stride);
            const bool desc = (lane & size) == 0;
            const bool lower = (lane & stride) == 0;
            v = (lower == desc) ? fmaxf(v, o) : fminf(v, o);
        }
    }
    return v;
}

// Warp w's candidates of the task: its region's top-k among scores >= thr
// (and > 0), sorted best first into wsel[w] with global ids.  Returns their
// number; *kth receives the region's k-th score when it is known exactly
// (k candidates, none filtered below it), else 0.
__device__ __forceinline__ int WarpRegionSelect(StreamShared &sh, const float *region, int region_docs, float thr,
                                                int k, int base_id, int lane, int warp, float *kth)
{
    const float4 *reg4 = reinterpret_cast<const float4 *>(region);
    const int r4 = region_docs / 4;  // multiple of 32: warp-uniform trip counts
    float tmax = 0.0f;
    int pass = 0;
    for (int i = lane; i < r4; i += 32) {
        const float4 x = reg4[i];
        tmax = fmaxf(tmax, fmaxf(fmaxf(x.x, x.y), fmaxf(x.z, x.w)));
        pass += (x.x >= thr && x.x > 0.0f) + (x.y >= thr && x.y > 0.0f) + (x.z >= thr && x.z > 0.0f) +
                (x.w >= thr && x.w > 0.0f);
    }
    int total = __reduce_add_sync(kFull, pass);
    *kth = 0.0f;
    if (total == 0)
        return 0;
    float tau = thr;
    if (total > k) {
        // k-th largest lane maximum: k lanes each hold a score >= it
        const float bound = __shfl_sync(kFull, WarpSortDesc(tmax, lane), k - 1);
        if (bound > tau) {
            tau = bound;
            pass = 0;
            for (int i = lane; i < r4; i += 32) {
                const float4 x = reg4[i];
                pass += (x.x >= tau && x.x > 0.0f) + (x.y >= tau && x.y > 0.0f) + (x.z >= tau && x.z > 0.0f) +
                        (x.w >= tau && x.w > 0.0f);
            }
            total = __reduce_add_sync(kFull, pass);
        }
    }
    int n = 0;
    if (total <= kWarpSurvCap) {
        // each lane writes its survivors at its exclusive prefix offset
        int at = pass;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(kFull, at, o);
            if (lane >= o)
                at += v;
        }
        at -= pass;
        if (pass) {
            for (int i = lane; i < r4; i += 32) {
                const float4 x = reg4[i];
                const float xs[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    if (xs[c] >= tau && xs[c] > 0.0f) {
                        sh.wbuf_s[warp][at] = xs[c];
                        sh.wbuf_i[warp][at] = base_id + 4 * i + c;
                        ++at;
                    }
            }
        }
        __syncwarp();
        for (int i = lane; i < total; i += 32) {
            const float s = sh.wbuf_s[warp][i];
            const int id = sh.wbuf_i[warp][i];
            int rank = 0;
            for (int t = 0; t < total; ++t)
                rank += Better(sh.wbuf_s[warp][t], sh.wbuf_i[warp][t], s, id);
            if (rank < k) {
                sh.wsel_s[warp][rank] = s;
                sh.wsel_i[warp][rank] = id;
            }
        }
        n = min(total, k);
    } else {
        // ties at the top overflow the buffer: insertion select over the region
        WarpTopK top;
        top.Reset();
        for (int i = lane; i < r4; i += 32) {
            const float4 x = reg4[i];
            const int id0 = base_id + 4 * i;
            top.Offer(x.x, id0 + 0, x.x > 0.0f && x.x >= tau, k, lane);
            top.Offer(x.y, id0 + 1, x.y > 0.0f && x.y >= tau, k, lane);
            top.Offer(x.z, id0 + 2, x.z > 0.0f && x.z >= tau, k, lane);
            top.Offer(x.w, id0 + 3, x.w > 0.0f && x.w >= tau, k, lane);
        }
        n = __popc(__ballot_sync(kFull, lane < k && top.li != kNoId));
        if (lane < n) {
            sh.wsel_s[warp][lane] = top.ls;
            sh.wsel_i[warp][lane] = top.li;
        }
    }
    __syncwarp();
    if (n == k)
        *kth = sh.wsel_s[warp][k - 1];
    return n;
}

// ---- plan kernel -------------------------------------------------------------

__device__ __forceinline__ long long LowerBoundGlobal(const int *ids, long long lo, long long hi, long long target)
{
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if ((long long)__ldg(ids + mid) < target)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

constexpr int kPlanTileChunk = 2048;  // tiles per plan CTA (grid.y)
constexpr int kPlanScanAll = 16384;   // lists up to this length are scanned whole

// First position in ids[lo, hi) (ascending) whose value is >= target; all 32 lanes
// of a warp, each step probing 32 evenly spaced positions.
__device__ __forceinline__ long long WarpLowerBoundGlobal(const int *ids, long long lo, long long hi,
                                                          long long target, int lane)
{
    while (hi - lo > 32) {
        const long long step = (hi - lo + 31) >> 5;
        const long long p = lo + lane * step;
        const bool less = p < hi && (long long)__ldg(ids + p) < target;
        const int c = __popc(__ballot_sync(kFull, less));
        if (c == 0)
            return lo;
        const long long nlo = lo + (long long)(c - 1) * step + 1;
        hi = min(hi, lo + (long long)c * step);
        lo = nlo;
    }
    const bool less = lo + lane < hi && (long long)__ldg(ids + lo + lane) < target;
    return lo + __popc(__ballot_sync(kFull, less));
}

// plan[w][tile] = absolute posting range of query word w inside tile (empty for
// unknown or negative words).  CTA (x, y) covers tiles [y * kPlanTileChunk,
// (y + 1) * kPlanTileChunk) of words x, x + gridDim.x, ...  A word with a
// directory row copies its per-tile offsets; any other word (a short list, or
// no directory at all: a.dir_row == nullptr) marks every tile empty and then
// lets each run of postings that falls in one tile write its own bounds:
// O(tiles + df) coalesced work per word.
__global__ void __launch_bounds__(kPlanThreads) PlanKernel(const StreamArgs a)
{
    __shared__ long long range[2];
    AllowDependents();  // the tile-group kernel sets up its shared memory meanwhile
    if (a.item_count && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x < 4)
        a.item_count[threadIdx.x] = 0u;  // the block path's work lists of this Search start empty
    long long total = a.qoffsets[a.q];
    if (total < 0 || total > a.word_cap) {
        if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0)
            atomicOr(a.status, kStatusBadQuery);
        total = total < 0 ? 0 : a.word_cap;
    }
    const int t0 = (int)blockIdx.y * kPlanTileChunk;
    const int t1 = min(a.tiles, t0 + kPlanTileChunk);
    if (t0 >= t1) {
        WaitPrerequisites();  // completes only after the kernel before it (the learned bounds)
        return;
    }
    const int tid = threadIdx.x;
    for (long long w = blockIdx.x; w < total; w += gridDim.x) {
        const int term = a.words[w];
        PlanEntry *out = a.plan + w * a.tiles;
        if (a.wrow && blockIdx.y == 0 && tid == 0)
            a.wrow[w] = term < 0 || term >= a.vocab ? -2 : (a.dir_row ? a.dir_row[term] : -1);
        if (term < 0 || term >= a.vocab) {
            if (term < 0 && tid == 0 && blockIdx.y == 0)
                atomicOr(a.status, kStatusBadWord);
            for (int t = t0 + tid; t < t1; t += kPlanThreads)
                out[t] = PlanEntry{0, 0};
            continue;
        }
        const long long s = a.indptr[term], e = a.indptr[term + 1];
        const int r = a.dir_row ? a.dir_row[term] : -1;
        if (r >= 0) {
            // the chunk's tiles, kPlanTileChunk / kPlanThreads per thread, every directory load
            // issued before the stores (which could otherwise alias them and serialise the loop)
            const int *__restrict__ d = a.dir + (long long)r * a.dir_stride;
            constexpr int kU = kPlanTileChunk / kPlanThreads;
            static_assert(kPlanTileChunk % kPlanThreads == 0, "whole rounds of tiles per plan CTA");
            int lo[kU], hi[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int t = t0 + tid + u * kPlanThreads;
                lo[u] = hi[u] = 0;
                if (t < t1) {
                    lo[u] = __ldg(d + t);
                    hi[u] = __ldg(d + t + 1);
                }
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int t = t0 + tid + u * kPlanThreads;
                if (t < t1)
                    out[t] = PlanEntry{s + lo[u], s + hi[u]};
            }
            continue;
        }
        for (int t = t0 + tid; t < t1; t += kPlanThreads)
            out[t] = PlanEntry{0, 0};
        if (tid < 32) {
            // lists up to kPlanScanAll postings are scanned whole by every CTA of the word; a
            // longer one (a list left out of the directory by its byte budget) is first cut to
            // this CTA's documents with a 32-way search: a few dependent loads, not ~log2(df)
            long long b = s, en = e;
            if (gridDim.y > 1 && e - s > kPlanScanAll) {
                b = WarpLowerBoundGlobal(a.indices, s, e, (long long)t0 * a.tile_docs, tid);
                en = WarpLowerBoundGlobal(a.indices, b, e, (long long)t1 * a.tile_docs, tid);
            }
            if (tid == 0) {
                range[0] = b;
                range[1] = en;
            }
        }
        __syncthreads();  // the empty marks land before the bounds; range is published
        const long long b = range[0], en = range[1];
        // sixteen postings per thread per round (a list of 4096 in one), their loads issued
        // before any store (the stores could otherwise alias the loads and serialise them)
        const int *__restrict__ ids = a.indices;
        constexpr int kU = 16;
        for (long long i0 = b + tid; i0 < en; i0 += kPlanThreads * kU) {
            int cur[kU], prv[kU], nxt[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const long long i = i0 + (long long)u * kPlanThreads;
                cur[u] = prv[u] = nxt[u] = -1;
                if (i < en) {
                    cur[u] = __ldg(ids + i);
                    prv[u] = i == s ? -1 : __ldg(ids + i - 1);
                    nxt[u] = i == e - 1 ? -1 : __ldg(ids + i + 1);
                }
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const long long i = i0 + (long long)u * kPlanThreads;
                if (i >= en)
                    continue;
                const int t = cur[u] / a.tile_docs;
                if (t < t0 || t >= t1)
                    continue;
                if (prv[u] < 0 || prv[u] / a.tile_docs != t)
                    out[t].b = i;
                if (nxt[u] < 0 || nxt[u] / a.tile_docs != t)
                    out[t].e = i + 1;
            }
        }
        __syncthreads();  // range[] is rewritten for the next word
    }
    // launched overlapped after the learned bounds: complete only after them, so that every
    // kernel waiting for this one sees the bounds too
    WaitPrerequisites();
}

// Grid of PlanKernel for a batch capacity of `words` query words.
inline dim3 PlanGrid(long long words, int tiles, int sms)
{
    const int chunks = (tiles + kPlanTileChunk - 1) / kPlanTileChunk;
    const long long x = std::max<long long>(1, std::min<long long>(words, std::max(1, sms * 8 / chunks)));
    return dim3((unsigned)x, (unsigned)chunks);
}

// ---- the streaming kernel -------------------------------------------------------

// First index in ids[a, b) (ascending) whose value is >= target; all lanes.
__device__ __forceinline__ int WarpLowerBound(const int *ids, int a, int b, long long target, int lane)
{
    while (b - a > 32) {
        const int step = (b - a + 31) >> 5;
        const int p = a + lane * step;
        const bool less = p < b && (long long)ids[p] < target;
        const int c = __popc(__ballot_sync(kFull, less));
        if (c == 0)
            return a;
        const int na = a + (c - 1) * step + 1;
        b = min(b, a + c * step);
        a = na;
    }
    const bool less = a + lane < b && (long long)ids[a + lane] < target;
    return a + __popc(__ballot_sync(kFull, less));
}

__global__ void __launch_bounds__(kStreamThreads, 1) StreamSearchKernel(const StreamArgs a)
{
    extern __shared__ __align__(128) unsigned char stream_smem[];
    float *row = reinterpret_cast<float *>(stream_smem);
    int *ring_ids = reinterpret_cast<int *>(stream_smem + (size_t)a.tile_docs * 4);
    float *ring_vals = reinterpret_cast<float *>(ring_ids + (size_t)a.stages * kChunk);
    StreamShared &sh = *reinterpret_cast<StreamShared *>(ring_vals + (size_t)a.stages * kChunk);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) {
        for (int i = 0; i < a.stages; ++i) {
            MbarInit(&sh.full[i], 1);
            MbarInit(&sh.empty[i], kConsumerWarps);
        }
        sh.bad = 0;
        sh.abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    {
        float4 *row4 = reinterpret_cast<float4 *>(row);
        for (int i = tid; i < a.tile_docs / 4; i += kStreamThreads)
            row4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    volatile int *abort = &sh.abort;
    const unsigned total = (unsigned)a.q * (unsigned)a.tiles;

    if (warp == kConsumerWarps) {
        // ================= producer warp =================
        unsigned long long g = 0;  // ring entries issued
        unsigned bad = 0;
        bool dead = false;

        // Claims the next ring stage (lane 0 waits, the warp learns the outcome).
        auto claim = [&](int &st) -> bool {
            st = (int)(g % (unsigned long long)a.stages);
            const unsigned long long k = g / (unsigned long long)a.stages;
            int ok = 1;
            if (k > 0 && lane == 0)
                ok = MbarWait(&sh.empty[st], (unsigned)((k - 1) & 1), abort, WaitBudget(a)) ? 1 : 0;
            return __shfl_sync(kFull, ok, 0) != 0;
        };

        while (!dead) {
            unsigned base = 0;
            if (lane == 0)
                base = atomicAdd(&a.ctrl->next, (unsigned)kTaskBatch);
            base = __shfl_sync(kFull, base, 0);
            if (base >= total)
                break;
            const unsigned task = base + lane;
            const bool valid = lane < kTaskBatch && task < total;
            int q = 0, tile = 0, nt = 0, last = -1;
            long long qb = 0;
            float thr = 0.0f;
            PlanEntry pc[kPlanCache];
#pragma unroll
            for (int s = 0; s < kPlanCache; ++s)
                pc[s] = PlanEntry{0, 0};
            if (valid) {
                tile = (int)(task / (unsigned)a.q);
                q = (int)(task % (unsigned)a.q);
                thr = __uint_as_float(__ldcg(a.threshold + q));
                qb = a.qoffsets[q];
                long long n = a.qoffsets[q + 1] - qb;
                if (n < 0 || n > kMaxTerms || qb < 0 || qb + n > a.word_cap) {
                    bad |= kStatusBadQuery;
                    n = 0;
                }
                nt = (int)n;
#pragma unroll
                for (int s = 0; s < kPlanCache; ++s)
                    if (s < nt)
                        pc[s] = a.plan[(qb + s) * a.tiles + tile];
#pragma unroll
                for (int s = 0; s < kPlanCache; ++s)
                    if (s < nt && pc[s].e > pc[s].b)
                        last = s;
                for (int s = kPlanCache; s < nt; ++s) {
                    const PlanEntry pe = a.plan[(qb + s) * a.tiles + tile];
                    if (pe.e > pe.b)
                        last = s;
                }
            }
            // tasks without postings contribute nothing: skip them
            unsigned work = __ballot_sync(kFull, valid && last >= 0);
            while (work && !dead) {
                const int src = __ffs(work) - 1;
                work &= work - 1;
                const int tq = __shfl_sync(kFull, q, src);
                const int ttile = __shfl_sync(kFull, tile, src);
                const long long tqb = __shfl_sync(kFull, qb, src);
                const int tlast = __shfl_sync(kFull, last, src);
                const float tthr = __shfl_sync(kFull, thr, src);
                bool first = true;
                for (int slot = 0; slot <= tlast && !dead; ++slot) {
                    long long b, e;
                    if (slot < kPlanCache) {
                        long long mb = 0, me = 0;
#pragma unroll
                        for (int s = 0; s < kPlanCache; ++s)
                            if (s == slot) {
                                mb = pc[s].b;
                                me = pc[s].e;
                            }
                        b = __shfl_sync(kFull, mb, src);
                        e = __shfl_sync(kFull, me, src);
                    } else {
                        const PlanEntry pe = a.plan[(tqb + slot) * a.tiles + ttile];
                        b = pe.b;
                        e = pe.e;
                    }
                    if (b >= e)
                        continue;
                    const long long a0 = b & ~3LL, a1 = (e + 3) & ~3LL;
                    for (long long c0 = a0; c0 < a1;) {
                        const long long c1 = min(c0 + (long long)kChunk, a1);
                        int st;
                        if (!claim(st)) {
                            dead = true;
                            break;
                        }
                        if (lane == 0) {
                            StageMeta &m = sh.meta[st];
                            m.base = c0;
                            m.count = (int)(c1 - c0);
                            m.lo = (int)max(0LL, b - c0);
                            m.hi = (int)min((long long)m.count, e - c0);
                            m.flags = (first ? kFirstOfTask : 0) | (slot == tlast && c1 == a1 ? kLastOfTask : 0);
                            m.q = tq;
                            m.tile = ttile;
                            m.thr = tthr;
                            const unsigned bytes = (unsigned)(c1 - c0) * 4u;
                            MbarArriveExpectTx(&sh.full[st], 2u * bytes);
                            BulkLoad(ring_ids + (size_t)st * kChunk, a.indices + c0, bytes, &sh.full[st]);
                            BulkLoad(ring_vals + (size_t)st * kChunk, a.data + c0, bytes, &sh.full[st]);
                        }
                        __syncwarp();
                        first = false;
                        ++g;
                        c0 = c1;
                    }
                }
            }
        }
        if (!dead) {
            int st;
            if (claim(st)) {
                if (lane == 0) {
                    StageMeta &m = sh.meta[st];
                    m.base = 0;
                    m.lo = m.hi = m.count = 0;
                    m.flags = kStop;
                    m.q = m.tile = 0;
                    m.thr = 0.0f;
                    MbarArrive(&sh.full[st]);
                }
                __syncwarp();
                ++g;
            } else {
                dead = true;
            }
        }
        if (lane == 0) {
            if (bad)
                atomicOr(a.status, bad);
            // the last producer to run dry resets the work counter for the next Search
            const unsigned d = atomicAdd(&a.ctrl->done, 1u);
            if (d == gridDim.x - 1) {
                a.ctrl->next = 0u;
                a.ctrl->done = 0u;
            }
        }
        if (dead && lane == 0) {
            // drain copies still in flight into this CTA's ring (bounded)
            for (unsigned long long h = (g > (unsigned long long)a.stages ? g - a.stages : 0); h < g; ++h) {
                const int st = (int)(h % (unsigned long long)a.stages);
                const long long t0 = clock64();
                while (!MbarTryWait(&sh.full[st], (unsigned)((h / a.stages) & 1)) && clock64() - t0 < WaitBudget(a)) {
                }
            }
        }
        return;
    }

    // ================= consumer warps (independent) =================
    const int region_docs = a.tile_docs / kConsumerWarps;
    float *region = row + warp * region_docs;
    unsigned long long g = 0;
    unsigned bad = 0;
    int q = 0, tile = 0;
    float thr = 0.0f;
    for (;;) {
        const int st = (int)(g % (unsigned long long)a.stages);
        const unsigned parity = (unsigned)((g / (unsigned long long)a.stages) & 1);
        if (!WarpWait(&sh.full[st], parity, abort, lane, WaitBudget(a)))
            break;
        const StageMeta m = sh.meta[st];
        if (m.flags & kStop)
            break;
        if (m.flags & kFirstOfTask) {
            q = m.q;
            tile = m.tile;
            thr = m.thr;
        }
        // this warp's slice of the chunk: postings of documents in its region
        const long long lo = (long long)tile * a.tile_docs;
        const long long dlo = lo + (long long)warp * region_docs, dhi = dlo + region_docs;
        const int *ids = ring_ids + (size_t)st * kChunk;
        const float *vals = ring_vals + (size_t)st * kChunk;
        if (m.hi > m.lo && (long long)ids[m.hi - 1] >= dlo && (long long)ids[m.lo] < dhi) {
            const int s0 = WarpLowerBound(ids, m.lo, m.hi, dlo, lane);
            const int s1 = WarpLowerBound(ids, s0, m.hi, dhi, lane);
#pragma unroll 4
            for (int i = s0 + lane; i < s1; i += 32) {
                const long long d = (long long)ids[i] - lo;
                const float sum = row[d] + vals[i];
                row[d] = sum;
                if (!(sum <= FLT_MAX))
                    bad |= kStatusOverflow;
            }
        }
        __syncwarp();
        if (lane == 0)
            MbarArrive(&sh.empty[st]);
        ++g;
        if (!(m.flags & kLastOfTask))
            continue;

        // ---- end of task: this warp's candidates, straight to the query's buffer ----
        float kth;
        const int n = WarpRegionSelect(sh, region, region_docs, thr, a.k, (int)dlo, lane, warp, &kth);
        if (n > 0) {
            unsigned at = 0;
            if (lane == 0) {
                at = atomicAdd(a.cand_count + q, (unsigned)n);
                if (kth > thr)
                    atomicMax(a.threshold + q, __float_as_uint(kth));
            }
            at = __shfl_sync(kFull, at, 0);
            if (lane < n) {
                if ((long long)at + lane < a.cand_cap) {
                    const long long off = (long long)q * a.cand_cap + at + lane;
                    a.cand_scores[off] = sh.wsel_s[warp][lane];
                    a.cand_ids[off] = sh.wsel_i[warp][lane];
                } else {
                    bad |= kStatusCandOverflow;
                }
            }
        }
        {
            float4 *reg4 = reinterpret_cast<float4 *>(region);
            for (int i = lane; i < region_docs / 4; i += 32)
                reg4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        __syncwarp();
    }
    bad = __reduce_or_sync(kFull, bad);
    if (lane == 0 && (bad || *abort))
        atomicOr(a.status, bad | (*abort ? kStatusTimeout : 0u));
}

// ---- final per-query selection ---------------------------------------------------

// Exact top-k of one query's candidates: bound from per-thread maxima (m warps
// with j threads each holding a score >= tau, j * m >= k), raised to the
// query's threshold; survivors ranked exactly (insertion select when ties
// overflow the buffer); zero-score fill; then the query's state is reset.
__global__ void __launch_bounds__(kFinalThreads) FinalSelectKernel(const StreamArgs a)
{
    constexpr int kWarps = kFinalThreads / 32;
    __shared__ float surv_s[kSurvCap];
    __shared__ int surv_i[kSurvCap];
    __shared__ float sel_s[32];
    __shared__ int sel_i[32];
    __shared__ float wl_s[kWarps][32];
    __shared__ int wl_i[kWarps][32];
    __shared__ float wv[kWarps];
    __shared__ unsigned surv_count;
    __shared__ int sel_count;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    AllowDependents();    // a retry pass may be placed meanwhile
    WaitPrerequisites();  // the candidates and bounds of the search kernel before it
    int q = blockIdx.x;
    if (a.retry) {  // block b answers the b-th query of the fail list
        if ((unsigned)q >= __ldcg(a.fail_in_count))
            return;
        q = __ldcg(a.fail_in + q);
    }
    const int k = QueryK(a, q);
    if (k > kMaxSmallK)
        return;  // FinalSelectLargeKernel's query
    const unsigned appended = __ldcg(a.cand_count + q);
    const int n = (int)min((long long)appended, a.cand_cap);
    if (tid == 0 && (long long)appended > a.cand_cap)
        atomicOr(a.status, kStatusCandOverflow);
    // floor: the query's threshold, or the least of the k group slots when higher (each slot is a
    // real document's score from its own group of tiles, so k documents reach the least one)
    float floor = __uint_as_float(__ldcg(a.threshold + q));
    {
        __shared__ unsigned slot_min;
        if (warp == 0) {
            const unsigned v = lane < k ? __ldcg(a.tslots + (long long)q * 32 + lane) : 0xffffffffu;
            const unsigned m = __reduce_min_sync(kFull, v);
            if (lane == 0)
                slot_min = m;
        }
        __syncthreads();
        floor = fmaxf(floor, __uint_as_float(slot_min));
    }
    const float *cs = a.cand_scores + (long long)q * a.cand_cap;
    const int *ci = a.cand_ids + (long long)q * a.cand_cap;
    // a row that starts on a 16-byte boundary is read 128 bits at a time, four loads in flight
    // per thread (the engine's rows all do: cand_cap is a multiple of 4); the rest one by one
    const float4 *cs4 = reinterpret_cast<const float4 *>(cs);
    const int n4 = (reinterpret_cast<uintptr_t>(cs) & 15u) == 0 ? n >> 2 : 0;

    auto keep = [&](float s, int i, float bound) {
        if (s > 0.0f && s >= bound) {
            const unsigned at = atomicAdd(&surv_count, 1u);
            if (at < (unsigned)kSurvCap) {
                surv_s[at] = s;
                surv_i[at] = __ldcg(ci + i);
            }
        }
    };
    auto filter = [&](float bound) {  // every candidate at or above bound joins the survivors
#pragma unroll 4
        for (int i = tid; i < n4; i += kFinalThreads) {
            const float4 v = __ldcg(cs4 + i);
            keep(v.x, 4 * i, bound);
            keep(v.y, 4 * i + 1, bound);
            keep(v.z, 4 * i + 2, bound);
            keep(v.w, 4 * i + 3, bound);
        }
        for (int i = 4 * n4 + tid; i < n; i += kFinalThreads)
            keep(__ldcg(cs + i), i, bound);
    };
    // One pass at the floor: each top-k document of the query is a candidate at or above it (its
    // tile appended its top-k above a lower bound than the floor).  Only when that leaves more
    // survivors than fit is a higher bound taken from the candidates themselves (below).
    if (tid == 0)
        surv_count = 0;
    __syncthreads();
    filter(floor);
    __syncthreads();
    float tau = floor;
    if (surv_count > (unsigned)kSurvCap) {
        float tmax = 0.0f;  // the largest of this thread's candidates: distinct threads, distinct documents
#pragma unroll 4
        for (int i = tid; i < n4; i += kFinalThreads) {
            const float4 v = __ldcg(cs4 + i);
            tmax = fmaxf(tmax, fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)));
        }
        for (int i = 4 * n4 + tid; i < n; i += kFinalThreads)
            tmax = fmaxf(tmax, __ldcg(cs + i));
        const int j = (k + kWarps - 1) / kWarps;
        float v = tmax, jth = 0.0f;
        for (int r = 0; r < j; ++r) {
            float mx = v;
#pragma unroll
            for (int o = 16; o; o >>= 1)
                mx = fmaxf(mx, __shfl_xor_sync(kFull, mx, o));
            jth = mx;
            const unsigned who = __ballot_sync(kFull, v == mx);
            if (lane == __ffs(who) - 1)
                v = -1.0f;
        }
        if (lane == 0)
            wv[warp] = fmaxf(jth, 0.0f);
        __syncthreads();
        if (tid == 0)
            surv_count = 0;
        const int m = (k + j - 1) / j;
        float w[kWarps];
#pragma unroll
        for (int i = 0; i < kWarps; ++i)
            w[i] = wv[i];
        float bound = 0.0f;
        for (int r = 0; r < m; ++r) {
            int best = 0;
#pragma unroll
            for (int i = 1; i < kWarps; ++i)
                if (w[i] > w[best])
                    best = i;
            bound = w[best];
#pragma unroll
            for (int i = 0; i < kWarps; ++i)
                if (i == best)
                    w[i] = -2.0f;
        }
        tau = fmaxf(bound, floor);
        __syncthreads();
        filter(tau);
        __syncthreads();
    }
    const unsigned c = surv_count;
    if (c <= 64u) {
        // a few survivors: each one's exact rank
        for (unsigned i = tid; i < c; i += kFinalThreads) {
            const float s = surv_s[i];
            const int id = surv_i[i];
            int rank = 0;
            for (unsigned t = 0; t < c; ++t)
                rank += Better(surv_s[t], surv_i[t], s, id);
            if (rank < k) {
                sel_s[rank] = s;
                sel_i[rank] = id;
            }
        }
        if (tid == 0)
            sel_count = (int)min(c, (unsigned)k);
    } else if (c <= (unsigned)kSurvCap) {
        // up to kSurvCap survivors: a bitonic sort by (score desc, id asc) in shared memory, padded
        // to a power of two with entries that order after every survivor
        unsigned p = 128u;
        while (p < c)
            p <<= 1;
        for (unsigned i = c + tid; i < p; i += kFinalThreads) {
            surv_s[i] = -1.0f;
            surv_i[i] = INT_MAX;
        }
        __syncthreads();
        for (unsigned size = 2; size <= p; size <<= 1)
            for (unsigned stride = size >> 1; stride > 0; stride >>= 1) {
                for (unsigned i = tid; i < p / 2; i += kFinalThreads) {
                    const unsigned lo = 2 * i - (i & (stride - 1)), hi = lo + stride;
                    const float ls = surv_s[lo], hs = surv_s[hi];
                    const int li = surv_i[lo], hid = surv_i[hi];
                    // runs whose bit `size` is clear end best-first, the others best-last
                    if (((lo & size) == 0) == Better(hs, hid, ls, li)) {
                        surv_s[lo] = hs;
                        surv_i[lo] = hid;
                        surv_s[hi] = ls;
                        surv_i[hi] = li;
                    }
                }
                __syncthreads();
            }
        for (int i = tid; i < k; i += kFinalThreads) {
            sel_s[i] = surv_s[i];
            sel_i[i] = surv_i[i];
        }
        if (tid == 0)
            sel_count = (int)min(c, (unsigned)k);
    } else {
        WarpTopK top;
        top.Reset();
        for (int base = warp * 32; base < n; base += kFinalThreads) {
            const int i = base + lane;
            float s = 0.0f;
            int id = kNoId;
            if (i < n) {
                s = __ldcg(cs + i);
                id = __ldcg(ci + i);
            }
            top.Offer(s, id, i < n && s > 0.0f && s >= tau, k, lane);
        }
        wl_s[warp][lane] = top.ls;
        wl_i[warp][lane] = top.li;
        __syncthreads();
        if (warp == 0) {
            top.Reset();
            for (int w2 = 0; w2 < kWarps; ++w2)
                top.Offer(wl_s[w2][lane], wl_i[w2][lane], wl_i[w2][lane] != kNoId, k, lane);
            const int cnt = __popc(__ballot_sync(kFull, lane < k && top.li != kNoId));
            if (lane < cnt) {
                sel_s[lane] = top.ls;
                sel_i[lane] = top.li;
            }
            if (lane == 0)
                sel_count = cnt;
        }
    }
    __syncthreads();
    if (warp == 0) {
        const int cnt = sel_count;
        float ls = -1.0f;
        int li = kNoId;
        if (lane < cnt) {
            ls = sel_s[lane];
            li = sel_i[lane];
        }
        int r = cnt;
        for (int d = 0; r < k && d < a.num_docs; ++d) {  // zero-score fill, smallest ids first
            if (!__any_sync(kFull, li == d)) {
                if (lane == r) {
                    ls = 0.0f;
                    li = d;
                }
                ++r;
            }
        }
        if (lane < k) {
            a.out_scores[OutRow(a, q) + lane] = ls;
            a.out_ids[OutRow(a, q) + lane] = li;
        }
        // K results at or above the starting bound, or no bound: the pruned result stands.  A
        // query that fell short keeps its group slots (real documents' scores, so still lower
        // bounds) for the retry pass; its threshold, which started at the guess, is dropped.
        const bool failed = a.exact && !a.retry && !(cnt == k || !(a.tau[q] > 0.0f));
        if (a.exact && !a.retry && lane == 0) {
            a.exact[q] = failed ? 0 : 1;
            if (failed)
                a.fail_out[atomicAdd(a.fail_out_count, 1u)] = q;
        }
        if (lane == 0) {
            a.cand_count[q] = 0u;
            a.threshold[q] = 0u;
        }
        if (!failed)
            a.tslots[(long long)q * 32 + lane] = 0u;
    }
}

// ---- final selection for K > 32 -------------------------------------------------
//
// One CTA per query over the query's candidate buffer (every document a tile
// appended at or above the running bound): candidates below the final floor are
// dropped, the K-th largest FP32 key (bit pattern of a positive score) is found by
// three radix passes (11/10/10 bits) of a shared-memory histogram, the documents
// above it are taken whole and the ties at it by ascending id (sorted in shared
// memory, or by a second radix select on ids when they do not fit), then the K
// results are sorted by (score desc, id asc) with a bitonic network and the
// zero-score fill takes the smallest free ids.  A query whose buffer overflowed is
// put on the fail list; a retry pass searches it again from its group slots (real
// documents' scores: its first pass has filled them).
constexpr int kLargeThreads = 512;
constexpr int kLargeMaxK = 1024;
constexpr int kLargeEqCap = 2048;
constexpr int kRadixBins = 2048;

struct LargeShared {
    unsigned hist[kRadixBins];
    float sel_s[kLargeMaxK];
    int sel_i[kLargeMaxK];
    int eq[kLargeEqCap];
    unsigned wsum[kLargeThreads / 32];
    unsigned fill[kLargeMaxK / 32];
    unsigned sel_count, eq_count, total;
    int bucket;
    unsigned above;
};

// Every thread calls.  Histogram of bits [shift, shift + log2 bins) of the keys that match
// `prefix` on `mask`; returns the bin holding the need-th largest such key and, in *above,
// the count of matching keys in higher bins (need >= 1 and at most the matching count).
template <class KeyOf>
__device__ int RadixStep(LargeShared &sh, int n, const KeyOf &key_of, unsigned prefix, unsigned mask, int shift,
                         int bins, unsigned need, unsigned *above)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < bins; i += kLargeThreads)
        sh.hist[i] = 0u;
    __syncthreads();
    for (int i = tid; i < n; i += kLargeThreads) {
        unsigned key;
        if (key_of(i, &key) && (key & mask) == prefix)
            atomicAdd(&sh.hist[(key >> shift) & (unsigned)(bins - 1)], 1u);
    }
    __syncthreads();
    // thread t owns bins [hi - per, hi), hi = bins - t * per: thread 0 holds the top bins
    const int per = bins / kLargeThreads;
    const int hi = bins - tid * per;
    unsigned local = 0;
    for (int b = hi - 1; b >= hi - per; --b)
        local += sh.hist[b];
    unsigned incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(kFull, incl, o);
        if (lane >= o)
            incl += v;
    }
    if (lane == 31)
        sh.wsum[warp] = incl;
    __syncthreads();
    for (int w = 0; w < warp; ++w)
        incl += sh.wsum[w];
    const unsigned excl = incl - local;
    if (excl < need && need <= incl) {
        unsigned c = excl;
        for (int b = hi - 1; b >= hi - per; --b) {
            if (c + sh.hist[b] >= need) {
                sh.bucket = b;
                sh.above = c;
                break;
            }
            c += sh.hist[b];
        }
    }
    __syncthreads();
    *above = sh.above;
    const int bucket = sh.bucket;
    __syncthreads();  // hist and the results are rewritten by the next step
    return bucket;
}

// The need-th largest 31-bit key among the candidates key_of accepts (three passes).
template <class KeyOf>
__device__ unsigned RadixSelect31(LargeShared &sh, int n, const KeyOf &key_of, unsigned need, unsigned *rest)
{
    unsigned above, prefix = 0, mask = 0;
    int b = RadixStep(sh, n, key_of, prefix, mask, 20, 2048, need, &above);
    prefix |= (unsigned)b << 20;
    mask |= 0x7ffu << 20;
    need -= above;
    b = RadixStep(sh, n, key_of, prefix, mask, 10, 1024, need, &above);
    prefix |= (unsigned)b << 10;
    mask |= 0x3ffu << 10;
    need -= above;
    b = RadixStep(sh, n, key_of, prefix, mask, 0, 1024, need, &above);
    prefix |= (unsigned)b;
    need -= above;
    *rest = need;  // keys equal to the result still to take (>= 1)
    return prefix;
}

// Bitonic sort of p (a power of two <= 2048) entries in shared memory; `before(i, j)`
// orders entry i ahead of entry j; `swap(i, j)` exchanges them.  Every thread calls.
template <class Before, class Swap>
__device__ void BlockBitonic(int p, const Before &before, const Swap &swap)
{
    for (int size = 2; size <= p; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < p; i += kLargeThreads) {
                const int j = i ^ stride;
                if (j > i) {
                    const bool up = (i & size) == 0;
                    if (up ? before(j, i) : before(i, j))
                        swap(i, j);
                }
            }
            __syncthreads();
        }
}

// Each listed term's posting scores at ranks 64, 128, 256, 512 and 1024 (largest first; 0 past the
// term's document frequency): ranks [term][kRankCount].  One CTA per term: a list of at most 1024
// postings is sorted whole in shared memory; a longer one takes its 1024-th largest score by three
// radix passes, then sorts the scores above it (fewer than 1024; the rest of the ranks tie at it).
constexpr int kRankCount = 5;
__global__ void __launch_bounds__(kLargeThreads) TermRanksKernel(const long long *indptr, const float *data,
                                                                 const int *terms, int n_terms, float *ranks)
{
    __shared__ LargeShared sh;
    const int tid = threadIdx.x;
    for (int ti = blockIdx.x; ti < n_terms; ti += gridDim.x) {
        const int t = terms[ti];
        const long long s = indptr[t];
        const int df = (int)(indptr[t + 1] - s);
        const float *v = data + s;
        float top = 0.0f;  // the 1024-th largest score when the list is longer
        if (tid == 0)
            sh.sel_count = 0u;
        __syncthreads();
        if (df <= kLargeMaxK) {
            for (int i = tid; i < kLargeMaxK; i += kLargeThreads)
                sh.sel_s[i] = i < df ? fmaxf(v[i], 0.0f) : -1.0f;
            if (tid == 0)
                sh.sel_count = (unsigned)df;
        } else {
            auto key_of = [&](int i, unsigned *key) {
                *key = __float_as_uint(fmaxf(__ldg(v + i), 0.0f)) & 0x7fffffffu;
                return true;
            };
            unsigned rest = 0;
            const unsigned kth = RadixSelect31(sh, df, key_of, (unsigned)kLargeMaxK, &rest);
            top = __uint_as_float(kth);
            for (int i = tid; i < kLargeMaxK; i += kLargeThreads)
                sh.sel_s[i] = -1.0f;
            __syncthreads();
            for (int i = tid; i < df; i += kLargeThreads) {
                const float x = fmaxf(__ldg(v + i), 0.0f);
                if (x > top)
                    sh.sel_s[atomicAdd(&sh.sel_count, 1u)] = x;  // fewer than 1024 are above the 1024-th
            }
        }
        __syncthreads();
        BlockBitonic(
            kLargeMaxK, [&](int i, int j) { return sh.sel_s[i] > sh.sel_s[j]; },
            [&](int i, int j) {
                const float x = sh.sel_s[i];
                sh.sel_s[i] = sh.sel_s[j];
                sh.sel_s[j] = x;
            });
        if (tid < kRankCount) {
            const int r = 64 << tid;  // rank r: sel_s[r - 1] when above the 1024-th, else that score
            const unsigned above = df <= kLargeMaxK ? (unsigned)df : sh.sel_count;
            float x = 0.0f;
            if (r <= df)
                x = (unsigned)r <= above ? sh.sel_s[r - 1] : top;
            ranks[(long long)t * kRankCount + tid] = x;
        }
        __syncthreads();  // sh is reused for the next term
    }
}

__global__ void __launch_bounds__(kLargeThreads) FinalSelectLargeKernel(const StreamArgs a)
{
    __shared__ LargeShared sh;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int q = blockIdx.x;
    if (a.retry) {
        if ((unsigned)q >= __ldcg(a.fail_in_count))
            return;
        q = __ldcg(a.fail_in + q);
    }
    const int k = QueryK(a, q);
    if (k <= kMaxSmallK)
        return;  // FinalSelectKernel's query
    const unsigned appended = __ldcg(a.cand_count + q);
    // floor: the query's threshold, or the least of the 32 slots (32 m >= K documents reach it)
    if (warp == 0) {
        const unsigned m = __reduce_min_sync(kFull, __ldcg(a.tslots + (long long)q * 32 + lane));
        if (lane == 0) {
            sh.above = m;
            sh.sel_count = 0u;
            sh.eq_count = 0u;
            sh.total = 0u;
        }
    }
    __syncthreads();
    const float floor = fmaxf(__uint_as_float(__ldcg(a.threshold + q)), __uint_as_float(sh.above));
    if ((long long)appended > a.cand_cap) {
        if (a.fail_out) {
            // search the query again: its group slots (real documents' scores) stay as the
            // starting bound; the threshold may hold a guess and is dropped
            if (tid == 0) {
                a.threshold[q] = 0u;
                a.cand_count[q] = 0u;
                if (a.exact && !a.retry)
                    a.exact[q] = 0;
                a.fail_out[atomicAdd(a.fail_out_count, 1u)] = q;
            }
            return;
        }
        if (tid == 0)
            atomicOr(a.status, kStatusCandOverflow);
    }
    const int n = (int)min((long long)appended, a.cand_cap);
    const float *cs = a.cand_scores + (long long)q * a.cand_cap;
    const int *ci = a.cand_ids + (long long)q * a.cand_cap;
    auto score_key = [&](int i, unsigned *key) -> bool {
        const float s = __ldcg(cs + i);
        *key = __float_as_uint(s);
        return s > 0.0f && s >= floor;
    };
    {
        unsigned c = 0, key;
        for (int i = tid; i < n; i += kLargeThreads)
            c += score_key(i, &key);
        c = __reduce_add_sync(kFull, c);
        if (lane == 0)
            atomicAdd(&sh.total, c);
    }
    __syncthreads();
    const unsigned total = sh.total;
    unsigned kth_key = 0, need = 0;
    if (total > (unsigned)k)
        kth_key = RadixSelect31(sh, n, score_key, (unsigned)k, &need);
    // documents above the K-th key (all of them when no more than K qualify); ties at it apart
    for (int i = tid; i < n; i += kLargeThreads) {
        unsigned key;
        if (!score_key(i, &key))
            continue;
        if (total <= (unsigned)k || key > kth_key) {
            const unsigned at = atomicAdd(&sh.sel_count, 1u);
            if (at < (unsigned)kLargeMaxK) {  // at most K - 1 by the radix select
                sh.sel_s[at] = __uint_as_float(key);
                sh.sel_i[at] = __ldcg(ci + i);
            }
        } else if (key == kth_key) {
            const unsigned at = atomicAdd(&sh.eq_count, 1u);
            if (at < (unsigned)kLargeEqCap)
                sh.eq[at] = __ldcg(ci + i);
        }
    }
    __syncthreads();
    if (total > (unsigned)k) {
        const unsigned eqn = sh.eq_count;
        const unsigned base = sh.sel_count;  // k - need
        if (eqn <= (unsigned)kLargeEqCap) {
            // the need smallest ids among the ties
            int p = 1;
            while (p < (int)eqn)
                p <<= 1;
            for (int i = (int)eqn + tid; i < p; i += kLargeThreads)
                sh.eq[i] = INT_MAX;
            __syncthreads();
            BlockBitonic(
                p, [&](int i, int j) { return sh.eq[i] < sh.eq[j]; },
                [&](int i, int j) {
                    const int t = sh.eq[i];
                    sh.eq[i] = sh.eq[j];
                    sh.eq[j] = t;
                });
            for (unsigned i = tid; i < need && base + i < (unsigned)kLargeMaxK && i < (unsigned)p; i += kLargeThreads) {
                sh.sel_s[base + i] = __uint_as_float(kth_key);
                sh.sel_i[base + i] = sh.eq[i];
            }
        } else {
            // too many ties to sort here: the need-th smallest id by a radix select on
            // 0x7fffffff - id over the tied candidates, then every tie at or below it
            auto id_key = [&](int i, unsigned *key) -> bool {
                const float s = __ldcg(cs + i);
                *key = 0x7fffffffu - (unsigned)__ldcg(ci + i);
                return __float_as_uint(s) == kth_key && s >= floor;
            };
            unsigned rest;
            const unsigned cut = 0x7fffffffu - RadixSelect31(sh, n, id_key, need, &rest);
            if (tid == 0)
                sh.eq_count = 0u;
            __syncthreads();
            for (int i = tid; i < n; i += kLargeThreads) {
                unsigned key;
                if (id_key(i, &key) && 0x7fffffffu - key <= cut) {
                    const unsigned at = base + atomicAdd(&sh.eq_count, 1u);
                    if (at < (unsigned)kLargeMaxK) {
                        sh.sel_s[at] = __uint_as_float(kth_key);
                        sh.sel_i[at] = (int)(0x7fffffffu - key);
                    }
                }
            }
        }
        if (tid == 0)
            sh.sel_count = (unsigned)k;
    }
    __syncthreads();
    const int c = (int)min(sh.sel_count, (unsigned)k);
    int p = 1;
    while (p < c)
        p <<= 1;
    for (int i = c + tid; i < p; i += kLargeThreads) {
        sh.sel_s[i] = -1.0f;
        sh.sel_i[i] = INT_MAX;
    }
    for (int i = tid; i < kLargeMaxK / 32; i += kLargeThreads)
        sh.fill[i] = 0u;
    __syncthreads();
    BlockBitonic(
        p, [&](int i, int j) { return Better(sh.sel_s[i], sh.sel_i[i], sh.sel_s[j], sh.sel_i[j]); },
        [&](int i, int j) {
            const float ts = sh.sel_s[i];
            const int ti = sh.sel_i[i];
            sh.sel_s[i] = sh.sel_s[j];
            sh.sel_i[i] = sh.sel_i[j];
            sh.sel_s[j] = ts;
            sh.sel_i[j] = ti;
        });
    float *os = a.out_scores + OutRow(a, q);
    int *oi = a.out_ids + OutRow(a, q);
    for (int i = tid; i < c; i += kLargeThreads) {
        os[i] = sh.sel_s[i];
        oi[i] = sh.sel_i[i];
        if (sh.sel_i[i] < k)
            atomicOr(&sh.fill[sh.sel_i[i] >> 5], 1u << (sh.sel_i[i] & 31));
    }
    __syncthreads();
    if (c < k && tid == 0) {  // zero-score fill, smallest free ids first (all below k)
        int r = c;
        for (int d = 0; r < k && d < a.num_docs; ++d)
            if (!((sh.fill[d >> 5] >> (d & 31)) & 1u)) {
                os[r] = 0.0f;
                oi[r] = d;
                ++r;
            }
    }
    const bool failed = a.exact && !a.retry && !(c == k || !(a.tau[q] > 0.0f));
    if (tid == 0) {
        if (a.exact && !a.retry) {
            a.exact[q] = failed ? 0 : 1;
            if (failed)
                a.fail_out[atomicAdd(a.fail_out_count, 1u)] = q;
        }
        a.cand_count[q] = 0u;
        a.threshold[q] = 0u;
    }
    if (warp == 0 && !failed)  // a failed query keeps its slots for the retry pass
        a.tslots[(long long)q * 32 + lane] = 0u;
}

} // namespace bm25k
