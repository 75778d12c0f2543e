// Tile-group BM25 Search kernel for sm_100a (kernel 4, the default).
//
// Work unit (a "claim"): one query and a group of 8 consecutive 1024-document
// tiles.  In one query word, the postings of the 8 tiles are one contiguous
// run of the word's list, so a CTA moves them with one bulk copy, and its 8
// consumer warps -- warp j owns tile j of the group, with a private 4 KB FP32
// row in shared memory -- each add their own tile's part, whose bounds the plan
// already holds:
//   * the producer warp claims work from the global counter three claims ahead
//     (the counter atomic, the query offsets and the plan entries of later
//     claims are in flight while the current claim's copies are issued), and
//     streams each non-empty word run of the claim into a ring of `stages`
//     shared-memory stages with 1-D bulk async copies (cp.async.bulk ...
//     mbarrier::complete_tx, no multicast), a.chunk postings per stage at
//     most, with the 8 tiles' bounds in the stage's meta;
//   * consumer warp j waits on each stage itself (bounded), adds the postings
//     of its tile in that stage into its row -- stages arrive in word order and
//     one warp owns the row, so every document's FP32 sum is built in
//     query-term order with no barrier between warps -- and releases the stage;
//   * after the claim's last stage, warp j takes its row into registers (32
//     scores per lane), clears it, and appends the row's top-K at or above the
//     query's running bound to the query's candidate buffer.
// The running bound of a query is the larger of two lower bounds on its K-th
// score: the best K-th score of any one tile (atomicMax), and the least of K
// group slots, slot g holding the best tile maximum among tiles with
// tile % K == g -- K documents from K different tiles reach it.  The second
// rises to near the final K-th score within the first few hundred tiles, so
// most tiles append nothing.  Consecutive claims walk the queries of one tile
// group, so every query gets tiles early and words that queries share are read
// from DRAM once and from L2 after.  FinalSelectKernel finishes every query.
//
// A retry pass (a.retry) covers only the queries on the fail list: those whose
// pruned pass fell short of K documents, or whose K > 32 candidate buffer
// overflowed (their running bound then starts at the final bound of the first
// pass).
#pragma once
#include "stream_kernel.cuh"

namespace bm25k {

constexpr int kWgTileDocs = 1024;                // default documents per tile (kTile: 1024 or 2048)
constexpr int kWgWarps = 8;                      // consumer warps = tiles per claim
constexpr int kWgThreads = (kWgWarps + 1) * 32;  // + the producer warp
constexpr int kWgChunkMin = 512, kWgChunkMax = 4096;  // postings per ring stage (a.chunk)
constexpr int kWgPlanWords = 8;                  // words per claim prefetched (2 per lane)

enum : int {
    kWgFirstOfClaim = 1,
    kWgLastOfClaim = 2,
    kWgStop = 4,
};

// One warp's selection scratch: survivors to rank, then its sorted top-k.
struct WarpSel {
    float buf_s[kWarpSurvCap];
    int buf_i[kWarpSurvCap];
    float sel_s[32];
    int sel_i[32];
};

struct __align__(16) WgMeta {
    int2 be[kWgWarps];  // tile j's postings [be[j].x, be[j].y) of the stage's word (absolute)
    int4 span;          // x: ring element 0 is posting x; y: elements copied; z: query; w: first tile
    int flags;
    float thr;          // the query's running bound when the claim was taken
    int pad[2];
};

struct WgShared {
    unsigned long long full[kMaxStages];
    unsigned long long empty[kMaxStages];
    WgMeta meta[kMaxStages];
    WarpSel wsel[kWgWarps];
    int abort;
    // the producer's counters (in shared memory, not registers: every register of the producer
    // is one of every consumer thread too)
    unsigned n_claims, n_tiles;
    unsigned long long n_copied;
};

inline size_t TileGroupSmem(int stages, int chunk, int tile_docs)
{
    return (size_t)kWgWarps * tile_docs * sizeof(float) + 2 * (size_t)stages * chunk * sizeof(int) +
           sizeof(WgShared);
}

// Moves a warp's row (32 * kVec float4, lane-interleaved: element e of a lane is
// document base_id + 4 * (lane + 32 * (e / 4)) + e % 4) into registers x and
// clears it, in one pass.
template <int kVec>
__device__ __forceinline__ void WarpTakeRow(float4 *reg4, int lane, float *x)
{
#pragma unroll
    for (int j = 0; j < kVec; ++j) {
        const float4 v = reg4[lane + 32 * j];
        x[4 * j] = v.x;
        x[4 * j + 1] = v.y;
        x[4 * j + 2] = v.z;
        x[4 * j + 3] = v.w;
    }
#pragma unroll
    for (int j = 0; j < kVec; ++j)
        reg4[lane + 32 * j] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// WarpTakeRow over the 128-document blocks of `mask` only (block j is float4 j of every lane);
// the other blocks read as 0 and are left as they are (the caller keeps them zero).
template <int kVec>
__device__ __forceinline__ void WarpTakeRowMasked(float4 *reg4, int lane, float *x, unsigned mask)
{
#pragma unroll
    for (int j = 0; j < kVec; ++j) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if ((mask >> j) & 1u) {  // uniform
            v = reg4[lane + 32 * j];
            reg4[lane + 32 * j] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        x[4 * j] = v.x;
        x[4 * j + 1] = v.y;
        x[4 * j + 2] = v.z;
        x[4 * j + 3] = v.w;
    }
}

// "x >= thr and x > 0" is "x >= max(thr, least positive float)" for thr >= 0
constexpr float kLeastPositive = 1.40129846e-45f;

// Top-k (k <= 32) of a warp's row held in registers (layout of WarpTakeRow) among
// scores >= thr and > 0, sorted best first into ws.sel with global ids.  Returns
// the count; *kth receives the row's k-th score when it is known exactly (k
// candidates, none filtered below it), else 0.
template <int kVec>
__device__ __forceinline__ int WarpSelectRegs(WarpSel &ws, const float *x, float thr, int k, int base_id, int lane,
                                              float *kth)
{
    float tmax = 0.0f;
#pragma unroll
    for (int e = 0; e < 4 * kVec; ++e)
        tmax = fmaxf(tmax, x[e]);
    *kth = 0.0f;
    float tau = fmaxf(thr, kLeastPositive);
    if (!__any_sync(kFull, tmax >= tau))
        return 0;  // nothing reaches the bound: the common case once the bound has risen
    int pass = 0;
#pragma unroll
    for (int e = 0; e < 4 * kVec; ++e)
        pass += x[e] >= tau;
    int total = __reduce_add_sync(kFull, pass);
    if (total > k) {
        // k-th largest lane maximum: k lanes each hold a score >= it
        const float bound = __shfl_sync(kFull, WarpSortDesc(tmax, lane), k - 1);
        if (bound > tau) {
            tau = bound;
            pass = 0;
#pragma unroll
            for (int e = 0; e < 4 * kVec; ++e)
                pass += x[e] >= tau;
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
#pragma unroll
            for (int e = 0; e < 4 * kVec; ++e)
                if (x[e] >= tau) {
                    ws.buf_s[at] = x[e];
                    ws.buf_i[at] = base_id + 4 * (lane + 32 * (e >> 2)) + (e & 3);
                    ++at;
                }
        }
        __syncwarp();
        for (int i = lane; i < total; i += 32) {
            const float sc = ws.buf_s[i];
            const int id = ws.buf_i[i];
            int rank = 0;
            for (int t = 0; t < total; ++t)
                rank += Better(ws.buf_s[t], ws.buf_i[t], sc, id);
            if (rank < k) {
                ws.sel_s[rank] = sc;
                ws.sel_i[rank] = id;
            }
        }
        n = min(total, k);
    } else {
        // ties at the top overflow the buffer: insertion select over the registers
        WarpTopK top;
        top.Reset();
#pragma unroll
        for (int e = 0; e < 4 * kVec; ++e)
            top.Offer(x[e], base_id + 4 * (lane + 32 * (e >> 2)) + (e & 3), x[e] >= tau, k, lane);
        n = __popc(__ballot_sync(kFull, lane < k && top.li != kNoId));
        if (lane < n) {
            ws.sel_s[lane] = top.ls;
            ws.sel_i[lane] = top.li;
        }
    }
    __syncwarp();
    if (n == k)
        *kth = ws.sel_s[k - 1];
    return n;
}

// WarpTakeRow (of the blocks of `mask`) + WarpSelectRegs.
template <int kVec>
__device__ __forceinline__ int WarpRowSelect(WarpSel &ws, float4 *reg4, float thr, int k, int base_id, int lane,
                                             float *kth, unsigned mask = ~0u)
{
    float x[4 * kVec];
    if (mask == ~0u)
        WarpTakeRow<kVec>(reg4, lane, x);
    else
        WarpTakeRowMasked<kVec>(reg4, lane, x, mask);
    return WarpSelectRegs<kVec>(ws, x, thr, k, base_id, lane, kth);
}

// End of a tile: takes the warp's row (clearing it) and appends its documents at or
// above the bound `thr` to query q's candidate buffer -- the top K for K <= 32, every
// one for K > 32 -- and raises the query's threshold and group slots.  Returns status
// bits.  Every lane of the warp calls.
// kSmallK: every query's K is a.k <= 32 (the lean instantiation of the plain Search).
template <int kTile, bool kSmallK = false>
__device__ __forceinline__ unsigned TileSelectAppend(const StreamArgs &a, WarpSel &ws, float4 *row4, float thr, int q,
                                                     int tile, int lane, unsigned mask = ~0u)
{
    const int base_doc = tile * kTile;
    unsigned bad = 0;
    const int k = kSmallK ? a.k : QueryK(a, q);
    if (kSmallK || k <= 32) {
        float kth;
        const int sel = WarpRowSelect<kTile / 128>(ws, row4, thr, k, base_doc, lane, &kth, mask);
        if (sel > 0) {
            if (!(ws.sel_s[0] <= FLT_MAX))
                bad |= kStatusOverflow;  // an overflowed sum would be the tile's best score
            unsigned at = 0;
            if (lane == 0) {
                at = atomicAdd(a.cand_count + q, (unsigned)sel);
                if (kth > thr)
                    atomicMax(a.threshold + q, __float_as_uint(kth));
                atomicMax(a.tslots + (long long)q * 32 + tile % k, __float_as_uint(ws.sel_s[0]));
            }
            at = __shfl_sync(kFull, at, 0);
            if (lane < sel) {
                if ((long long)at + lane < a.cand_cap) {
                    const long long o = (long long)q * a.cand_cap + at + lane;
                    a.cand_scores[o] = ws.sel_s[lane];
                    a.cand_ids[o] = ws.sel_i[lane];
                } else {
                    bad |= kStatusCandOverflow;
                }
            }
        }
    } else if constexpr (!kSmallK) {
        // K > 32: slot tile % 32 takes the tile's m-th best (m = ceil(K / 32)), so the 32
        // slots stand for 32 m >= K documents; every document at or above the bound is
        // appended (the final select ranks them; a query whose buffer overflows is
        // searched again from its final bound)
        constexpr int kElems = kTile / 32;
        float x[kElems];
        if (mask == ~0u)
            WarpTakeRow<kTile / 128>(row4, lane, x);
        else
            WarpTakeRowMasked<kTile / 128>(row4, lane, x, mask);
        const int m = (k + 31) >> 5;
        float mth;
        const int sel = WarpSelectRegs<kTile / 128>(ws, x, thr, m, base_doc, lane, &mth);
        if (sel > 0 && !(ws.sel_s[0] <= FLT_MAX))
            bad |= kStatusOverflow;
        if (sel == m && lane == 0)
            atomicMax(a.tslots + (long long)q * 32 + tile % 32, __float_as_uint(mth));
        const float tau = fmaxf(thr, kLeastPositive);
        int pass = 0;
#pragma unroll
        for (int e = 0; e < kElems; ++e)
            pass += x[e] >= tau;
        const int total = __reduce_add_sync(kFull, pass);
        if (total) {
            int at = pass;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(kFull, at, o);
                if (lane >= o)
                    at += v;
            }
            unsigned base = 0;
            if (lane == 0)
                base = atomicAdd(a.cand_count + q, (unsigned)total);
            long long o = (long long)__shfl_sync(kFull, base, 0) + at - pass;
#pragma unroll
            for (int e = 0; e < kElems; ++e)
                if (x[e] >= tau) {
                    if (o < a.cand_cap) {
                        const long long g = (long long)q * a.cand_cap + o;
                        a.cand_scores[g] = x[e];
                        a.cand_ids[g] = base_doc + 4 * (lane + 32 * (e >> 2)) + (e & 3);
                    }
                    ++o;
                }
        }
    }
    return bad;
}

// A claim as the producer holds it: uniform fields plus one plan entry pair per lane.
struct WgClaim {
    bool valid;
    int q, tile0, n;
    long long qb, qe;    // qoffsets[q], qoffsets[q + 1]
    unsigned thr_bits;   // the query's threshold
    unsigned slot_bits;  // lane g < k: group slot g (others: all ones)
    int2 p0, p1;         // lane l: word l / 8 (p0) and 4 + l / 8 (p1) in tile tile0 + l % 8; .x = b, .y = e
};

// Range of word s (>= kWgPlanWords, warp-uniform) in tile j of the claim, from the plan.
__device__ __forceinline__ int2 WgFarRange(const StreamArgs &a, const WgClaim &c, int s, int j)
{
    if (c.tile0 + j >= a.tiles)
        return make_int2(0, 0);
    const PlanEntry pe = a.plan[(c.qb + s) * a.tiles + c.tile0 + j];
    return make_int2((int)pe.b, (int)pe.e);
}

// kTile: documents per tile (a.tile_docs), 1024 or 2048.  kLean: the plain first pass with one
// K <= 32 for every query (no retry list, no K per query): the instantiation with the fewest
// registers, so the most resident warps.
template <int kTile, bool kLean = false>
__global__ void __launch_bounds__(kWgThreads, kTile == 1024 ? 3 : 2) TileGroupKernel(const StreamArgs a)
{
    extern __shared__ __align__(128) unsigned char wg_smem[];
    float *rows = reinterpret_cast<float *>(wg_smem);
    const int chunk = a.chunk;
    int *ring_ids = reinterpret_cast<int *>(rows + (size_t)kWgWarps * kTile);
    float *ring_vals = reinterpret_cast<float *>(ring_ids + (size_t)a.stages * chunk);
    WgShared &sh = *reinterpret_cast<WgShared *>(ring_vals + (size_t)a.stages * chunk);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    AllowDependents();  // the final select may be placed as this kernel's CTAs retire

    if (tid == 0) {
        for (int i = 0; i < a.stages; ++i) {
            MbarInit(&sh.full[i], 1);
            MbarInit(&sh.empty[i], kWgWarps);
        }
        sh.abort = 0;
        sh.n_claims = sh.n_tiles = 0u;
        sh.n_copied = 0ull;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < kWgWarps * kTile / 4; i += kWgThreads)
        reinterpret_cast<float4 *>(rows)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    WaitPrerequisites();  // the plan (or the fail list) of the kernel before this one
    if (!kLean && a.retry && __ldcg(a.fail_in_count) == 0u)
        return;  // nothing to retry: the work counter is left untouched
    volatile int *abort = &sh.abort;
    const unsigned groups = (unsigned)((a.tiles + kWgWarps - 1) / kWgWarps);
    // a retry pass covers only the queries on the fail list (possibly none)
    const unsigned nq = !kLean && a.retry ? __ldcg(a.fail_in_count) : (unsigned)a.q;
    const unsigned claims = nq * groups;

    if (warp == kWgWarps) {
        // ================= producer warp =================
        unsigned long long g = 0;  // stages issued
        int pst = 0;               // next stage to issue
        unsigned wraps = 0;        // times the ring has wrapped
        unsigned bad = 0;
        bool dead = false;

        // Waits until stage pst is free (its previous use released).
        auto claim_stage = [&]() -> bool {
            int ok = 1;
            if (wraps > 0 && lane == 0)
                ok = MbarWait(&sh.empty[pst], (wraps - 1) & 1u, abort, WaitBudget(a)) ? 1 : 0;
            return __shfl_sync(kFull, ok, 0) != 0;
        };
        auto advance_stage = [&]() {
            ++g;
            if (++pst == a.stages) {
                pst = 0;
                ++wraps;
            }
        };
        // Claim pipeline, three claims deep so no fetch is waited on right after it is
        // issued: each round uses the current claim's plan entries and bounds (loaded one
        // round earlier), loads the next claim's, fetches the query offsets of the claim
        // after it, and issues the counter atomic for the one after that.
        // claim index -> query and group: consecutive claims walk the queries of one group
        auto decode = [&](unsigned c, WgClaim &w) {
            w.valid = c < claims;
            w.q = w.valid ? (int)(c % nq) : 0;
            if (!kLean && a.retry && w.valid)
                w.q = __ldcg(a.fail_in + w.q);
            w.tile0 = w.valid ? (int)(c / nq) * kWgWarps : 0;
            w.n = 0;
            w.qb = w.qe = 0;
            w.p0 = make_int2(0, 0);
            w.p1 = make_int2(0, 0);
            w.thr_bits = 0u;
            w.slot_bits = 0xffffffffu;
        };
        auto fetch_offsets = [&](WgClaim &w) {  // loads only; checked in fetch_plan
            if (w.valid) {
                w.qb = a.qoffsets[w.q];
                w.qe = a.qoffsets[w.q + 1];
            }
        };
        auto fetch_plan = [&](WgClaim &w) {  // loads only; the bounds are reduced when used
            if (!w.valid)
                return;
            long long nw = w.qe - w.qb;
            if (nw < 0 || nw > kMaxTerms || w.qb < 0 || w.qb + nw > a.word_cap) {
                bad |= kStatusBadQuery;
                nw = 0;
            }
            w.n = (int)nw;
            const int s0 = lane >> 3, j = lane & 7;
            const bool tile_ok = w.tile0 + j < a.tiles;
            if (tile_ok && s0 < w.n) {
                const PlanEntry pe = a.plan[(w.qb + s0) * a.tiles + w.tile0 + j];
                w.p0 = make_int2((int)pe.b, (int)pe.e);
            }
            if (tile_ok && s0 + 4 < w.n) {
                const PlanEntry pe = a.plan[(w.qb + s0 + 4) * a.tiles + w.tile0 + j];
                w.p1 = make_int2((int)pe.b, (int)pe.e);
            }
            w.thr_bits = __ldcg(a.threshold + w.q);
            if (lane < (kLean ? a.k : QueryK(a, w.q)))
                w.slot_bits = __ldcg(a.tslots + (long long)w.q * 32 + lane);
        };
        auto take_claim = [&]() -> unsigned {
            unsigned c = 0;
            if (lane == 0)
                c = atomicAdd(&a.ctrl->next, 1u);
            return c;  // lane 0's value; broadcast when decoded
        };

        // test hook: a stalled producer issues no stage (not even the stop), so every consumer's
        // bounded wait runs out and the launch reports kStatusTimeout
        if (a.inject && __ldcg(a.inject) != 0u)
            dead = true;
        WgClaim cur, nx1, nx2;
        decode(__shfl_sync(kFull, take_claim(), 0), nx1);
        fetch_offsets(nx1);
        fetch_plan(nx1);
        decode(__shfl_sync(kFull, take_claim(), 0), nx2);
        fetch_offsets(nx2);
        unsigned c3 = take_claim();
        while (!dead && nx1.valid) {
            cur = nx1;
            nx1 = nx2;
            fetch_plan(nx1);
            decode(__shfl_sync(kFull, c3, 0), nx2);
            fetch_offsets(nx2);
            c3 = take_claim();

            const float thr =
                fmaxf(__uint_as_float(cur.thr_bits), __uint_as_float(__reduce_min_sync(kFull, cur.slot_bits)));
            if (lane == 0) {
                ++sh.n_claims;
                sh.n_tiles += (unsigned)min(kWgWarps, a.tiles - cur.tile0);
            }
            // each word's run over the group, reduced within its 8 lanes
            const bool ne0 = cur.p0.x < cur.p0.y, ne1 = cur.p1.x < cur.p1.y;
            int lo0 = ne0 ? cur.p0.x : 0x7fffffff, hi0 = ne0 ? cur.p0.y : -1;
            int lo1 = ne1 ? cur.p1.x : 0x7fffffff, hi1 = ne1 ? cur.p1.y : -1;
#pragma unroll
            for (int o = 1; o < 8; o <<= 1) {
                lo0 = min(lo0, __shfl_xor_sync(kFull, lo0, o));
                hi0 = max(hi0, __shfl_xor_sync(kFull, hi0, o));
                lo1 = min(lo1, __shfl_xor_sync(kFull, lo1, o));
                hi1 = max(hi1, __shfl_xor_sync(kFull, hi1, o));
            }
            const unsigned m0 = __ballot_sync(kFull, ne0), m1 = __ballot_sync(kFull, ne1);
            // last non-empty word, for the last-of-claim flag
            int last_word = -1;
            for (int s = cur.n - 1; s >= kWgPlanWords && last_word < 0; --s)
                for (int j = 0; j < kWgWarps; ++j) {
                    const int2 r = WgFarRange(a, cur, s, j);
                    if (r.x < r.y) {
                        last_word = s;
                        break;
                    }
                }
            if (last_word < 0 && m1)
                last_word = 4 + (31 - __clz((int)m1)) / 8;
            if (last_word < 0 && m0)
                last_word = (31 - __clz((int)m0)) / 8;

            bool first = true;
            for (int s = 0; s <= last_word && !dead; ++s) {
                int lo, hi;
                if (s < 4) {
                    lo = __shfl_sync(kFull, lo0, s * 8);
                    hi = __shfl_sync(kFull, hi0, s * 8);
                } else if (s < kWgPlanWords) {
                    lo = __shfl_sync(kFull, lo1, (s - 4) * 8);
                    hi = __shfl_sync(kFull, hi1, (s - 4) * 8);
                } else {
                    lo = 0x7fffffff;
                    hi = -1;
                    for (int j = 0; j < kWgWarps; ++j) {
                        const int2 r = WgFarRange(a, cur, s, j);
                        if (r.x < r.y) {
                            lo = min(lo, r.x);
                            hi = max(hi, r.y);
                        }
                    }
                }
                if (hi < 0)
                    continue;  // the word has no postings in this group
                const long long a0 = (long long)lo & ~3LL, a1 = ((long long)hi + 3) & ~3LL;
                for (long long c0 = a0; c0 < a1;) {
                    const long long c1 = min(c0 + (long long)chunk, a1);
                    if (!claim_stage()) {
                        dead = true;
                        break;
                    }
                    const int st = pst;
                    WgMeta &m = sh.meta[st];
                    // tile bounds of word s: lane 8 * (s % 4) + j holds tile j
                    if (s < kWgPlanWords) {
                        if ((lane >> 3) == (s & 3))
                            m.be[lane & 7] = s < 4 ? cur.p0 : cur.p1;
                    } else if (lane < kWgWarps) {
                        m.be[lane] = WgFarRange(a, cur, s, lane);
                    }
                    if (lane == 0) {
                        m.span = make_int4((int)c0, (int)(c1 - c0), cur.q, cur.tile0);
                        m.flags = (first ? kWgFirstOfClaim : 0) | (s == last_word && c1 == a1 ? kWgLastOfClaim : 0);
                        m.thr = thr;
                    }
                    __syncwarp();  // the meta is complete before lane 0 starts the stage
                    if (lane == 0) {
                        const unsigned bytes = (unsigned)(c1 - c0) * 4u;
                        sh.n_copied += (unsigned long long)(c1 - c0);
                        MbarArriveExpectTx(&sh.full[st], 2u * bytes);
                        BulkLoad(ring_ids + (size_t)st * chunk, a.indices + c0, bytes, &sh.full[st]);
                        BulkLoad(ring_vals + (size_t)st * chunk, a.data + c0, bytes, &sh.full[st]);
                    }
                    __syncwarp();
                    first = false;
                    advance_stage();
                    c0 = c1;
                }
            }
        }
        if (!dead) {
            if (claim_stage()) {
                if (lane == 0) {
                    sh.meta[pst].flags = kWgStop;
                    MbarArrive(&sh.full[pst]);
                }
                __syncwarp();
                advance_stage();
            } else {
                dead = true;
            }
        }
        if (lane == 0) {
            if (bad)
                atomicOr(a.status, bad);
            if (a.stats) {
                atomicAdd(a.stats + kStatClaims, (unsigned long long)sh.n_claims);
                atomicAdd(a.stats + kStatTilesScanned, (unsigned long long)sh.n_tiles);
                atomicAdd(a.stats + kStatPostingsCopied, sh.n_copied);
            }
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

    // ================= consumer warp `warp` owns tile tile0 + warp of each claim =================
    float *row = rows + (size_t)warp * kTile;
    float4 *row4 = reinterpret_cast<float4 *>(row);
    WarpSel &ws = sh.wsel[warp];
    int st = 0;
    unsigned parity = 0;
    unsigned bad = 0;
    bool touched = false;
    for (;;) {
        if (!WarpWaitAll(&sh.full[st], parity, abort, WaitBudget(a)))
            break;
        const WgMeta &m = sh.meta[st];
        const int flags = m.flags;
        if (flags & kWgStop)
            break;
        const int4 span = m.span;
        const int2 be = m.be[warp];
        const int c0 = span.x;
        const int lo = max(be.x, c0) - c0, hi = min(be.y, c0 + span.y) - c0;
        const int q = span.z, tile = span.w + warp;
        const float thr = m.thr;
        const int base_doc = tile * kTile;
        const int *ids = ring_ids + (size_t)st * chunk;
        const float *vals = ring_vals + (size_t)st * chunk;
        if (lo < hi)
            touched = true;
        // windows of 128 ring elements from the 16-byte boundary at or below lo; lane l takes
        // elements 4l..4l+3 of a window with one 128-bit load of ids and one of scores
        for (int w0 = lo & ~3; w0 < hi; w0 += 128) {
            const int x = w0 + 4 * lane;
            int4 id4 = make_int4(0, 0, 0, 0);
            float4 v4 = make_float4(0.f, 0.f, 0.f, 0.f);
            if (x < hi) {
                id4 = *reinterpret_cast<const int4 *>(ids + x);
                v4 = *reinterpret_cast<const float4 *>(vals + x);
            }
            const int idv[4] = {id4.x, id4.y, id4.z, id4.w};
            const float vv[4] = {v4.x, v4.y, v4.z, v4.w};
            int d[4];
            bool ok[4];
            float r[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const bool in = x + u >= lo && x + u < hi;
                d[u] = idv[u] - base_doc;
                ok[u] = in && (unsigned)d[u] < (unsigned)kTile;
                if (in && !ok[u])
                    bad |= kStatusBadPosting;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (ok[u])
                    r[u] = row[d[u]];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (ok[u])
                    row[d[u]] = r[u] + vv[u];
        }
        __syncwarp();
        if (lane == 0)
            MbarArrive(&sh.empty[st]);
        if (++st == a.stages) {
            st = 0;
            parity ^= 1u;
        }
        if (!(flags & kWgLastOfClaim) || !touched)
            continue;
        touched = false;

        // ---- end of the claim: select this warp's tile ----
        bad |= TileSelectAppend<kTile, kLean>(a, ws, row4, thr, q, tile, lane);
        __syncwarp();
    }
    bad = __reduce_or_sync(kFull, bad);
    if (lane == 0 && (bad || *abort))
        atomicOr(a.status, bad | (*abort ? kStatusTimeout : 0u));
}

inline const void *TileGroupKernelFor(int tile_docs, bool lean = false)
{
    if (lean)
        return tile_docs == 2048 ? reinterpret_cast<const void *>(&TileGroupKernel<2048, true>)
                                 : reinterpret_cast<const void *>(&TileGroupKernel<1024, true>);
    return tile_docs == 2048 ? reinterpret_cast<const void *>(&TileGroupKernel<2048>)
                             : reinterpret_cast<const void *>(&TileGroupKernel<1024>);
}

} // namespace bm25k
