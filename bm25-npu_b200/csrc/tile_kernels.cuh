// Fused BM25 scoring + local top-K + tiered merge for sm_100a.
//
// One CTA owns one (query, tile) pair, a tile being `tile_docs` consecutive
// documents whose FP32 scores live in shared memory.  This replaces the
// reference's per-(query, 8192-doc leaf) task of
//   feature_retrieval/src/ascendfaiss/ops/ascendc/bm25/fused/op_kernel/bm25_fused_score_top_k.cpp:637-936
// and its separate 32-way merge operator
//   feature_retrieval/src/ascendfaiss/ops/ascendc/bm25/merge/op_kernel/bm25_top_k_merge.cpp:10-98
// with a single launch:
//   1. posting sub-range of every query term inside the tile, from the per-tile
//      posting directory (long lists) or a cooperative count over the whole list
//      (short lists);
//   2. term-ordered accumulation: for each term in query order the CTA streams
//      the term's (doc id, FP32 score) postings with 128-bit read-only loads and
//      adds them into the shared-memory row; a barrier between terms makes every
//      document's sum exactly ((0 + s_t1) + s_t2) + ... in query order, the
//      order of cpu_index_search.h:176-188;
//   3. documents whose score first turns positive are appended to a shared
//      candidate list with one warp ballot and one shared atomic per warp
//      (the reference's append, bm25_fused_score_top_k.cpp:755-769);
//   4. exact local top-K by warp insertion select over the candidates (or the
//      whole row when the list overflowed), ordered score desc, id asc;
//   5. merge tree: the CTA writes its list and arrives on its parent node; the
//      last child to arrive merges the node's children (fan-in F) and climbs,
//      so tree levels run inside the same launch as the scoring;
//   6. the root adds the zero-score fill (smallest ids not already ranked) and
//      writes the query's final K results.
#pragma once
#include <cfloat>
#include <cstdint>

namespace bm25k {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxTerms = 64;  // per query, the reference's packet limit (fixed_query_packet.h:32)
constexpr int kCandCap = 2048; // shared candidate slots; overflow falls back to a full-row scan
constexpr int kMaxLevels = 8;
constexpr int kMaxSmallK = 32; // warp insertion select keeps one candidate per lane
constexpr unsigned kFull = 0xffffffffu;
constexpr int kNoId = 0x7fffffff;

enum : uint32_t {
    kStatusOverflow = 1u,    // a document sum left the finite FP32 range
    kStatusBadWord = 2u,     // negative word id reached the device
    kStatusBadPosting = 4u,  // posting outside its tile (corrupt directory or index)
    kStatusBadQuery = 8u,    // query offsets out of contract
};

struct Level {
    float *scores;       // [Q][n][K]
    int *ids;            // [Q][n][K]
    int *counts;         // [Q][n]
    unsigned *arrivals;  // [Q][n] children arrived (levels >= 1)
    int n;               // lists per query at this level
};

struct TileArgs {
    const long long *indptr;  // [V + 1]
    const int *indices;       // [M + pad]
    const float *data;        // [M + pad]
    const int *dir_row;       // [V] row of the term in `dir`, -1 for short lists
    const int *dir;           // [rows][tiles + 1] posting offsets relative to indptr[t]
    long long dir_stride;
    const long long *qoffsets;  // [Q + 1]
    const int *words;
    long long word_cap;         // words readable; a query reaching beyond is rejected
    int vocab, num_docs, tile_docs, tiles, k, fan_in, levels;
    Level lv[kMaxLevels];
    float *out_scores;  // [Q][K]
    int *out_ids;
    unsigned *status;
};

struct TileShared {
    long long beg[kMaxTerms];
    long long end[kMaxTerms];
    unsigned cnt_lo[kMaxTerms];
    unsigned cnt_hi[kMaxTerms];
    int scan[kMaxTerms];
    float wl_s[kWarps][32];
    int wl_i[kWarps][32];
    int cand[kCandCap];
    unsigned cand_count;
    unsigned bad;
    int nonempty;
    int last;
};

// Programmatic dependent launch.  A kernel launched with programmatic stream serialization may
// start while the kernel before it in the stream still runs: it waits in WaitPrerequisites
// (until that kernel has completed and its writes are visible) before reading anything that
// kernel wrote.  AllowDependents lets the next such kernel start early.  Both are no-ops when
// no launch in the stream uses the attribute.
__device__ __forceinline__ void WaitPrerequisites() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void AllowDependents() { asm volatile("griddepcontrol.launch_dependents;" :::); }

__device__ __forceinline__ bool Better(float as, int ai, float bs, int bi)
{
    return as > bs || (as == bs && ai < bi);
}

// Warp insertion select.  Lane l holds the l-th best (score, id) seen by the
// warp, l < k <= 32, sorted best first; empty slots hold (-1, kNoId).  Offers one
// candidate per lane; only those beating the current K-th entry are inserted,
// one at a time, by a ballot-ranked shift.
__device__ __forceinline__ void WarpOffer(float cs, int ci, bool has, float &ls, int &li, int k, int lane)
{
    float ts = __shfl_sync(kFull, ls, k - 1);
    int ti = __shfl_sync(kFull, li, k - 1);
    unsigned pending = __ballot_sync(kFull, has && Better(cs, ci, ts, ti));
    while (pending) {
        const int src = __ffs(pending) - 1;
        pending &= pending - 1;
        const float s = __shfl_sync(kFull, cs, src);
        const int id = __shfl_sync(kFull, ci, src);
        ts = __shfl_sync(kFull, ls, k - 1);
        ti = __shfl_sync(kFull, li, k - 1);
        if (Better(s, id, ts, ti)) {  // uniform: every lane sees the same values
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
        }
    }
}

// Every thread calls; afterwards warp 0 holds the merge of all warps' lists.
__device__ __forceinline__ void BlockMerge(TileShared &sh, float &ls, int &li, int k, int lane, int warp)
{
    sh.wl_s[warp][lane] = ls;
    sh.wl_i[warp][lane] = li;
    __syncthreads();
    if (warp == 0) {
        ls = -1.0f;
        li = kNoId;
        for (int w = 0; w < kWarps; ++w) {
            const float cs = sh.wl_s[w][lane];
            const int ci = sh.wl_i[w][lane];
            WarpOffer(cs, ci, ci != kNoId, ls, li, k, lane);
        }
    }
    __syncthreads();
}

// Warp 0 only: zero-score fill and final write of one query's K results.
__device__ __forceinline__ void WriteFinal(const TileArgs &a, int q, float ls, int li, int lane)
{
    int r = __popc(__ballot_sync(kFull, lane < a.k && li != kNoId));
    for (int d = 0; r < a.k && d < a.num_docs; ++d) {  // warp-uniform
        const bool present = __any_sync(kFull, li == d);
        if (!present) {
            if (lane == r) {
                ls = 0.0f;
                li = d;
            }
            ++r;
        }
    }
    if (lane < a.k) {
        a.out_scores[(long long)q * a.k + lane] = ls;
        a.out_ids[(long long)q * a.k + lane] = li;
    }
}

// Publishes the list held by warp 0 as node `idx` of `level` and arrives at the
// parent.  Returns true in every thread of the CTA that must merge the parent.
__device__ __forceinline__ bool EmitAndArrive(const TileArgs &a, TileShared &sh, int q, int level, int idx, float ls,
                                              int li, int tid, int lane, int warp)
{
    const Level &L = a.lv[level];
    if (L.n == 1) {
        if (warp == 0)
            WriteFinal(a, q, ls, li, lane);
        return false;
    }
    if (warp == 0) {
        const long long node = (long long)q * L.n + idx;
        const int count = __popc(__ballot_sync(kFull, lane < a.k && li != kNoId));
        if (lane < count) {
            L.scores[node * a.k + lane] = ls;
            L.ids[node * a.k + lane] = li;
        }
        if (lane == 0)
            L.counts[node] = count;
        __threadfence();
    }
    __syncthreads();
    if (tid == 0) {
        const Level &P = a.lv[level + 1];
        const int parent = idx / a.fan_in;
        const int children = min(a.fan_in, L.n - parent * a.fan_in);
        unsigned *counter = P.arrivals + (long long)q * P.n + parent;
        const unsigned ticket = atomicAdd(counter, 1u);
        const int last = ticket == (unsigned)(children - 1);
        if (last)
            *counter = 0u;  // every child has arrived: reset for the next Search
        sh.last = last;
    }
    __syncthreads();
    const bool last = sh.last != 0;
    if (last)
        __threadfence();
    return last;
}

// Merges the children of node `parent` (level + 1) from `level`; warp 0 ends with the result.
__device__ __forceinline__ void MergeChildren(const TileArgs &a, TileShared &sh, int q, int level, int parent,
                                              float &ls, int &li, int lane, int warp)
{
    const Level &L = a.lv[level];
    const int c0 = parent * a.fan_in;
    const int c1 = min(c0 + a.fan_in, L.n);
    const int entries = (c1 - c0) * a.k;
    ls = -1.0f;
    li = kNoId;
    for (int base = warp * 32; base < entries; base += kThreads) {
        const int e = base + lane;
        bool has = false;
        float cs = -1.0f;
        int ci = kNoId;
        if (e < entries) {
            const long long node = (long long)q * L.n + c0 + e / a.k;
            const int r = e % a.k;
            if (r < __ldcg(L.counts + node)) {
                has = true;
                cs = __ldcg(L.scores + node * a.k + r);
                ci = __ldcg(L.ids + node * a.k + r);
            }
        }
        WarpOffer(cs, ci, has, ls, li, a.k, lane);
    }
    BlockMerge(sh, ls, li, a.k, lane, warp);
}

__device__ __forceinline__ int4 LoadNc(const int *p) { return __ldg(reinterpret_cast<const int4 *>(p)); }
__device__ __forceinline__ float4 LoadNc(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }

// Adds one posting into the row; returns true when the document first turns positive.
__device__ __forceinline__ bool AddPosting(float *row, long long pos, long long b, long long e, int id, float v,
                                           long long lo, int tile_docs, unsigned &bad, int &local)
{
    if (pos < b || pos >= e)
        return false;
    const long long d = (long long)id - lo;
    if (d < 0 || d >= tile_docs) {
        bad |= kStatusBadPosting;
        return false;
    }
    local = (int)d;
    const float old = row[d];
    const float sum = old + v;
    row[d] = sum;
    if (!(sum <= FLT_MAX))
        bad |= kStatusOverflow;
    return old == 0.0f && sum > 0.0f;
}

__device__ __forceinline__ void Append(TileShared &sh, bool first, int local, int lane)
{
    const unsigned hits = __ballot_sync(kFull, first);
    if (hits) {
        const int leader = __ffs(hits) - 1;
        unsigned base = 0;
        if (lane == leader)
            base = atomicAdd(&sh.cand_count, (unsigned)__popc(hits));
        base = __shfl_sync(kFull, base, leader);
        if (first) {
            const unsigned slot = base + __popc(hits & ((1u << lane) - 1u));
            if (slot < (unsigned)kCandCap)
                sh.cand[slot] = local;
        }
    }
}

// Streams one term's postings [b, e) into the row; warp-uniform loop bounds.
__device__ __forceinline__ void ScoreTerm(const TileArgs &a, float *row, TileShared &sh, long long b, long long e,
                                          long long lo, int lane, int warp, unsigned &bad)
{
    const long long a0 = b & ~3LL;
    constexpr long long kStep = (long long)kThreads * 4;
    for (long long base = a0 + (long long)warp * 128; base < e; base += 2 * kStep) {
        const long long p0 = base + lane * 4;
        const long long p1 = p0 + kStep;
        const bool second = base + kStep < e;  // warp-uniform
        const int4 i0 = LoadNc(a.indices + p0);
        const float4 v0 = LoadNc(a.data + p0);
        int4 i1 = make_int4(0, 0, 0, 0);
        float4 v1 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (second) {
            i1 = LoadNc(a.indices + p1);
            v1 = LoadNc(a.data + p1);
        }
        int local = 0;
        bool f;
        f = AddPosting(row, p0 + 0, b, e, i0.x, v0.x, lo, a.tile_docs, bad, local);
        Append(sh, f, local, lane);
        f = AddPosting(row, p0 + 1, b, e, i0.y, v0.y, lo, a.tile_docs, bad, local);
        Append(sh, f, local, lane);
        f = AddPosting(row, p0 + 2, b, e, i0.z, v0.z, lo, a.tile_docs, bad, local);
        Append(sh, f, local, lane);
        f = AddPosting(row, p0 + 3, b, e, i0.w, v0.w, lo, a.tile_docs, bad, local);
        Append(sh, f, local, lane);
        if (second) {
            f = AddPosting(row, p1 + 0, b, e, i1.x, v1.x, lo, a.tile_docs, bad, local);
            Append(sh, f, local, lane);
            f = AddPosting(row, p1 + 1, b, e, i1.y, v1.y, lo, a.tile_docs, bad, local);
            Append(sh, f, local, lane);
            f = AddPosting(row, p1 + 2, b, e, i1.z, v1.z, lo, a.tile_docs, bad, local);
            Append(sh, f, local, lane);
            f = AddPosting(row, p1 + 3, b, e, i1.w, v1.w, lo, a.tile_docs, bad, local);
            Append(sh, f, local, lane);
        }
    }
}

__global__ void __launch_bounds__(kThreads, 2) TileSearchKernel(const TileArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    float *row = reinterpret_cast<float *>(smem);
    TileShared &sh = *reinterpret_cast<TileShared *>(smem + (size_t)a.tile_docs * sizeof(float));
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tile = blockIdx.x, q = blockIdx.y;
    const long long lo = (long long)tile * a.tile_docs, hi = lo + a.tile_docs;
    const long long qb = a.qoffsets[q];
    long long nq = a.qoffsets[q + 1] - qb;
    if (tid == 0) {
        sh.cand_count = 0;
        sh.bad = 0;
        sh.nonempty = 0;
    }
    if (nq < 0 || nq > kMaxTerms || qb < 0 || qb + nq > a.word_cap) {
        if (tid == 0)
            sh.bad = kStatusBadQuery;
        nq = 0;
    }
    const int nterms = (int)nq;
    if (tid < kMaxTerms) {
        sh.cnt_lo[tid] = 0;
        sh.cnt_hi[tid] = 0;
        sh.scan[tid] = 0;
        sh.beg[tid] = 0;
        sh.end[tid] = 0;
    }
    __syncthreads();
    unsigned bad = 0;
    // 1. posting sub-range of each term inside [lo, hi)
    if (tid < nterms) {
        const int term = a.words[qb + tid];
        if (term < 0) {
            bad |= kStatusBadWord;
        } else if (term < a.vocab) {
            const long long s = a.indptr[term], t = a.indptr[term + 1];
            const int r = a.dir_row[term];
            if (r >= 0) {
                const int *d = a.dir + (long long)r * a.dir_stride;
                sh.beg[tid] = s + d[tile];
                sh.end[tid] = s + d[tile + 1];
            } else {
                sh.beg[tid] = s;
                sh.end[tid] = t;
                sh.scan[tid] = 1;
            }
        }
    }
    __syncthreads();
    for (int s = 0; s < nterms; ++s) {
        if (!sh.scan[s])
            continue;
        const long long b = sh.beg[s], e = sh.end[s];
        unsigned clo = 0, chi = 0;
        for (long long p = b + tid; p < e; p += kThreads) {
            const int d = __ldg(a.indices + p);
            clo += d < lo;
            chi += d < hi;
        }
        clo = __reduce_add_sync(kFull, clo);
        chi = __reduce_add_sync(kFull, chi);
        if (lane == 0 && chi) {
            atomicAdd(&sh.cnt_lo[s], clo);
            atomicAdd(&sh.cnt_hi[s], chi);
        }
    }
    __syncthreads();
    if (tid < nterms) {
        if (sh.scan[tid]) {
            const long long b = sh.beg[tid];
            sh.end[tid] = b + sh.cnt_hi[tid];
            sh.beg[tid] = b + sh.cnt_lo[tid];
        }
        if (sh.end[tid] > sh.beg[tid])
            atomicOr(&sh.nonempty, 1);
    }
    __syncthreads();
    float ls = -1.0f;
    int li = kNoId;
    if (sh.nonempty) {
        // 2. zero the tile row
        float4 *row4 = reinterpret_cast<float4 *>(row);
        for (int i = tid; i < a.tile_docs / 4; i += kThreads)
            row4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        // 3. term-ordered accumulation
        for (int s = 0; s < nterms; ++s) {
            const long long b = sh.beg[s], e = sh.end[s];
            if (b < e)
                ScoreTerm(a, row, sh, b, e, lo, lane, warp, bad);
            __syncthreads();
        }
        // 4. local top-K
        const unsigned n = sh.cand_count;
        if (n <= (unsigned)kCandCap) {
            for (unsigned base = (unsigned)warp * 32; base < n; base += kThreads) {
                const unsigned i = base + lane;
                const bool has = i < n;
                float cs = -1.0f;
                int ci = kNoId;
                if (has) {
                    ci = sh.cand[i];
                    cs = row[ci];
                }
                WarpOffer(cs, ci, has, ls, li, a.k, lane);
            }
        } else {
            const int per = a.tile_docs / kWarps;
            for (int base = warp * per; base < (warp + 1) * per; base += 32) {
                const int d = base + lane;
                const float cs = row[d];
                WarpOffer(cs, d, cs > 0.0f, ls, li, a.k, lane);
            }
        }
    }
    if (bad)
        atomicOr(&sh.bad, bad);
    BlockMerge(sh, ls, li, a.k, lane, warp);
    if (warp == 0 && li != kNoId)
        li += (int)lo;
    if (tid == 0 && sh.bad)
        atomicOr(a.status, sh.bad);
    // 5./6. merge tree inside the same launch
    int level = 0, idx = tile;
    while (EmitAndArrive(a, sh, q, level, idx, ls, li, tid, lane, warp)) {
        const int parent = idx / a.fan_in;
        MergeChildren(a, sh, q, level, parent, ls, li, lane, warp);
        ++level;
        idx = parent;
    }
}

// ---------------------------------------------------------------------------
// Index preparation kernels (Init only, outside the Search timer).

// Eager posting scores from the reference's lazy index:
// data[p] = (idf[t] * (tf[p] * k1p1)) / (tf[p] + norm[doc]) with every operation
// rounded to FP32 (no contraction), bm25_fused_score_top_k.cpp:738-739.
// Each block takes a contiguous chunk of postings; each thread finds the term of
// its first posting by binary search and then walks the term forward.
constexpr long long kBuildChunk = 8192;

__device__ __forceinline__ long long TermOf(const long long *offsets, int vocab, long long p)
{
    long long lo = 0, hi = vocab;  // largest t with offsets[t] <= p
    while (hi - lo > 1) {
        const long long mid = lo + (hi - lo) / 2;
        if (offsets[mid] <= p)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

__global__ void BuildContributionsKernel(const long long *offsets, int vocab, long long postings, const int *docs,
                                         const float *tf, const float *norm, const float *idf, float k1p1,
                                         float *data, unsigned *status)
{
    for (long long c0 = (long long)blockIdx.x * kBuildChunk; c0 < postings; c0 += (long long)gridDim.x * kBuildChunk) {
        const long long c1 = min(c0 + kBuildChunk, postings);
        long long p = c0 + threadIdx.x;
        if (p >= c1)
            continue;
        long long t = TermOf(offsets, vocab, p);
        for (; p < c1; p += blockDim.x) {
            while (offsets[t + 1] <= p)
                ++t;
            const float f = tf[p];
            const float numerator = __fmul_rn(f, k1p1);
            const float c = __fdiv_rn(__fmul_rn(idf[t], numerator), __fadd_rn(f, norm[docs[p]]));
            if (!(c >= 0.0f && c <= FLT_MAX))
                atomicOr(status, kStatusOverflow);
            data[p] = c;
        }
    }
}

// Per-tile posting directory for long lists:
// dir[row][j] = (first posting of the term with doc >= j * tile_docs) - indptr[t],
// one thread per entry, lower_bound over the term's sorted doc ids.
// Dense rows: dense[r][doc] = the posting score of term dense_terms[r] in doc (the rows are
// zeroed before).  Grid y: rows; grid x strides over the term's postings.
__global__ void BuildDenseKernel(const long long *indptr, const int *indices, const float *data,
                                 const int *dense_terms, float *dense, long long stride)
{
    const int t = dense_terms[blockIdx.y];
    const long long s = indptr[t], e = indptr[t + 1];
    float *row = dense + (long long)blockIdx.y * stride;
    for (long long p = s + (long long)blockIdx.x * blockDim.x + threadIdx.x; p < e;
         p += (long long)gridDim.x * blockDim.x)
        row[indices[p]] = data[p];
}

__global__ void BuildDirectoryKernel(const long long *indptr, const int *indices, const int *dir_terms, long long rows,
                                     int tile_docs, int tiles, int *dir, long long stride)
{
    const long long total = rows * (long long)(tiles + 1);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / (tiles + 1);
        const int j = (int)(i % (tiles + 1));
        const int t = dir_terms[r];
        const long long s = indptr[t];
        long long lo = s, hi = indptr[t + 1];
        const long long target = (long long)j * tile_docs;
        while (lo < hi) {
            const long long mid = lo + (hi - lo) / 2;
            if ((long long)indices[mid] < target)
                lo = mid + 1;
            else
                hi = mid;
        }
        dir[r * stride + j] = (int)(lo - s);
    }
}

} // namespace bm25k
