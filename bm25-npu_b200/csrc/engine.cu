// Host runtime of the B200 BM25 engine and its C ABI (include/bm25_b200.h).
//
// Replaces the reference's ACL session layer
//   feature_retrieval/src/ascendfaiss/ascendhost/src/bm25/large_search.cpp:107-212
//   feature_retrieval/src/ascendfaiss/ascendhost/src/bm25/planned_search.{h,cpp}
//   feature_retrieval/src/ascendfaiss/ascendhost/src/bm25/runtime.cpp
// with the CUDA runtime: a resident index in HBM, a per-tile posting directory
// built on the device, pinned host arenas for the query packet and the result,
// and one CUDA graph per (Q, K) holding H2D -> fused scoring/selection/merge ->
// D2H.  Search = validate + pack, graph replay, synchronise, validate result.
#include "bm25_b200.h"
#include "block_kernels.cuh"
#include "block_tile_kernel.cuh"
#include "learned_kernels.cuh"
#include "merge_kernel.cuh"
#include "stream_kernel.cuh"
#include "tile_group_kernel.cuh"
#include "tile_kernels.cuh"
#include "warp_tile_kernel.cuh"

#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

namespace bm25b200 {

// Exception classes of common/bm25/error.h:8-31.
struct InvalidArgument : std::runtime_error {
    explicit InvalidArgument(const std::string &m) : std::runtime_error(m) {}
};
struct InvalidState : std::runtime_error {
    explicit InvalidState(const std::string &m) : std::runtime_error(m) {}
};
struct DeviceError : std::runtime_error {
    DeviceError(int64_t c, const std::string &m) : std::runtime_error(m), code(c) {}
    int64_t code;
};

static void Check(bool ok, const std::string &message)
{
    if (!ok)
        throw InvalidArgument(message);
}

static void Cuda(cudaError_t e, const char *what)
{
    if (e != cudaSuccess)
        throw DeviceError((int64_t)e, std::string(what) + ": " + cudaGetErrorString(e));
}

// A kernel's dynamic shared memory cap is one value per process and device,
// shared by every session: raise it to what this session needs, never lower it
// under a session created earlier with larger tiles.
static void RaiseSmemCap(const void *kernel, size_t bytes)
{
    cudaFuncAttributes attr{};
    Cuda(cudaFuncGetAttributes(&attr, kernel), "cudaFuncGetAttributes");
    if ((size_t)attr.maxDynamicSharedSizeBytes < bytes)
        Cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
             "cudaFuncSetAttribute");
}

static size_t Align32(size_t n) { return (n + 31) & ~size_t(31); }

// The kernels with 1024-document tiles, a K per query, K up to 1024 and the pruned paths: the
// warp-tile kernel (plain Searches; pruned Searches stream their routed and retried queries with
// the tile-group kernel) and the tile-group kernel.
static bool TileFamily(int kernel) { return kernel == BM25_KERNEL_TILE_GROUP || kernel == BM25_KERNEL_WARP_TILE; }

static_assert(bm25k::kTermTop == bm25k::kTermTopK, "one layout of the per-term top scores");

// Tiles per claim of the warp-tile kernel: the default, and the sizes a tuning may pick.
constexpr int kWtClaimTiles = 4;

// The warp-tile kernel with kC tiles per claim (2, 4 or 8).
template <bool kLean> static void (*WarpTileFor(int claim_tiles))(const bm25k::StreamArgs)
{
    switch (claim_tiles) {
    case 2:
        return bm25k::WarpTileKernel<2, kLean>;
    case 8:
        return bm25k::WarpTileKernel<8, kLean>;
    default:
        return bm25k::WarpTileKernel<4, kLean>;
    }
}

// Test hook: the next host-buffer Search of any session fails as a device error (bm25_test_inject
// with no handle).
static std::atomic<int> g_fail_next{0};

// Launch with programmatic stream serialization: the kernel may start while the kernel before it
// in the stream runs (the kernel waits in WaitPrerequisites before reading that kernel's output).
template <class... Params, class... Args>
static void LaunchOverlapped(void (*kernel)(Params...), dim3 grid, unsigned block, size_t smem, cudaStream_t s,
                             Args &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    Cuda(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...), "overlapped kernel launch");
}

constexpr int kPad = 256; // zero elements after the posting arrays for 128-bit tail loads

// ---------------------------------------------------------------------------
// Index validation (host, OpenMP over terms).

// Eager CSC rules: bm25s layout with sorted unique ids and finite non-negative scores.
static void ValidateEager(const int64_t *indptr, const int32_t *indices, const float *data, int64_t vocab,
                          int64_t docs)
{
    Check(indptr && indices && data, "Null index array");
    Check(vocab >= 1 && vocab < INT32_MAX && docs >= 1 && docs <= INT32_MAX, "Empty or oversized index");
    Check(indptr[0] == 0, "Index dimensions/endpoints differ");
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(| : bad)
    for (int64_t t = 0; t < vocab; ++t) {
        const int64_t b = indptr[t], e = indptr[t + 1];
        if (b < 0 || e < b) {
            bad |= 1;
            continue;
        }
        for (int64_t p = b; p < e; ++p) {
            const int32_t d = indices[p];
            if (d < 0 || d >= docs || (p > b && indices[p - 1] >= d))
                bad |= 2;
            const float v = data[p];
            if (!(v >= 0.0f && v <= 3.402823466e+38F))
                bad |= 4;
        }
    }
    Check(!(bad & 1), "Invalid posting bounds");
    Check(!(bad & 2), "Unsorted/duplicate/out-of-range posting ID");
    Check(!(bad & 4), "Invalid posting score");
}

// Lazy index rules of common/bm25/index_data.h:18-40.
static void ValidateLazy(const int64_t *offsets, const int32_t *docs, const float *tf, const float *norm,
                         const float *idf, int64_t vocab, int64_t ndocs)
{
    Check(offsets && docs && tf && norm && idf, "Null index array");
    Check(ndocs >= 1 && ndocs <= INT32_MAX && vocab >= 1 && vocab < INT32_MAX, "Empty or oversized index");
    Check(offsets[0] == 0 && offsets[vocab] >= 0 && offsets[vocab] <= INT32_MAX, "Index dimensions/endpoints differ");
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int64_t d = 0; d < ndocs; ++d)
        if (!(std::isfinite(norm[d]) && norm[d] > 0))
            bad |= 8;
    Check(!(bad & 8), "Invalid article norm");
#pragma omp parallel for schedule(dynamic, 1024) reduction(| : bad)
    for (int64_t t = 0; t < vocab; ++t) {
        if (!(std::isfinite(idf[t]) && idf[t] >= 0))
            bad |= 16;
        const int64_t b = offsets[t], e = offsets[t + 1];
        if (b < 0 || e < b) {
            bad |= 1;
            continue;
        }
        for (int64_t p = b; p < e; ++p) {
            const int32_t d = docs[p];
            if (d < 0 || d >= ndocs || (p > b && docs[p - 1] >= d))
                bad |= 2;
            const float f = tf[p];
            if (!(std::isfinite(f) && f >= 1 && f <= 16777216.0F && std::floor(f) == f))
                bad |= 4;
        }
    }
    Check(!(bad & 16), "Invalid IDF");
    Check(!(bad & 1), "Invalid posting bounds");
    Check(!(bad & 2), "Unsorted/duplicate/out-of-range posting ID");
    Check(!(bad & 4), "Invalid posting TF");
}

// ---------------------------------------------------------------------------

class Engine {
  public:
    struct Plan {
        int tile_docs = 0, tiles = 0, fan_in = 32, levels = 0;
        std::vector<int> lists;  // lists per query at each level
        int64_t dir_rows = 0, dir_min_df = 0;
        int kernel = 0, stages = 0, grid = 0, chunk = 0;
    };

    Engine(const bm25_options &o, int64_t vocab, int64_t docs, int64_t postings)
        : opts_(o), vocab_(vocab), docs_(docs), postings_(postings)
    {
        Check(o.max_k >= 1 && o.max_k <= bm25k::kLargeMaxK, "max_k must be in [1, 1024]");
        Check(o.max_k <= bm25k::kMaxSmallK || TileFamily(o.kernel),
              "max_k above 32 needs the warp-tile or tile-group kernel");
        Check(o.max_k <= docs, "max_k exceeds the document count");
        Check(o.query_capacity >= 1 && o.query_capacity <= 65535, "query_capacity must be in [1, 65535]");
        Check(o.wait_budget_cycles >= 0, "wait_budget_cycles must be >= 0");
        Check(std::isfinite(o.dense_density) && o.dense_density <= 1.0f, "dense_density must be at most 1");
        Check(o.word_capacity >= 0 && o.word_capacity <= 16777216, "word_capacity must be in [0, 2^24]");
        Check(!o.prune || TileFamily(o.kernel), "prune needs the warp-tile or tile-group kernel");
        Cuda(cudaSetDevice(o.device_id), "cudaSetDevice");
        device_ = o.device_id;
        size_t total = 0;
        Cuda(cudaMemGetInfo(&free_at_start_, &total), "cudaMemGetInfo");
        if (o.stream) {
            stream_ = static_cast<cudaStream_t>(o.stream);
        } else {
            Cuda(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
            own_stream_ = true;
        }
        Cuda(cudaEventCreateWithFlags(&done_, cudaEventDisableTiming), "cudaEventCreate");
        MakePlan();
        tuning_.prune_route = o.prune_route;
    }

    ~Engine() { Release(); }

    // Uploads an eager CSC index.
    void UploadEager(const int64_t *indptr, const int32_t *indices, const float *data)
    {
        AllocIndex();
        Cuda(cudaMemcpy(d_indptr_, indptr, (vocab_ + 1) * sizeof(int64_t), cudaMemcpyHostToDevice), "index upload");
        Cuda(cudaMemcpy(d_indices_, indices, postings_ * sizeof(int32_t), cudaMemcpyHostToDevice), "index upload");
        Cuda(cudaMemcpy(d_data_, data, postings_ * sizeof(float), cudaMemcpyHostToDevice), "index upload");
        Finish(indptr);
    }

    // Uploads the reference's lazy index and builds the eager scores on the device.
    void UploadLazy(const int64_t *offsets, const int32_t *docs, const float *tf, const float *norm, const float *idf,
                    float k1)
    {
        Check(std::isfinite(k1) && k1 >= 0, "Invalid k1");
        AllocIndex();
        Cuda(cudaMemcpy(d_indptr_, offsets, (vocab_ + 1) * sizeof(int64_t), cudaMemcpyHostToDevice), "index upload");
        Cuda(cudaMemcpy(d_indices_, docs, postings_ * sizeof(int32_t), cudaMemcpyHostToDevice), "index upload");
        float *d_tf = nullptr, *d_norm = nullptr, *d_idf = nullptr;
        unsigned *d_status = nullptr;
        try {
            Cuda(cudaMalloc(&d_tf, std::max<int64_t>(postings_, 1) * sizeof(float)), "cudaMalloc tf");
            Cuda(cudaMalloc(&d_norm, docs_ * sizeof(float)), "cudaMalloc norm");
            Cuda(cudaMalloc(&d_idf, vocab_ * sizeof(float)), "cudaMalloc idf");
            Cuda(cudaMalloc(&d_status, sizeof(unsigned)), "cudaMalloc status");
            Cuda(cudaMemcpy(d_tf, tf, postings_ * sizeof(float), cudaMemcpyHostToDevice), "index upload");
            Cuda(cudaMemcpy(d_norm, norm, docs_ * sizeof(float), cudaMemcpyHostToDevice), "index upload");
            Cuda(cudaMemcpy(d_idf, idf, vocab_ * sizeof(float), cudaMemcpyHostToDevice), "index upload");
            Cuda(cudaMemset(d_status, 0, sizeof(unsigned)), "cudaMemset");
            // f32(k1 + 1) with the sum in double: k1 = 1.2 gives the reference's 2.2F.
            const float k1p1 = (float)((double)k1 + 1.0);
            if (postings_ > 0) {
                const long long chunks = (postings_ + bm25k::kBuildChunk - 1) / bm25k::kBuildChunk;
                const int grid = (int)std::min<long long>(chunks, 148 * 16);
                bm25k::BuildContributionsKernel<<<grid, 256, 0, stream_>>>(
                    (const long long *)d_indptr_, (int)vocab_, postings_, d_indices_, d_tf, d_norm, d_idf, k1p1,
                    d_data_, d_status);
                Cuda(cudaGetLastError(), "contribution kernel launch");
            }
            unsigned status = 0;
            Cuda(cudaMemcpyAsync(&status, d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_), "status");
            Cuda(cudaStreamSynchronize(stream_), "contribution kernel");
            Check(status == 0, "Posting contribution outside the finite FP32 range");
        } catch (...) {
            cudaFree(d_tf);
            cudaFree(d_norm);
            cudaFree(d_idf);
            cudaFree(d_status);
            throw;
        }
        cudaFree(d_tf);
        cudaFree(d_norm);
        cudaFree(d_idf);
        cudaFree(d_status);
        Finish(offsets);
    }

    void Search(const int64_t *qoffsets, const int32_t *words, int64_t q, int32_t k, float *out_scores,
                int32_t *out_ids)
    {
        RequireUsable();
        Check(out_scores && out_ids, "Null output buffer");
        Pack(qoffsets, words, q, k);  // validates everything before touching the arena
        try {
            Cuda(cudaSetDevice(device_), "cudaSetDevice");
            cudaGraphExec_t exec = GraphFor((int)q, k);
            Cuda(cudaStreamWaitEvent(stream_, done_, 0), "cudaStreamWaitEvent");
            const bool stall = stall_armed_, fail = fail_armed_ || g_fail_next.exchange(0) != 0;
            stall_armed_ = fail_armed_ = false;
            if (stall)
                Cuda(cudaMemsetAsync(d_inject_, 0x01, sizeof(unsigned), stream_), "arm stall");
            ++searches_;
            Cuda(cudaGraphLaunch(exec, stream_), "cudaGraphLaunch");
            ++replays_;
            if (stall)
                Cuda(cudaMemsetAsync(d_inject_, 0, sizeof(unsigned), stream_), "disarm stall");
            Cuda(cudaEventRecord(done_, stream_), "cudaEventRecord");
            Cuda(cudaStreamSynchronize(stream_), "complete Search through result D2H");
            if (fail)
                throw DeviceError(0, "Injected device failure (bm25_test_inject)");
            Receive(q, k, out_scores, out_ids);
        } catch (...) {
            failed_ = true;
            throw;
        }
    }

    void SearchDevice(const int64_t *qoffsets, const int32_t *words, int64_t q, int32_t k, float *out_scores,
                      int32_t *out_ids, cudaStream_t stream)
    {
        RequireUsable();
        Check(q >= 1 && q <= opts_.query_capacity, "Query batch exceeds declared capacity or is empty");
        Check(k >= 1 && k <= opts_.max_k && k <= docs_, "K outside [1, min(max_k, N)]");
        Check(qoffsets && words && out_scores && out_ids, "Null device buffer");
        try {
            Cuda(cudaSetDevice(device_), "cudaSetDevice");
            cudaStream_t s = stream ? stream : stream_;
            Cuda(cudaStreamWaitEvent(s, done_, 0), "cudaStreamWaitEvent");
            ++searches_;
            marking_ = !timing_.empty();
            Launch((int)q, k, qoffsets, words, out_scores, out_ids, d_dev_status_, s);
            if (marking_)
                ++timed_;
            marking_ = false;
            Cuda(cudaEventRecord(done_, s), "cudaEventRecord");
        } catch (...) {
            failed_ = true;
            throw;
        }
    }

    // Pruned Search on device buffers: tau [q] starting bounds (nullptr: learned bounds),
    // out_exact [q] flags; queries whose bound proved too high are answered by the retry pass.
    void SearchPrunedDevice(const int64_t *qoffsets, const int32_t *words, const float *tau, int64_t q, int32_t k,
                            float *out_scores, int32_t *out_ids, int32_t *out_exact, cudaStream_t stream)
    {
        RequireUsable();
        RequirePrune();
        Check(q >= 1 && q <= opts_.query_capacity, "Query batch exceeds declared capacity or is empty");
        Check(k >= 1 && k <= opts_.max_k && k <= docs_, "K outside [1, min(max_k, N)]");
        Check(qoffsets && words && out_scores && out_ids && out_exact, "Null device buffer");
        try {
            Cuda(cudaSetDevice(device_), "cudaSetDevice");
            cudaStream_t s = stream ? stream : stream_;
            Cuda(cudaStreamWaitEvent(s, done_, 0), "cudaStreamWaitEvent");
            ++searches_;
            marking_ = !timing_.empty();
            Launch((int)q, k, qoffsets, words, out_scores, out_ids, d_dev_status_, s, tau ? tau : d_tau_, out_exact,
                   tau == nullptr);
            if (marking_)
                ++timed_;
            marking_ = false;
            Cuda(cudaEventRecord(done_, s), "cudaEventRecord");
        } catch (...) {
            failed_ = true;
            throw;
        }
    }

    // Pruned Search on host buffers: one graph replay (H2D, pruned Search, retry pass, D2H).
    // out_exact[i] = 1 where the pruned result stood, 0 where the retry pass answered.
    // tau == nullptr: the starting bounds come from the learned-bound kernel (the session's
    // threshold model, or the safe bounds alone without one).
    void SearchPruned(const int64_t *qoffsets, const int32_t *words, const float *tau, int64_t q, int32_t k,
                      float *out_scores, int32_t *out_ids, int32_t *out_exact)
    {
        RequireUsable();
        RequirePrune();
        Check(out_scores && out_ids && out_exact, "Null buffer");
        Pack(qoffsets, words, q, k);
        if (tau)
            std::memcpy(static_cast<unsigned char *>(h_in_) + tau_offset_, tau, q * sizeof(float));
        try {
            Cuda(cudaSetDevice(device_), "cudaSetDevice");
            cudaGraphExec_t exec = GraphFor((int)q, k, tau ? kModePruned : kModeLearned);
            Cuda(cudaStreamWaitEvent(stream_, done_, 0), "cudaStreamWaitEvent");
            ++searches_;
            Cuda(cudaGraphLaunch(exec, stream_), "cudaGraphLaunch");
            ++replays_;
            Cuda(cudaEventRecord(done_, stream_), "cudaEventRecord");
            Cuda(cudaStreamSynchronize(stream_), "complete pruned Search through result D2H");
            Receive(q, k, out_scores, out_ids);
        } catch (...) {
            failed_ = true;
            throw;
        }
        const int32_t *exact =
            reinterpret_cast<const int32_t *>(static_cast<const unsigned char *>(h_out_) + ExactOffset((int)q, k));
        for (int64_t i = 0; i < q; ++i)
            out_exact[i] = exact[i] ? 1 : 0;
    }

    // A batch with a K per query (host buffers): results packed by query, query i's ks[i] rows from
    // the sum of the K before it.  learned: starting bounds from the learned-bound kernel, out_exact
    // as in SearchPruned.
    void SearchBatch(const int64_t *qoffsets, const int32_t *words, const int32_t *ks, int64_t q, bool learned,
                     float *out_scores, int32_t *out_ids, int32_t *out_exact)
    {
        RequireUsable();
        if (learned)
            RequirePrune();
        Check(TileFamily(plan_.kernel), "A K per query needs the warp-tile or tile-group kernel");
        Check(ks && out_scores && out_ids && (!learned || out_exact), "Null buffer");
        Check(q >= 1 && q <= opts_.query_capacity, "Query batch exceeds declared capacity or is empty");
        int kmax = 1;
        for (int64_t i = 0; i < q; ++i) {
            Check(ks[i] >= 1 && ks[i] <= opts_.max_k && ks[i] <= docs_, "K outside [1, min(max_k, N)]");
            kmax = std::max(kmax, ks[i]);
        }
        Check(qoffsets != nullptr, "Null query offsets");
        // The batch runs in the graph of its capacity bucket (queries rounded up to a power of two,
        // the largest K up to 32, 128 or 1024): the extra queries are empty with K = 1 and their
        // results come after the real ones, so a few graphs serve every batch a server forms.
        const int qb = BatchBucket((int)q), kb = KBucket(kmax);
        std::vector<int64_t> offsets(qoffsets, qoffsets + q + 1);
        offsets.resize((size_t)qb + 1, qoffsets[q]);
        std::vector<int32_t> kpad(ks, ks + q);
        kpad.resize((size_t)qb, 1);
        std::vector<int64_t> kout(qb);
        int64_t total = 0;
        for (int i = 0; i < qb; ++i) {
            kout[i] = total;
            total += kpad[i];
        }
        total = kout[q - 1] + ks[q - 1];  // the real queries' results
        Pack(offsets.data(), words, qb, kb);
        unsigned char *in = static_cast<unsigned char *>(h_in_);
        std::memcpy(in + ks_offset_, kpad.data(), (size_t)qb * sizeof(int32_t));
        std::memcpy(in + kout_offset_, kout.data(), (size_t)qb * sizeof(int64_t));
        kmax = kb;
        try {
            Cuda(cudaSetDevice(device_), "cudaSetDevice");
            cudaGraphExec_t exec = GraphFor(qb, kmax, (learned ? kModeLearned : kModePlain) | kModeMixed);
            Cuda(cudaStreamWaitEvent(stream_, done_, 0), "cudaStreamWaitEvent");
            ++searches_;
            Cuda(cudaGraphLaunch(exec, stream_), "cudaGraphLaunch");
            ++replays_;
            unsigned char *ho = static_cast<unsigned char *>(h_out_);
            // the status word and the scores in one copy, then the ids (and the flags)
            Cuda(cudaMemcpyAsync(ho, d_out_, kScoreOffset + total * sizeof(float), cudaMemcpyDeviceToHost, stream_),
                 "D2H");
            const size_t ids = IdOffset(qb, kmax);
            Cuda(cudaMemcpyAsync(ho + ids, d_out_ + ids, total * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_),
                 "D2H");
            if (learned) {
                const size_t ex = ExactOffset(qb, kmax);
                Cuda(cudaMemcpyAsync(ho + ex, d_out_ + ex, (size_t)q * 4, cudaMemcpyDeviceToHost, stream_), "D2H");
            }
            Cuda(cudaEventRecord(done_, stream_), "cudaEventRecord");
            Cuda(cudaStreamSynchronize(stream_), "complete batch Search through result D2H");
            unsigned status = 0;
            std::memcpy(&status, ho, sizeof(unsigned));
            if (status)
                throw DeviceError(0, "Device reported invalid Search state, status=" + std::to_string(status));
            const float *scores = reinterpret_cast<const float *>(ho + kScoreOffset);
            const int32_t *idv = reinterpret_cast<const int32_t *>(ho + ids);
            for (int64_t i = 0; i < q; ++i)
                for (int64_t r = kout[i]; r < kout[i] + ks[i]; ++r) {
                    if (!(idv[r] >= 0 && idv[r] < docs_ && std::isfinite(scores[r]) && scores[r] >= 0))
                        throw DeviceError(0, "Invalid real-document result");
                    if (r > kout[i] && !(scores[r - 1] > scores[r] || (scores[r - 1] == scores[r] && idv[r - 1] < idv[r])))
                        throw DeviceError(0, "Strict global ranking failure");
                }
            std::memcpy(out_scores, scores, total * sizeof(float));
            std::memcpy(out_ids, idv, total * sizeof(int32_t));
            if (learned) {
                const int32_t *ex = reinterpret_cast<const int32_t *>(ho + ExactOffset(qb, kmax));
                for (int64_t i = 0; i < q; ++i)
                    out_exact[i] = ex[i] ? 1 : 0;
            }
        } catch (...) {
            failed_ = true;
            throw;
        }
    }

    // Device-resident batch with a K per query: ks [q], kout [q] (first output slot of each query,
    // rows packed), kmax >= every ks[i]; learned: learned bounds and out_exact [q].
    void SearchBatchDevice(const int64_t *qoffsets, const int32_t *words, const int32_t *ks, const int64_t *kout,
                           int64_t q, int32_t kmax, bool learned, float *out_scores, int32_t *out_ids,
                           int32_t *out_exact, cudaStream_t stream)
    {
        RequireUsable();
        if (learned)
            RequirePrune();
        Check(TileFamily(plan_.kernel), "A K per query needs the warp-tile or tile-group kernel");
        Check(q >= 1 && q <= opts_.query_capacity, "Query batch exceeds declared capacity or is empty");
        Check(kmax >= 1 && kmax <= opts_.max_k && kmax <= docs_, "K outside [1, min(max_k, N)]");
        Check(qoffsets && words && ks && kout && out_scores && out_ids && (!learned || out_exact), "Null device buffer");
        try {
            Cuda(cudaSetDevice(device_), "cudaSetDevice");
            cudaStream_t s = stream ? stream : stream_;
            Cuda(cudaStreamWaitEvent(s, done_, 0), "cudaStreamWaitEvent");
            ++searches_;
            marking_ = !timing_.empty();
            Launch((int)q, kmax, qoffsets, words, out_scores, out_ids, d_dev_status_, s, learned ? d_tau_ : nullptr,
                   learned ? out_exact : nullptr, learned, ks, kout);
            if (marking_)
                ++timed_;
            marking_ = false;
            Cuda(cudaEventRecord(done_, s), "cudaEventRecord");
        } catch (...) {
            failed_ = true;
            throw;
        }
    }

    // Runtime tuning (bm25_set_tuning): validated, applied to the launch parameters, and the
    // instantiated graphs (which hold the old ones by value) dropped.
    void GetTuning(bm25_tuning *t) const
    {
        *t = tuning_;
        t->ring_stages = plan_.stages;
        t->ring_chunk = plan_.chunk;
    }
    void SetTuning(const bm25_tuning &t)
    {
        RequireUsable();
        Check(t.claim_tiles == 2 || t.claim_tiles == 4 || t.claim_tiles == 8, "claim_tiles must be 2, 4 or 8");
        Check(t.tail_claims >= 0 && t.tail_claims <= 8, "tail_claims must be in [0, 8]");
        Check(std::isfinite(t.prune_route), "prune_route must be finite");
        const bool ring = TileFamily(plan_.kernel);
        int stages = plan_.stages, chunk = plan_.chunk;
        if (ring) {
            Check(t.ring_stages >= 2 && t.ring_stages <= bm25k::kMaxStages, "ring_stages must be in [2, 8]");
            Check(t.ring_chunk >= bm25k::kWgChunkMin && t.ring_chunk <= bm25k::kWgChunkMax && t.ring_chunk % 4 == 0,
                  "ring_chunk must be a multiple of 4 in [512, 4096]");
            stages = t.ring_stages;
            chunk = t.ring_chunk;
        }
        long long cap = 0;
        if (opts_.max_k > bm25k::kMaxSmallK && t.candidate_cap != 0) {
            // the retry passes start from a bound that may sit below the K-th score (the running bounds
            // of concurrent warps), so the buffer keeps some slack over K: at least 8 max_k and 2048
            cap = (t.candidate_cap + 3) & ~3LL;
            const long long least = std::min<long long>(cand_cap_, std::max<long long>(2048, 8LL * opts_.max_k));
            Check(cap >= least && cap <= cand_cap_,
                  "candidate_cap must be in [max(2048, 8 max_k), candidate_capacity]");
        }
        Cuda(cudaSetDevice(device_), "cudaSetDevice");
        size_t tg_smem = tg_smem_;
        int tg_grid = tg_grid_;
        if (ring && (stages != plan_.stages || chunk != plan_.chunk)) {
            tg_smem = bm25k::TileGroupSmem(stages, chunk, plan_.tile_docs);
            const void *kernel = bm25k::TileGroupKernelFor(plan_.tile_docs);
            int per_sm = 0;
            RaiseSmemCap(kernel, tg_smem);
            RaiseSmemCap(bm25k::TileGroupKernelFor(plan_.tile_docs, true), tg_smem);
            Cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, bm25k::kWgThreads, tg_smem),
                 "occupancy");
            Check(per_sm >= 1, "ring_stages x ring_chunk exceed the shared memory of one SM");
            tg_grid = per_sm * sms_;
        }
        Cuda(cudaStreamWaitEvent(stream_, done_, 0), "cudaStreamWaitEvent");
        Cuda(cudaStreamSynchronize(stream_), "tuning");
        for (auto &g : graphs_)
            cudaGraphExecDestroy(g.second.exec);
        graphs_.clear();
        tuning_ = t;
        tuning_.candidate_cap = cap;
        plan_.stages = stages;
        plan_.chunk = chunk;
        if (ring) {
            tg_smem_ = tg_smem;
            tg_grid_ = tg_grid;
            if (plan_.kernel == BM25_KERNEL_TILE_GROUP) {
                smem_bytes_ = tg_smem;
                plan_.grid = tg_grid;
            }
        }
    }

    // Capacity buckets of bm25_search_batch's graphs.
    int BatchBucket(int q) const
    {
        int b = 1;
        while (b < q)
            b <<= 1;
        return (int)std::min<int64_t>(b, opts_.query_capacity);
    }
    int KBucket(int kmax) const
    {
        const int cap = (int)std::min<int64_t>(opts_.max_k, docs_);
        for (const int b : {32, 128, 1024})
            if (kmax <= b && b <= cap)
                return b;
        return cap;
    }

    // Instantiates every graph bm25_search_batch (learned or plain) replays for batches of up to
    // max_batch queries, so that none is instantiated on a serving loop's request path.
    void PrepareBatchGraphs(int max_batch, bool learned)
    {
        RequireUsable();
        if (learned)
            RequirePrune();
        Check(TileFamily(plan_.kernel), "A K per query needs the warp-tile or tile-group kernel");
        Check(max_batch >= 1 && max_batch <= opts_.query_capacity, "max_batch must be in [1, query_capacity]");
        Cuda(cudaSetDevice(device_), "cudaSetDevice");
        std::vector<int> kbs;
        for (const int k : {1, 33, 129})
            if (k <= std::min<int64_t>(opts_.max_k, docs_) && (kbs.empty() || KBucket(k) != kbs.back()))
                kbs.push_back(KBucket(k));
        const int top = BatchBucket(max_batch);
        for (int qb = 1;; qb = std::min(qb * 2, top)) {
            for (const int kb : kbs)
                (void)GraphFor(qb, kb, (learned ? kModeLearned : kModePlain) | kModeMixed);
            if (qb == top)
                break;
        }
    }

    // Threshold model of the learned bounds (host params, bm25mlp::kParams floats), or none.
    void SetThresholdModel(const float *params, float margin)
    {
        RequireUsable();
        RequirePrune();
        Check(!params || std::isfinite(margin), "margin must be finite");
        if (params)
            for (int i = 0; i < bm25mlp::kParams; ++i)
                Check(std::isfinite(params[i]), "Threshold model holds a non-finite parameter");
        Cuda(cudaSetDevice(device_), "cudaSetDevice");
        Cuda(cudaStreamWaitEvent(stream_, done_, 0), "cudaStreamWaitEvent");
        Cuda(cudaStreamSynchronize(stream_), "model update");
        if (params)
            Cuda(cudaMemcpy(d_model_, params, bm25mlp::kParams * sizeof(float), cudaMemcpyHostToDevice),
                 "model upload");
        has_model_ = params != nullptr;
        margin_ = params ? margin : 0.0f;
        // graphs hold the model pointer and margin by value: rebuild the learned ones
        for (auto it = graphs_.begin(); it != graphs_.end();) {
            if (std::get<2>(it->first) & kModeLearned) {
                cudaGraphExecDestroy(it->second.exec);
                it = graphs_.erase(it);
            } else {
                ++it;
            }
        }
    }

    // Query features [q][32] and safe bounds [q] on device buffers (training data of the model).
    void QueryFeaturesDevice(const int64_t *qoffsets, const int32_t *words, int64_t q, int32_t k, float *features,
                             float *safe, cudaStream_t stream)
    {
        RequireUsable();
        RequirePrune();
        Check(q >= 1 && q <= opts_.query_capacity, "Query batch exceeds declared capacity or is empty");
        Check(k >= 1 && k <= opts_.max_k && k <= docs_, "K outside [1, min(max_k, N)]");
        Check(qoffsets && words && features, "Null device buffer");
        Cuda(cudaSetDevice(device_), "cudaSetDevice");
        cudaStream_t s = stream ? stream : stream_;
        Cuda(cudaStreamWaitEvent(s, done_, 0), "cudaStreamWaitEvent");
        bm25k::LearnedArgs la = LearnedArgsFor((int)q, k, qoffsets, words);
        la.features = features;
        la.safe = safe;
        bm25k::QueryFeaturesKernel<<<(int)((q + 7) / 8), 256, 0, s>>>(la);
        Cuda(cudaGetLastError(), "feature kernel launch");
        Cuda(cudaEventRecord(done_, s), "cudaEventRecord");
    }

    // Search counters since the last reset (bm25_search_stats).
    void SearchStats(uint64_t *out, bool reset)
    {
        RequireUsable();
        Check(out != nullptr, "Null output");
        Cuda(cudaSetDevice(device_), "cudaSetDevice");
        Cuda(cudaStreamWaitEvent(stream_, done_, 0), "cudaStreamWaitEvent");
        Cuda(cudaStreamSynchronize(stream_), "stats");
        if (!d_stats_) {
            std::memset(out, 0, bm25k::kStats * sizeof(uint64_t));
            return;
        }
        Cuda(cudaMemcpy(out, d_stats_, bm25k::kStats * sizeof(uint64_t), cudaMemcpyDeviceToHost), "stats D2H");
        if (reset)
            Cuda(cudaMemset(d_stats_, 0, bm25k::kStats * sizeof(uint64_t)), "stats reset");
    }

    bm25k::LearnedArgs LearnedArgsFor(int q, int k, const int64_t *qoffsets, const int32_t *words) const
    {
        bm25k::LearnedArgs la{};
        la.indptr = (const long long *)d_indptr_;
        la.top = d_term_top_;
        la.rank = d_term_rank_;
        la.mean = d_term_mean_;
        la.vocab = (int)vocab_;
        la.qoffsets = (const long long *)qoffsets;
        la.words = words;
        la.q = q;
        la.k = k;
        la.word_cap = std::max<int64_t>(1, opts_.word_capacity);
        la.params = has_model_ ? d_model_ : nullptr;
        la.margin = margin_;
        la.tau = d_tau_;
        return la;
    }

    // Event timing of the main search kernel (StreamSearchKernel or
    // TileSearchKernel) for device-resident Searches: a ring of event pairs
    // recorded on the launching stream around that one launch.
    void KernelTiming(bool enable)
    {
        RequireUsable();
        Cuda(cudaSetDevice(device_), "cudaSetDevice");
        if (enable && timing_.empty()) {
            timing_.resize(2 * kTimingRing);
            for (auto &e : timing_)
                Cuda(cudaEventCreate(&e), "cudaEventCreate");
        } else if (!enable) {
            Cuda(cudaStreamWaitEvent(stream_, done_, 0), "cudaStreamWaitEvent");
            Cuda(cudaStreamSynchronize(stream_), "timing drain");
            DestroyTiming();
        }
        timed_ = 0;
    }

    int64_t KernelTimes(float *ms, int64_t capacity)
    {
        RequireUsable();
        Check(!timing_.empty(), "Kernel timing is not enabled");
        Check(ms != nullptr || capacity == 0, "Null output");
        Cuda(cudaSetDevice(device_), "cudaSetDevice");
        const int64_t n = std::min<int64_t>(timed_, kTimingRing);
        const int64_t first = timed_ - n;
        int64_t out = 0;
        for (int64_t i = first; i < timed_ && out < capacity; ++i) {
            const size_t slot = (size_t)(i % kTimingRing);
            Cuda(cudaEventSynchronize(timing_[2 * slot + 1]), "cudaEventSynchronize");
            Cuda(cudaEventElapsedTime(&ms[out++], timing_[2 * slot], timing_[2 * slot + 1]), "cudaEventElapsedTime");
        }
        timed_ = 0;
        return out;
    }

    // Test hook (bm25_test_inject): one-shot failure of the next host-buffer Search.
    void Inject(int what)
    {
        RequireUsable();
        Check(what == BM25_INJECT_HOST_FAILURE || what == BM25_INJECT_STALL, "Unknown injection");
        if (what == BM25_INJECT_HOST_FAILURE)
            fail_armed_ = true;
        else
            stall_armed_ = true;
    }

    uint32_t DeviceStatus()
    {
        RequireUsable();
        unsigned status = 0;
        try {
            Cuda(cudaSetDevice(device_), "cudaSetDevice");
            Cuda(cudaStreamWaitEvent(stream_, done_, 0), "cudaStreamWaitEvent");
            Cuda(cudaMemcpyAsync(&status, d_dev_status_, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_),
                 "status D2H");
            Cuda(cudaMemsetAsync(d_dev_status_, 0, sizeof(unsigned), stream_), "status reset");
            Cuda(cudaStreamSynchronize(stream_), "status sync");
        } catch (...) {
            failed_ = true;
            throw;
        }
        return status;
    }

    void Close()
    {
        if (closed_)
            return;
        Cuda(cudaSetDevice(device_), "cudaSetDevice");
        Cuda(cudaStreamSynchronize(stream_), "drain before close");
        Release();
        closed_ = true;
    }

    void Info(bm25_info *info) const
    {
        info->num_docs = docs_;
        info->vocab = vocab_;
        info->postings = postings_;
        info->tile_docs = plan_.tile_docs;
        info->tiles = plan_.tiles;
        info->merge_fan_in = plan_.fan_in;
        info->merge_levels = plan_.levels;
        info->directory_rows = plan_.dir_rows;
        info->directory_min_df = plan_.dir_min_df;
        info->index_bytes = index_bytes_;
        info->device_bytes = device_bytes_;
        info->graph_replays = replays_;
        info->searches = searches_;
        info->kernel = plan_.kernel;
        info->ring_stages = plan_.stages;
        info->ring_chunk = plan_.chunk;
        info->grid = plan_.grid;
        info->smem_bytes = (int32_t)smem_bytes_;
        info->query_capacity = opts_.query_capacity;
        info->word_capacity = opts_.word_capacity;
        info->max_k = opts_.max_k;
        info->prune = opts_.prune ? 1 : 0;
        info->graph_instantiations = instantiations_;
        info->graphs_cached = (int64_t)graphs_.size();
        info->dense_rows = dense_rows_;
    }

  private:
    void RequirePrune() const
    {
        if (!opts_.prune || !TileFamily(plan_.kernel))
            throw InvalidState("Pruned Search needs a session created with prune = 1 and the warp-tile or tile-group "
                               "kernel");
    }

    void RequireUsable() const
    {
        if (closed_ || failed_)
            throw InvalidState(closed_ ? "BM25 session is closed" : "BM25 session failed; Close and re-create it");
    }

    void *Alloc(size_t bytes, const char *what)
    {
        void *p = nullptr;
        Cuda(cudaMalloc(&p, std::max<size_t>(bytes, 16)), what);
        allocations_.push_back(p);
        device_bytes_ += (int64_t)bytes;
        return p;
    }

    void MakePlan()
    {
        Check(opts_.kernel == BM25_KERNEL_STREAM || opts_.kernel == BM25_KERNEL_PER_TILE ||
                  TileFamily(opts_.kernel),
              "kernel must be 0 (streaming), 1 (per-tile), 4 (tile groups) or 5 (warp tiles)");
        plan_.kernel = opts_.kernel;
        int t = opts_.tile_docs;
        if (plan_.kernel == BM25_KERNEL_WARP_TILE) {
            Check(t == 0 || t == bm25k::kWtTile, "tile_docs of the warp-tile kernel must be 1024");
            Check(postings_ + kPad < INT32_MAX, "Posting count exceeds the INT32 contract");
            t = bm25k::kWtTile;
        } else if (plan_.kernel == BM25_KERNEL_TILE_GROUP) {
            Check(t == 0 || t == 1024 || t == 2048, "tile_docs of the tile-group kernel must be 1024 or 2048");
            Check(postings_ + kPad < INT32_MAX, "Posting count exceeds the INT32 contract");
            t = t ? t : bm25k::kWgTileDocs;
        } else if (t == 0) {
            const int64_t per_sm = (docs_ + 147) / 148;
            t = 2048;
            while (t < per_sm && t < (plan_.kernel == 0 ? 8192 : 16384))
                t <<= 1;
        }
        Check(TileFamily(plan_.kernel) || (t >= 2048 && t <= 32768 && (t & (t - 1)) == 0),
              "tile_docs must be a power of two in [2048, 32768]");
        plan_.tile_docs = t;
        plan_.tiles = (int)((docs_ + t - 1) / t);
        Check((int64_t)plan_.tiles * opts_.query_capacity < (int64_t(1) << 31),
              "query_capacity x tiles exceeds the work counter");
        int f = opts_.merge_fan_in ? opts_.merge_fan_in : 32;
        Check(f >= 2 && f <= 1024, "merge_fan_in must be in [2, 1024]");
        for (;;) {
            plan_.lists.clear();
            int n = plan_.tiles;
            plan_.lists.push_back(n);
            while (n > 1) {
                n = (n + f - 1) / f;
                plan_.lists.push_back(n);
            }
            if ((int)plan_.lists.size() <= bm25k::kMaxLevels)
                break;
            f *= 2;
        }
        plan_.fan_in = f;
        plan_.levels = (int)plan_.lists.size();
        if (plan_.kernel != 1) {
            // tile-group kernel: 3 stages of 1536 postings keep 3 CTAs on an SM (measured best at 10M docs)
            // (the warp-tile kernel has no ring; its pruned Searches stream with the tile-group kernel)
            const int st = opts_.ring_stages ? opts_.ring_stages : (TileFamily(plan_.kernel) ? 3 : 4);
            Check(st >= 2 && st <= bm25k::kMaxStages, "ring_stages must be in [2, 8]");
            plan_.stages = st;
            if (TileFamily(plan_.kernel)) {
                const int c = opts_.ring_chunk ? opts_.ring_chunk : 1536;
                Check(c >= bm25k::kWgChunkMin && c <= bm25k::kWgChunkMax && c % 4 == 0,
                      "ring_chunk must be a multiple of 4 in [512, 4096]");
                plan_.chunk = c;
            }
        }
    }

    void AllocIndex()
    {
        d_indptr_ = static_cast<int64_t *>(Alloc((vocab_ + 1) * sizeof(int64_t), "cudaMalloc indptr"));
        d_indices_ = static_cast<int32_t *>(Alloc((postings_ + kPad) * sizeof(int32_t), "cudaMalloc indices"));
        d_data_ = static_cast<float *>(Alloc((postings_ + kPad) * sizeof(float), "cudaMalloc data"));
        Cuda(cudaMemset(d_indices_ + postings_, 0, kPad * sizeof(int32_t)), "cudaMemset pad");
        Cuda(cudaMemset(d_data_ + postings_, 0, kPad * sizeof(float)), "cudaMemset pad");
        index_bytes_ = (vocab_ + 1) * 8 + postings_ * 8;
    }

    // Directory, arenas, merge-tree storage and kernel attributes.
    void Finish(const int64_t *indptr)
    {
        const int tiles = plan_.tiles;
        // Long lists (df >= min_df) get one directory row of tiles + 1 offsets;
        // shorter lists are counted cooperatively inside the tile CTA.
        std::vector<int64_t> dfs(vocab_);
        for (int64_t t = 0; t < vocab_; ++t)
            dfs[t] = indptr[t + 1] - indptr[t];
        int64_t min_df = std::max<int64_t>(32, tiles);
        const int64_t row_bytes = (int64_t)(tiles + 1) * 4;
        int64_t budget = opts_.directory_bytes;
        if (budget <= 0)
            budget = std::max<int64_t>(int64_t(64) << 20, std::min<int64_t>(int64_t(4) << 30, index_bytes_ / 4));
        int64_t rows = 0;
        for (int64_t t = 0; t < vocab_; ++t)
            rows += dfs[t] >= min_df;
        if (rows * row_bytes > budget) {
            std::vector<int64_t> sorted(dfs);
            const int64_t keep = std::max<int64_t>(0, budget / row_bytes);
            std::nth_element(sorted.begin(), sorted.begin() + keep, sorted.end(), std::greater<int64_t>());
            min_df = sorted[keep] + 1;
            rows = 0;
            for (int64_t t = 0; t < vocab_; ++t)
                rows += dfs[t] >= min_df;
        }
        plan_.dir_min_df = min_df;
        plan_.dir_rows = rows;
        std::vector<int32_t> dir_row(vocab_, -1), dir_terms;
        dir_terms.reserve(rows);
        for (int64_t t = 0; t < vocab_; ++t)
            if (dfs[t] >= min_df) {
                dir_row[t] = (int32_t)dir_terms.size();
                dir_terms.push_back((int32_t)t);
            }
        d_dir_row_ = static_cast<int32_t *>(Alloc(vocab_ * sizeof(int32_t), "cudaMalloc dir_row"));
        Cuda(cudaMemcpy(d_dir_row_, dir_row.data(), vocab_ * sizeof(int32_t), cudaMemcpyHostToDevice), "dir upload");
        d_dir_ = static_cast<int32_t *>(Alloc(std::max<int64_t>(rows, 1) * row_bytes, "cudaMalloc directory"));
        if (rows > 0) {
            int32_t *d_terms = static_cast<int32_t *>(Alloc(rows * sizeof(int32_t), "cudaMalloc dir terms"));
            Cuda(cudaMemcpy(d_terms, dir_terms.data(), rows * sizeof(int32_t), cudaMemcpyHostToDevice), "dir upload");
            const long long total = rows * (long long)(tiles + 1);
            const int grid = (int)std::min<long long>((total + 255) / 256, 148 * 64);
            bm25k::BuildDirectoryKernel<<<grid, 256, 0, stream_>>>((const long long *)d_indptr_, d_indices_, d_terms,
                                                                   rows, plan_.tile_docs, tiles, d_dir_, tiles + 1);
            Cuda(cudaGetLastError(), "directory kernel launch");
            if (opts_.prune) {
                // 128-document block index of the directory rows: offsets (uint16) and maxima
                const size_t cells = (size_t)rows * tiles * (plan_.tile_docs / bm25k::kBlockDocs);
                d_boff_ = static_cast<unsigned short *>(Alloc(cells * sizeof(unsigned short), "cudaMalloc block offsets"));
                d_bmax_ = static_cast<__half *>(Alloc(cells * sizeof(__half), "cudaMalloc block maxima"));
                const long long pairs = rows * (long long)tiles;
                bm25k::BuildBlockIndexKernel<<<(int)std::min<long long>((pairs + 255) / 256, 148 * 64), 256, 0,
                                               stream_>>>((const long long *)d_indptr_, d_indices_, d_data_, d_terms,
                                                          d_dir_, rows, tiles, tiles + 1, plan_.tile_docs, d_boff_,
                                                          d_bmax_);
                Cuda(cudaGetLastError(), "block index kernel launch");
            }
            Cuda(cudaStreamSynchronize(stream_), "directory kernel");
        }
        if (plan_.kernel == BM25_KERNEL_WARP_TILE && opts_.dense_density >= 0.0f)
            BuildDense(dfs);
        if (opts_.prune || plan_.kernel == BM25_KERNEL_WARP_TILE) {
            // per-term statistics: the 32 largest posting scores (the warp-tile kernel's starting
            // bounds; the learned bounds' features) and the mean posting score
            d_term_top_ = static_cast<float *>(Alloc(vocab_ * bm25k::kTermTop * sizeof(float), "cudaMalloc term top"));
            d_term_mean_ = static_cast<float *>(Alloc(vocab_ * sizeof(float), "cudaMalloc term mean"));
            const int grid = (int)std::min<long long>((vocab_ + 7) / 8, 148 * 16);
            bm25k::TermStatsKernel<<<grid, 256, 0, stream_>>>((const long long *)d_indptr_, d_data_, vocab_,
                                                               d_term_top_, d_term_mean_);
            Cuda(cudaGetLastError(), "term statistics kernel launch");
            if (plan_.kernel == BM25_KERNEL_WARP_TILE) {
                // scores at ranks 64 .. 1024 of every term with more than 32 postings: the warp-tile
                // kernel's starting bounds for K above 32
                d_term_rank_ = static_cast<float *>(Alloc(vocab_ * bm25k::kRankCount * sizeof(float),
                                                          "cudaMalloc term ranks"));
                Cuda(cudaMemsetAsync(d_term_rank_, 0, vocab_ * bm25k::kRankCount * sizeof(float), stream_),
                     "cudaMemset term ranks");
                std::vector<int32_t> long_terms;
                for (int64_t t = 0; t < vocab_; ++t)
                    if (dfs[t] > 32)
                        long_terms.push_back((int32_t)t);
                if (!long_terms.empty()) {
                    int32_t *d_lt = static_cast<int32_t *>(Alloc(long_terms.size() * sizeof(int32_t),
                                                                 "cudaMalloc rank terms"));
                    Cuda(cudaMemcpy(d_lt, long_terms.data(), long_terms.size() * sizeof(int32_t),
                                    cudaMemcpyHostToDevice),
                         "rank terms upload");
                    bm25k::TermRanksKernel<<<(int)std::min<size_t>(long_terms.size(), 148 * 4), bm25k::kLargeThreads,
                                             0, stream_>>>((const long long *)d_indptr_, d_data_, d_lt,
                                                           (int)long_terms.size(), d_term_rank_);
                    Cuda(cudaGetLastError(), "term rank kernel launch");
                }
            }
            Cuda(cudaStreamSynchronize(stream_), "term statistics kernel");
        }
        if (opts_.prune) {
            item_cap_ = (long long)opts_.query_capacity * tiles;
            d_items_ = static_cast<uint4 *>(Alloc(item_cap_ * sizeof(uint4), "cudaMalloc block work list"));
            d_wrow_ = static_cast<int *>(Alloc(std::max<size_t>(1, opts_.word_capacity) * sizeof(int),
                                               "cudaMalloc word rows"));
            d_item_count_ = static_cast<unsigned *>(Alloc(4 * sizeof(unsigned), "cudaMalloc block work count"));
            d_safe_ = static_cast<float *>(Alloc(opts_.query_capacity * sizeof(float), "cudaMalloc safe bounds"));
            d_model_ = static_cast<float *>(Alloc(bm25mlp::kParams * sizeof(float), "cudaMalloc model"));
            d_tau_ = static_cast<float *>(Alloc(opts_.query_capacity * sizeof(float), "cudaMalloc tau"));
        }
        // Query packet / result arenas (fixed_query_packet.h:15-25 layout).
        word_offset_ = Align32((opts_.query_capacity + 1) * sizeof(int64_t));
        tau_offset_ = Align32(word_offset_ + std::max<int64_t>(1, opts_.word_capacity) * sizeof(int32_t));
        ks_offset_ = tau_offset_ + (opts_.prune ? Align32(opts_.query_capacity * sizeof(float)) : 0);
        kout_offset_ = ks_offset_ + Align32(opts_.query_capacity * sizeof(int32_t));
        in_bytes_ = kout_offset_ + Align32(opts_.query_capacity * sizeof(int64_t));
        const size_t qk = (size_t)opts_.query_capacity * opts_.max_k;
        out_bytes_ = Align32(qk * 4) * 2 + 32 + Align32(opts_.query_capacity * sizeof(int32_t));
        Cuda(cudaHostAlloc(&h_in_, in_bytes_, cudaHostAllocDefault), "cudaHostAlloc");
        Cuda(cudaHostAlloc(&h_out_, out_bytes_, cudaHostAllocDefault), "cudaHostAlloc");
        std::memset(h_in_, 0, in_bytes_);
        d_in_ = static_cast<unsigned char *>(Alloc(in_bytes_, "cudaMalloc input arena"));
        d_out_ = static_cast<unsigned char *>(Alloc(out_bytes_, "cudaMalloc output arena"));
        Cuda(cudaMemset(d_out_, 0, out_bytes_), "cudaMemset output arena");  // the status word starts 0
        d_dev_status_ = static_cast<unsigned *>(Alloc(sizeof(unsigned), "cudaMalloc status"));
        Cuda(cudaMemset(d_dev_status_, 0, sizeof(unsigned)), "cudaMemset");
        d_inject_ = static_cast<unsigned *>(Alloc(sizeof(unsigned), "cudaMalloc inject word"));
        Cuda(cudaMemset(d_inject_, 0, sizeof(unsigned)), "cudaMemset");
        // Merge tree of the per-tile kernel: level 0 holds tile lists, the root level is the output.
        for (int l = 0; l < plan_.levels && plan_.kernel == 1; ++l) {
            bm25k::Level lv{};
            lv.n = plan_.lists[l];
            if (lv.n > 1) {
                const size_t nodes = (size_t)opts_.query_capacity * lv.n;
                lv.scores = static_cast<float *>(Alloc(nodes * opts_.max_k * sizeof(float), "cudaMalloc tree"));
                lv.ids = static_cast<int *>(Alloc(nodes * opts_.max_k * sizeof(int), "cudaMalloc tree"));
                lv.counts = static_cast<int *>(Alloc(nodes * sizeof(int), "cudaMalloc tree"));
            }
            if (l > 0) {
                const size_t nodes = (size_t)opts_.query_capacity * lv.n;
                lv.arrivals = static_cast<unsigned *>(Alloc(nodes * sizeof(unsigned), "cudaMalloc arrivals"));
                Cuda(cudaMemset(lv.arrivals, 0, nodes * sizeof(unsigned)), "cudaMemset arrivals");
            }
            levels_.push_back(lv);
        }
        if (plan_.kernel == 1) {
            smem_bytes_ = (size_t)plan_.tile_docs * sizeof(float) + sizeof(bm25k::TileShared);
            RaiseSmemCap(reinterpret_cast<const void *>(bm25k::TileSearchKernel), smem_bytes_);
        } else {
            const void *kernel;
            int threads;
            long long per_tile;  // candidates one tile can append per query
            if (plan_.kernel == 0) {
                smem_bytes_ = (size_t)plan_.tile_docs * sizeof(float) +
                              2 * (size_t)plan_.stages * bm25k::kChunk * sizeof(int) + sizeof(bm25k::StreamShared);
                kernel = reinterpret_cast<const void *>(bm25k::StreamSearchKernel);
                threads = bm25k::kStreamThreads;
                per_tile = (long long)bm25k::kConsumerWarps * opts_.max_k;  // every warp region
            } else {
                // the tile-group kernel: the main kernel of kernel 4; with kernel 5 it streams the
                // routed and retried queries of pruned Searches
                tg_smem_ = bm25k::TileGroupSmem(plan_.stages, plan_.chunk, plan_.tile_docs);
                kernel = bm25k::TileGroupKernelFor(plan_.tile_docs);
                RaiseSmemCap(bm25k::TileGroupKernelFor(plan_.tile_docs, true), tg_smem_);
                RaiseSmemCap(kernel, tg_smem_);
                int tg_per_sm = 0, n_sms = 0;
                Cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&tg_per_sm, kernel, bm25k::kWgThreads, tg_smem_),
                     "occupancy");
                Check(tg_per_sm >= 1, "tile_docs / ring_stages exceed the shared memory of one SM");
                Cuda(cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, device_), "SM count");
                tg_grid_ = tg_per_sm * n_sms;
                smem_bytes_ = tg_smem_;
                threads = bm25k::kWgThreads;
                per_tile = opts_.max_k;
                if (plan_.kernel == BM25_KERNEL_WARP_TILE) {
                    smem_bytes_ = bm25k::WarpTileSmem();
                    for (const int c : {2, 4, 8}) {
                        RaiseSmemCap(reinterpret_cast<const void *>(WarpTileFor<true>(c)), smem_bytes_);
                        RaiseSmemCap(reinterpret_cast<const void *>(WarpTileFor<false>(c)), smem_bytes_);
                    }
                    RaiseSmemCap(reinterpret_cast<const void *>(&bm25k::BlockTileKernel), smem_bytes_);
                    kernel = bm25k::WarpTileKernelFor<kWtClaimTiles>(false);
                    threads = bm25k::kWtThreads;
                }
            }
            RaiseSmemCap(kernel, smem_bytes_);
            int per_sm = 0, sms = 0;
            Cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem_bytes_), "occupancy");
            Cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_), "SM count");
            Check(per_sm >= 1, "tile_docs / ring_stages exceed the shared memory of one SM");
            plan_.grid = per_sm * sms;
            sms_ = sms;
            const size_t qc = (size_t)opts_.query_capacity, tiles_z = (size_t)plan_.tiles;
            // worst case for K <= 32: every selection of every tile appends max_k candidates.  For
            // K > 32 a tile appends every document at or above the running bound; the buffer holds
            // 512 K (at least 2^18) and a query that overflows it is searched again from its final
            // bound by the retry pass.
            cand_cap_ = (long long)tiles_z * per_tile;
            if (opts_.max_k > bm25k::kMaxSmallK) {
                cand_cap_ = (long long)tiles_z * plan_.tile_docs;  // every document: the worst case
                Check(opts_.candidate_capacity == 0 || opts_.candidate_capacity >= opts_.max_k,
                      "candidate_capacity must be 0 or at least max_k");
                cand_cap_ = std::min<long long>(cand_cap_, opts_.candidate_capacity
                                                               ? opts_.candidate_capacity
                                                               : std::max<long long>(1 << 18, 512LL * opts_.max_k));
            }
            cand_cap_ = (cand_cap_ + 3) & ~3LL;  // rows start on 16-byte boundaries (128-bit reads)
            if (opts_.prune || opts_.max_k > bm25k::kMaxSmallK) {
                // lists: retry pass 1, retry pass 2, routed queries
                d_fail_list_ = static_cast<int *>(Alloc(3 * qc * sizeof(int), "cudaMalloc fail lists"));
                d_fail_count_ = static_cast<unsigned *>(Alloc(3 * sizeof(unsigned), "cudaMalloc fail counts"));
                Cuda(cudaMemset(d_fail_count_, 0, 3 * sizeof(unsigned)), "cudaMemset");
                d_qkept_ = static_cast<unsigned *>(Alloc(qc * sizeof(unsigned), "cudaMalloc kept counts"));
            }
            if (opts_.prune) {
                bs_smem_ = bm25k::BlockScoreSmem(plan_.tile_docs);
                const void *bs = bm25k::BlockScoreKernelFor(plan_.tile_docs);
                RaiseSmemCap(bs, bs_smem_);
                int bs_per_sm = 0;
                Cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bs_per_sm, bs, bm25k::kBsThreads, bs_smem_),
                     "occupancy");
                Check(bs_per_sm >= 1, "block score kernel does not fit an SM");
                bs_grid_ = bs_per_sm * sms;
            }
            ctrl_ = static_cast<bm25k::StreamCtrl *>(Alloc(sizeof(bm25k::StreamCtrl), "cudaMalloc ctrl"));
            threshold_ = static_cast<unsigned *>(Alloc(qc * sizeof(unsigned), "cudaMalloc threshold"));
            tslots_ = static_cast<unsigned *>(Alloc(qc * 32 * sizeof(unsigned), "cudaMalloc threshold slots"));
            Cuda(cudaMemset(tslots_, 0, qc * 32 * sizeof(unsigned)), "cudaMemset");
            cand_count_ = static_cast<unsigned *>(Alloc(qc * sizeof(unsigned), "cudaMalloc cand count"));
            cand_scores_ = static_cast<float *>(Alloc(qc * cand_cap_ * sizeof(float), "cudaMalloc candidates"));
            cand_ids_ = static_cast<int *>(Alloc(qc * cand_cap_ * sizeof(int), "cudaMalloc candidates"));
            // the (query word, tile) plan of every kernel but the warp-tile one, which uses it for the
            // Searches it hands to the tile-group kernel
            plan_entries_ = static_cast<bm25k::PlanEntry *>(Alloc(
                std::max<size_t>(1, opts_.word_capacity) * tiles_z * sizeof(bm25k::PlanEntry), "cudaMalloc plan"));
            if (plan_.kernel == BM25_KERNEL_WARP_TILE) {
                plan_rows_ = static_cast<int *>(Alloc(std::max<size_t>(1, opts_.word_capacity) * (tiles_z + 1) *
                                                          sizeof(int),
                                                      "cudaMalloc plan rows"));
                word_rec_ = static_cast<int4 *>(
                    Alloc(std::max<size_t>(1, opts_.word_capacity) * sizeof(int4), "cudaMalloc word records"));
            }
            Cuda(cudaMemset(ctrl_, 0, sizeof(bm25k::StreamCtrl)), "cudaMemset");
            d_stats_ = static_cast<unsigned long long *>(Alloc(bm25k::kStats * sizeof(unsigned long long), "cudaMalloc stats"));
            Cuda(cudaMemset(d_stats_, 0, bm25k::kStats * sizeof(unsigned long long)), "cudaMemset");
            Cuda(cudaMemset(threshold_, 0, qc * sizeof(unsigned)), "cudaMemset");
            Cuda(cudaMemset(cand_count_, 0, qc * sizeof(unsigned)), "cudaMemset");
        }
        Cuda(cudaDeviceSynchronize(), "index preparation");
    }

    // Dense rows of the warp-tile kernel: the terms with df >= density * N, largest first, within a
    // byte budget (the index's own size, at most 16 GiB); each row holds tiles * 1024 scores.
    void BuildDense(const std::vector<int64_t> &dfs)
    {
        const double density = opts_.dense_density > 0.0f ? opts_.dense_density : 0.25;
        const int64_t min_df = std::max<int64_t>(1, (int64_t)std::ceil(density * (double)docs_));
        dense_stride_ = (int64_t)plan_.tiles * plan_.tile_docs;
        const int64_t budget = std::min<int64_t>(int64_t(16) << 30, std::max<int64_t>(index_bytes_, 1));
        std::vector<int32_t> terms;
        for (int64_t t = 0; t < vocab_; ++t)
            if (dfs[t] >= min_df)
                terms.push_back((int32_t)t);
        std::sort(terms.begin(), terms.end(), [&](int32_t x, int32_t y) { return dfs[x] > dfs[y] || (dfs[x] == dfs[y] && x < y); });
        const int64_t fit = budget / (dense_stride_ * (int64_t)sizeof(float));
        if ((int64_t)terms.size() > fit)
            terms.resize((size_t)std::max<int64_t>(0, fit));
        dense_rows_ = (int64_t)terms.size();
        std::vector<int32_t> row_of(vocab_, -1);
        for (size_t r = 0; r < terms.size(); ++r)
            row_of[terms[r]] = (int32_t)r;
        d_dense_row_ = static_cast<int32_t *>(Alloc(vocab_ * sizeof(int32_t), "cudaMalloc dense row"));
        Cuda(cudaMemcpy(d_dense_row_, row_of.data(), vocab_ * sizeof(int32_t), cudaMemcpyHostToDevice), "dense upload");
        if (terms.empty())
            return;
        d_dense_ = static_cast<float *>(Alloc((size_t)dense_rows_ * dense_stride_ * sizeof(float), "cudaMalloc dense rows"));
        Cuda(cudaMemset(d_dense_, 0, (size_t)dense_rows_ * dense_stride_ * sizeof(float)), "cudaMemset dense rows");
        int32_t *d_terms = static_cast<int32_t *>(Alloc(terms.size() * sizeof(int32_t), "cudaMalloc dense terms"));
        Cuda(cudaMemcpy(d_terms, terms.data(), terms.size() * sizeof(int32_t), cudaMemcpyHostToDevice), "dense upload");
        bm25k::BuildDenseKernel<<<dim3(256, (unsigned)dense_rows_), 256, 0, stream_>>>(
            (const long long *)d_indptr_, d_indices_, d_data_, d_terms, d_dense_, dense_stride_);
        Cuda(cudaGetLastError(), "dense row kernel launch");
        Cuda(cudaStreamSynchronize(stream_), "dense row kernel");
    }

    // tau / exact: the pruned Search's starting bounds and exactness flags (nullptr: plain Search).
    void Launch(int q, int k, const int64_t *qoffsets, const int32_t *words, float *out_scores, int32_t *out_ids,
                unsigned *status, cudaStream_t s, const float *tau = nullptr, int32_t *exact = nullptr,
                bool learned = false, const int32_t *kq = nullptr, const int64_t *kout = nullptr)
    {
        bm25k::TileArgs a{};
        a.indptr = (const long long *)d_indptr_;
        a.indices = d_indices_;
        a.data = d_data_;
        a.dir_row = d_dir_row_;
        a.dir = d_dir_;
        a.dir_stride = plan_.tiles + 1;
        a.qoffsets = (const long long *)qoffsets;
        a.words = words;
        a.word_cap = std::max<int64_t>(1, opts_.word_capacity);
        a.vocab = (int)vocab_;
        a.num_docs = (int)docs_;
        a.tile_docs = plan_.tile_docs;
        a.tiles = plan_.tiles;
        a.k = k;
        a.fan_in = plan_.fan_in;
        a.levels = plan_.levels;
        for (int l = 0; l < (int)levels_.size(); ++l)
            a.lv[l] = levels_[l];
        a.out_scores = out_scores;
        a.out_ids = out_ids;
        a.status = status;
        if (plan_.kernel == 1) {
            dim3 grid(plan_.tiles, q);
            MarkKernel(0, s);
            bm25k::TileSearchKernel<<<grid, bm25k::kThreads, smem_bytes_, s>>>(a);
            MarkKernel(1, s);
        } else {
            bm25k::StreamArgs sa{};
            sa.indptr = a.indptr;
            sa.indices = a.indices;
            sa.data = a.data;
            sa.dir_row = a.dir_row;
            sa.dir = a.dir;
            sa.dir_stride = a.dir_stride;
            sa.qoffsets = a.qoffsets;
            sa.words = a.words;
            sa.vocab = a.vocab;
            sa.num_docs = a.num_docs;
            sa.tile_docs = a.tile_docs;
            sa.tiles = a.tiles;
            sa.k = k;
            sa.q = q;
            sa.word_cap = a.word_cap;
            sa.plan = plan_entries_;
            sa.threshold = threshold_;
            sa.tslots = tslots_;
            sa.cand_count = cand_count_;
            sa.cand_scores = cand_scores_;
            sa.cand_ids = cand_ids_;
            // a tuned capacity (bm25_set_tuning) is a narrower stride over the same rows, for batches of
            // one K > 32 only: a query of those that overflows it is searched again (a K <= 32 query's
            // final select has no retry and counts on the allocated worst case)
            sa.cand_cap = tuning_.candidate_cap > 0 && k > bm25k::kMaxSmallK && !kq ? tuning_.candidate_cap
                                                                                    : cand_cap_;
            sa.ctrl = ctrl_;
            sa.stages = plan_.stages;
            sa.chunk = plan_.chunk;
            sa.out_scores = out_scores;
            sa.out_ids = out_ids;
            sa.status = status;
            sa.stats = TileFamily(plan_.kernel) ? d_stats_ : nullptr;
            // the retry pass answers the queries on the fail list: those whose starting bound proved
            // too high, and (K > 32) those whose candidate buffer overflowed
            // a batch with a K per query (kq): k is its largest K, each final select takes its queries
            sa.kq = kq;
            sa.kout = (const long long *)kout;
            // pass 1 lists the queries it could not answer; retry pass 1 searches them on the plain
            // path; with K > 32 a query whose buffer overflowed there (its slots were weak: a pruned
            // first pass fell short) is searched once more from the slots that pass filled
            const bool retry = tau != nullptr || k > bm25k::kMaxSmallK;
            const bool retry2 = k > bm25k::kMaxSmallK;
            int *list_a = d_fail_list_, *list_b = d_fail_list_ + opts_.query_capacity;
            if (retry) {
                sa.fail_out = list_a;
                sa.fail_out_count = d_fail_count_;
                Cuda(cudaMemsetAsync(d_fail_count_, 0, 3 * sizeof(unsigned), s), "fail count reset");
            }
            // routing (pruned batches of 32 queries or more): the queries whose bounds keep too many
            // blocks are streamed by the tile-group kernel, the others scored block by block
            const float route = tuning_.prune_route != 0.0f ? tuning_.prune_route
                                : plan_.kernel == BM25_KERNEL_WARP_TILE ? 1.0f
                                                                        : 0.3f;
            const bool routing = tau != nullptr && q >= 32 && route > 0.0f && route < 1.0f;
            if (routing) {
                sa.qkept = d_qkept_;
                sa.route_limit =
                    (unsigned)std::max(1.0, (double)route * plan_.tiles * (plan_.tile_docs / bm25k::kBlockDocs));
                sa.route_list = d_fail_list_ + 2 * (size_t)opts_.query_capacity;
                sa.route_count = d_fail_count_ + 2;
                Cuda(cudaMemsetAsync(d_qkept_, 0, (size_t)q * sizeof(unsigned), s), "kept count reset");
            }
            if (learned) {
                // tau is this session's bound array, written here; the plan kernel, launched
                // overlapped, is built meanwhile and waits for these bounds before it completes
                bm25k::LearnedArgs la = LearnedArgsFor(q, k, qoffsets, words);
                la.kq = kq;
                la.safe = d_safe_;
                bm25k::LearnedBoundKernel<<<(q + bm25k::kLearnedQueries - 1) / bm25k::kLearnedQueries,
                                            bm25k::kLearnedThreads, 0, s>>>(la);
                Cuda(cudaGetLastError(), "learned bound kernel launch");
            }
            if (tau) {
                sa.boff = d_boff_;
                sa.bmax = d_bmax_;
                sa.tau = tau;
                sa.exact = exact;
                sa.items = d_items_;
                sa.wrow = d_wrow_;
                sa.item_count = d_item_count_;
                sa.item_cap = item_cap_;
            }
            // A warp-tile session runs the warp-tile kernel for plain Searches of one K <= 32 and for
            // every pass that streams from a bound already set (the routed queries of a pruned Search,
            // from their learned bound; retry passes, from their proven one), all on the plan rows of
            // the Search's words.  The first pass of a pruned Search is block-scored (block-tile
            // kernel, also on the plan rows); that of a batch with a K per query or K > 32 runs the
            // tile-group kernel on the (query word, tile) plan (the warp-tile kernel's wider first
            // wave of claims would append far more candidates there).
            const bool wt_session = plan_.kernel == BM25_KERNEL_WARP_TILE;
            const bool warp_tile = wt_session && !tau && !kq && k <= bm25k::kMaxSmallK;
            // the streaming passes after a first pass (retries, routed queries) run the warp-tile kernel
            // too, on the plan rows; a pruned Search of a warp-tile session takes its block path's
            // ranges from the plan rows as well and builds no (query word, tile) plan
            const bool wt_streams = wt_session;
            const bool rows_only = wt_session && tau != nullptr;
            sa.rows_plan = rows_only ? 1 : 0;
            sa.plan_rows = plan_rows_;
            sa.word_rec = word_rec_;
            sa.prefetch = 1;
            sa.wait_budget = opts_.wait_budget_cycles;
            sa.term_top = plan_.kernel == BM25_KERNEL_WARP_TILE ? d_term_top_ : nullptr;
            sa.term_rank = d_term_rank_;
            sa.dense = d_dense_;
            sa.dense_row = d_dense_row_;
            sa.dense_stride = dense_stride_;
            sa.inject = d_inject_;
            if (warp_tile) {
                bm25k::PlanRowsKernel<<<bm25k::PlanRowsGrid(opts_.word_capacity, plan_.tiles, sms_),
                                        bm25k::kPlanThreads, 0, s>>>(sa);
            } else if (rows_only) {
                // after the learned bounds kernel: set up while it runs (it writes nothing the rows read)
                LaunchOverlapped(bm25k::PlanRowsKernel, bm25k::PlanRowsGrid(opts_.word_capacity, plan_.tiles, sms_),
                                 bm25k::kPlanThreads, 0, s, sa);
            } else {
                if (learned)
                    LaunchOverlapped(bm25k::PlanKernel, bm25k::PlanGrid(opts_.word_capacity, plan_.tiles, sms_),
                                     bm25k::kPlanThreads, 0, s, sa);
                else
                    bm25k::PlanKernel<<<bm25k::PlanGrid(opts_.word_capacity, plan_.tiles, sms_), bm25k::kPlanThreads,
                                        0, s>>>(sa);
                if (wt_streams)  // for the streaming passes; set up while the plan kernel runs
                    LaunchOverlapped(bm25k::PlanRowsKernel, bm25k::PlanRowsGrid(opts_.word_capacity, plan_.tiles, sms_),
                                     bm25k::kPlanThreads, 0, s, sa);
            }
            Cuda(cudaGetLastError(), "plan kernel launch");
            const long long claims = (long long)q * ((plan_.tiles + bm25k::kWgWarps - 1) / bm25k::kWgWarps);
            const int wg_grid = (int)std::max<long long>(1, std::min<long long>(tg_grid_, claims));
            const int ct = tuning_.claim_tiles;
            const long long wt_claims = (long long)q * ((plan_.tiles + ct - 1) / ct);
            const int wt_grid = (int)std::max<long long>(
                1, std::min<long long>(plan_.grid, (wt_claims + bm25k::kWtWarps - 1) / bm25k::kWtWarps));
            {
                // single-tile claims for the last tiles: tail_claims per warp of the launch
                const long long tail = ((long long)tuning_.tail_claims * wt_grid * bm25k::kWtWarps + q - 1) / q;
                sa.wt_bulk = (int)std::max<long long>(0, (plan_.tiles - tail) / ct);
            }
            auto tile_group = [&](const bm25k::StreamArgs &args) {
                const bool lean = !args.retry && !args.kq && k <= bm25k::kMaxSmallK;
                if (warp_tile || (wt_streams && args.retry)) {
                    if (!args.retry)  // right after the plan rows: set up while they are built
                        LaunchOverlapped(lean ? WarpTileFor<true>(ct) : WarpTileFor<false>(ct), wt_grid,
                                         bm25k::kWtThreads, smem_bytes_, s, args);
                    else
                        WarpTileFor<false>(ct)<<<wt_grid, bm25k::kWtThreads, smem_bytes_, s>>>(args);
                } else if (plan_.tile_docs == 2048) {
                    if (lean)
                        bm25k::TileGroupKernel<2048, true><<<wg_grid, bm25k::kWgThreads, tg_smem_, s>>>(args);
                    else
                        bm25k::TileGroupKernel<2048><<<wg_grid, bm25k::kWgThreads, tg_smem_, s>>>(args);
                } else {
                    if (lean)  // right after the plan kernel: set up while it runs
                        LaunchOverlapped(bm25k::TileGroupKernel<1024, true>, wg_grid, bm25k::kWgThreads, tg_smem_, s,
                                         args);
                    else
                        bm25k::TileGroupKernel<1024><<<wg_grid, bm25k::kWgThreads, tg_smem_, s>>>(args);
                }
            };
            // the kept blocks of a pruned pass: the warp-tile style scorer in a warp-tile session
            // (1024-document tiles, its counter and shared memory), else the staging block scorer
            auto block_score = [&](const bm25k::StreamArgs &args) {
                if (wt_session)
                    LaunchOverlapped(bm25k::BlockTileKernel, plan_.grid, bm25k::kWtThreads, smem_bytes_, s, args);
                else if (plan_.tile_docs == 2048)
                    LaunchOverlapped(bm25k::BlockScoreKernel<2048>, bs_grid_, bm25k::kBsThreads, bs_smem_, s, args);
                else
                    LaunchOverlapped(bm25k::BlockScoreKernel<1024>, bs_grid_, bm25k::kBsThreads, bs_smem_, s, args);
            };
            auto final_select = [&](const bm25k::StreamArgs &args) {
                if (k <= bm25k::kMaxSmallK || kq)
                    LaunchOverlapped(bm25k::FinalSelectKernel, q, bm25k::kFinalThreads, 0, s, args);
                if (k > bm25k::kMaxSmallK)
                    bm25k::FinalSelectLargeKernel<<<q, bm25k::kLargeThreads, 0, s>>>(args);
            };
            if (tau) {
                // block-max pruned pass: bounds per (query, tile, block), then the kept blocks
                const dim3 bgrid((plan_.tiles + bm25k::kBbThreads - 1) / bm25k::kBbThreads, q);
                if (plan_.tile_docs == 2048)
                    LaunchOverlapped(bm25k::BlockBoundKernel<2048>, bgrid, bm25k::kBbThreads, 0, s, sa);
                else
                    LaunchOverlapped(bm25k::BlockBoundKernel<1024>, bgrid, bm25k::kBbThreads, 0, s, sa);
                Cuda(cudaGetLastError(), "block bound kernel launch");
                if (routing) {
                    bm25k::RouteKernel<<<1, 256, 0, s>>>(sa);
                    Cuda(cudaGetLastError(), "route kernel launch");
                }
                MarkKernel(0, s);
                block_score(sa);
                Cuda(cudaGetLastError(), "block score kernel launch");
                MarkKernel(1, s);
                if (routing) {  // the routed queries, streamed from their starting bound
                    bm25k::StreamArgs xa = sa;
                    xa.retry = 1;
                    xa.fail_in = sa.route_list;
                    xa.fail_in_count = sa.route_count;
                    tile_group(xa);
                    Cuda(cudaGetLastError(), "routed tile group launch");
                }
            } else if (plan_.kernel == 0) {
                const int grid = (int)std::min<long long>(
                    plan_.grid, ((long long)q * plan_.tiles + bm25k::kTaskBatch - 1) / bm25k::kTaskBatch);
                MarkKernel(0, s);
                bm25k::StreamSearchKernel<<<std::max(grid, 1), bm25k::kStreamThreads, smem_bytes_, s>>>(sa);
                Cuda(cudaGetLastError(), "stream kernel launch");
                MarkKernel(1, s);
            } else {
                MarkKernel(0, s);
                tile_group(sa);
                Cuda(cudaGetLastError(), "tile group kernel launch");
                MarkKernel(1, s);
            }
            final_select(sa);
            Cuda(cudaGetLastError(), "final select launch");
            if (retry) {
                // retry pass on the plain path (an empty fail list ends both kernels at once)
                bm25k::StreamArgs ra = sa;
                ra.tau = nullptr;
                ra.exact = nullptr;
                ra.retry = 1;
                ra.fail_in = list_a;
                ra.fail_in_count = d_fail_count_;
                ra.fail_out = retry2 ? list_b : nullptr;
                ra.fail_out_count = retry2 ? d_fail_count_ + 1 : nullptr;
                ra.qkept = nullptr;
                ra.route_limit = 0;
                if (tau) {
                    // a pruned first pass: the retry is block-pruned too, from each query's proven
                    // bound (its slots, its safe bound), so a wrong guess costs little
                    ra.item_count = d_item_count_ + 2;
                    ra.safe = learned ? d_safe_ : nullptr;
                    const dim3 bgrid((plan_.tiles + bm25k::kBbThreads - 1) / bm25k::kBbThreads, q);
                    if (plan_.tile_docs == 2048)
                        LaunchOverlapped(bm25k::BlockBoundKernel<2048>, bgrid, bm25k::kBbThreads, 0, s, ra);
                    else
                        LaunchOverlapped(bm25k::BlockBoundKernel<1024>, bgrid, bm25k::kBbThreads, 0, s, ra);
                    block_score(ra);
                } else {
                    ra.items = nullptr;
                    ra.wrow = nullptr;
                    ra.item_count = nullptr;
                    tile_group(ra);
                }
                Cuda(cudaGetLastError(), "retry kernel launch");
                final_select(ra);
                if (retry2) {
                    bm25k::StreamArgs rb = ra;
                    rb.items = nullptr;
                    rb.wrow = nullptr;
                    rb.item_count = nullptr;
                    rb.safe = nullptr;
                    rb.fail_in = list_b;
                    rb.fail_in_count = d_fail_count_ + 1;
                    rb.fail_out = nullptr;
                    rb.fail_out_count = nullptr;
                    tile_group(rb);
                    Cuda(cudaGetLastError(), "second retry kernel launch");
                    final_select(rb);
                }
            }
        }
        Cuda(cudaGetLastError(), "search kernel launch");
    }

    // Output arena: the status word first (32 bytes, at the same place for every graph), then the
    // scores, the ids and the exactness flags.  A Search that succeeds leaves the status 0 (any bit
    // fails the Search and poisons the session), so no graph has to clear it before its kernels.
    static constexpr size_t kScoreOffset = 32;
    size_t IdOffset(int q, int k) const { return kScoreOffset + Align32((size_t)q * k * 4); }
    size_t ExactOffset(int q, int k) const { return IdOffset(q, k) + Align32((size_t)q * k * 4); }

    void MarkKernel(int which, cudaStream_t s)
    {
        if (marking_)
            Cuda(cudaEventRecord(timing_[2 * (size_t)(timed_ % kTimingRing) + which], s), "cudaEventRecord");
    }

    void DestroyTiming()
    {
        for (auto e : timing_)
            cudaEventDestroy(e);
        timing_.clear();
        timed_ = 0;
    }

    static constexpr int kModePlain = 0, kModePruned = 1, kModeLearned = 2, kModeMixed = 4;

    cudaGraphExec_t GraphFor(int q, int k, int mode = kModePlain)
    {
        const auto key = std::make_tuple(q, k, mode);
        const bool mixed = (mode & kModeMixed) != 0;
        mode &= ~kModeMixed;
        const bool pruned = mode != kModePlain;
        auto it = graphs_.find(key);
        if (it != graphs_.end()) {
            it->second.last_use = ++graph_uses_;
            return it->second.exec;
        }
        if (graphs_.size() >= kGraphCacheMax) {  // bounded: drop the least recently used graph
            auto old = graphs_.begin();
            for (auto g = graphs_.begin(); g != graphs_.end(); ++g)
                if (g->second.last_use < old->second.last_use)
                    old = g;
            Cuda(cudaStreamWaitEvent(stream_, done_, 0), "cudaStreamWaitEvent");
            Cuda(cudaStreamSynchronize(stream_), "graph eviction");
            cudaGraphExecDestroy(old->second.exec);
            graphs_.erase(old);
        }
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        Cuda(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin graph capture");
        try {
            // the plain Search sends the query packet; the pruned one adds the bounds after it
            Cuda(cudaMemcpyAsync(d_in_, h_in_,
                                 mixed ? in_bytes_
                                       : (mode == kModePruned ? tau_offset_ + (size_t)q * sizeof(float) : tau_offset_),
                                 cudaMemcpyHostToDevice, stream_),
                 "query H2D");
            unsigned *status = reinterpret_cast<unsigned *>(d_out_);  // 0 unless a Search failed
            Launch(q, k, reinterpret_cast<const int64_t *>(d_in_), reinterpret_cast<const int32_t *>(d_in_ + word_offset_),
                   reinterpret_cast<float *>(d_out_ + kScoreOffset), reinterpret_cast<int32_t *>(d_out_ + IdOffset(q, k)),
                   status,
                   stream_,
                   mode == kModePruned ? reinterpret_cast<const float *>(d_in_ + tau_offset_)
                                       : (mode == kModeLearned ? d_tau_ : nullptr),
                   pruned ? reinterpret_cast<int32_t *>(d_out_ + ExactOffset(q, k)) : nullptr,
                   mode == kModeLearned, mixed ? reinterpret_cast<const int32_t *>(d_in_ + ks_offset_) : nullptr,
                   mixed ? reinterpret_cast<const int64_t *>(d_in_ + kout_offset_) : nullptr);
            if (!mixed)  // a batch's result size varies per call: copied after the replay
                Cuda(cudaMemcpyAsync(h_out_, d_out_,
                                     pruned ? ExactOffset(q, k) + (size_t)q * 4 : ExactOffset(q, k),
                                     cudaMemcpyDeviceToHost, stream_),
                     "top-K D2H");
        } catch (...) {
            cudaStreamEndCapture(stream_, &graph);
            if (graph)
                cudaGraphDestroy(graph);
            throw;
        }
        Cuda(cudaStreamEndCapture(stream_, &graph), "end graph capture");
        const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        Cuda(e, "cudaGraphInstantiate");
        ++instantiations_;
        graphs_[key] = CachedGraph{exec, ++graph_uses_};
        return exec;
    }

    // Validates the whole request before writing the arena (fixed_query_packet.h:26-49).
    void Pack(const int64_t *qoffsets, const int32_t *words, int64_t q, int32_t k)
    {
        Check(q >= 1 && q <= opts_.query_capacity, "Query batch exceeds declared capacity or is empty");
        Check(k >= 1 && k <= opts_.max_k && k <= docs_, "K outside [1, min(max_k, N)]");
        Check(qoffsets != nullptr && qoffsets[0] == 0, "Query offsets must start at 0");
        for (int64_t i = 0; i < q; ++i) {
            const int64_t n = qoffsets[i + 1] - qoffsets[i];
            Check(n >= 0 && n <= bm25k::kMaxTerms, "Query exceeds fixed word/64-term capacity");
        }
        const int64_t total = qoffsets[q];
        Check(total <= opts_.word_capacity, "Word IDs exceed declared query capacity");
        Check(total == 0 || words != nullptr, "Null word buffer");
        for (int64_t w = 0; w < total; ++w)
            Check(words[w] >= 0 && words[w] < INT32_MAX, "Invalid public word ID");
        std::memset(h_in_, 0, in_bytes_);
        std::memcpy(h_in_, qoffsets, (q + 1) * sizeof(int64_t));
        if (total)
            std::memcpy(static_cast<unsigned char *>(h_in_) + word_offset_, words, total * sizeof(int32_t));
    }

    // Host-side result checks of large_search.cpp:153-174.
    void Receive(int64_t q, int32_t k, float *out_scores, int32_t *out_ids)
    {
        const unsigned char *base = static_cast<const unsigned char *>(h_out_);
        unsigned status = 0;
        std::memcpy(&status, base, sizeof(unsigned));
        if (status)
            throw DeviceError(0, "Device reported invalid Search state, status=" + std::to_string(status));
        const float *scores = reinterpret_cast<const float *>(base + kScoreOffset);
        const int32_t *ids = reinterpret_cast<const int32_t *>(base + IdOffset((int)q, k));
        const size_t n = (size_t)q * k;
        for (size_t i = 0; i < n; ++i) {
            if (!(ids[i] >= 0 && ids[i] < docs_ && std::isfinite(scores[i]) && scores[i] >= 0))
                throw DeviceError(0, "Invalid real-document result");
            if (i % k && !(scores[i - 1] > scores[i] || (scores[i - 1] == scores[i] && ids[i - 1] < ids[i])))
                throw DeviceError(0, "Strict global ranking failure");
        }
        std::memcpy(out_scores, scores, n * sizeof(float));
        std::memcpy(out_ids, ids, n * sizeof(int32_t));
    }

    void Release()
    {
        for (auto &g : graphs_)
            cudaGraphExecDestroy(g.second.exec);
        graphs_.clear();
        for (void *p : allocations_)
            cudaFree(p);
        allocations_.clear();
        levels_.clear();
        if (h_in_)
            cudaFreeHost(h_in_);
        if (h_out_)
            cudaFreeHost(h_out_);
        h_in_ = h_out_ = nullptr;
        DestroyTiming();
        if (done_)
            cudaEventDestroy(done_);
        done_ = nullptr;
        if (own_stream_ && stream_)
            cudaStreamDestroy(stream_);
        stream_ = nullptr;
        own_stream_ = false;
    }

    bm25_options opts_;
    int64_t vocab_, docs_, postings_;
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    bool own_stream_ = false;
    cudaEvent_t done_ = nullptr;
    size_t free_at_start_ = 0;
    Plan plan_;
    bm25_tuning tuning_{kWtClaimTiles, 2, 0, 0, 0, 0.0f, 0};
    std::vector<void *> allocations_;
    int64_t device_bytes_ = 0, index_bytes_ = 0;
    int64_t *d_indptr_ = nullptr;
    int32_t *d_indices_ = nullptr;
    float *d_data_ = nullptr;
    int32_t *d_dir_row_ = nullptr, *d_dir_ = nullptr;
    std::vector<bm25k::Level> levels_;
    size_t word_offset_ = 0, tau_offset_ = 0, ks_offset_ = 0, kout_offset_ = 0, in_bytes_ = 0, out_bytes_ = 0,
           smem_bytes_ = 0;
    unsigned short *d_boff_ = nullptr;
    __half *d_bmax_ = nullptr;
    uint4 *d_items_ = nullptr;
    int *d_wrow_ = nullptr;
    float *d_safe_ = nullptr;
    unsigned *d_item_count_ = nullptr;
    long long item_cap_ = 0;
    size_t bs_smem_ = 0;
    int bs_grid_ = 0;
    void *h_in_ = nullptr, *h_out_ = nullptr;
    unsigned char *d_in_ = nullptr, *d_out_ = nullptr;
    unsigned *d_dev_status_ = nullptr;
    unsigned *d_inject_ = nullptr;  // test hook word read by the tile-group kernel's producer
    bool stall_armed_ = false, fail_armed_ = false;
    int64_t instantiations_ = 0;
    bm25k::StreamCtrl *ctrl_ = nullptr;
    unsigned *threshold_ = nullptr, *cand_count_ = nullptr, *tslots_ = nullptr;
    float *cand_scores_ = nullptr;
    int *cand_ids_ = nullptr;
    long long cand_cap_ = 0;
    bm25k::PlanEntry *plan_entries_ = nullptr;
    int *plan_rows_ = nullptr;
    int4 *word_rec_ = nullptr;  // warp-tile sessions: per query word (seed bits, dense row, directory row)
    float *d_dense_ = nullptr;  // dense rows of the most frequent terms (warp-tile kernel)
    float *d_term_rank_ = nullptr;  // [vocab][5] scores at ranks 64 .. 1024 (warp-tile kernel)
    int32_t *d_dense_row_ = nullptr;
    int64_t dense_rows_ = 0, dense_stride_ = 0;
    size_t tg_smem_ = 0;  // tile-group kernel: dynamic shared memory and grid
    int tg_grid_ = 0;
    int sms_ = 148;
    struct CachedGraph {
        cudaGraphExec_t exec;
        int64_t last_use;
    };
    static constexpr size_t kGraphCacheMax = 64;  // instantiated graphs kept; the least recently used goes
    std::map<std::tuple<int, int, int>, CachedGraph> graphs_;
    int64_t graph_uses_ = 0;
    float *d_term_top_ = nullptr, *d_term_mean_ = nullptr, *d_model_ = nullptr, *d_tau_ = nullptr;
    unsigned long long *d_stats_ = nullptr;
    int *d_fail_list_ = nullptr;
    unsigned *d_fail_count_ = nullptr, *d_qkept_ = nullptr;
    bool has_model_ = false;
    float margin_ = 0.0f;
    bool closed_ = false, failed_ = false;
    int64_t replays_ = 0, searches_ = 0;
    static constexpr int64_t kTimingRing = 4096;
    std::vector<cudaEvent_t> timing_;  // [start, end] per ring slot
    int64_t timed_ = 0;
    bool marking_ = false;
};

} // namespace bm25b200

// ---------------------------------------------------------------------------
// C ABI

struct bm25_handle {
    std::mutex mutex;
    std::unique_ptr<bm25b200::Engine> engine;
    std::string error;
    int64_t code = 0;
};

namespace {
thread_local std::string g_create_error;
thread_local int64_t g_create_code = 0;

// Error mapping of Bm25ErrorAdapter.h:11-45.
template <class F> int Invoke(F &&f, std::string &error, int64_t &code) noexcept
{
    error.clear();
    code = 0;
    try {
        f();
        return BM25_OK;
    } catch (const bm25b200::InvalidArgument &e) {
        error = e.what();
        return BM25_ERR_INVALID_PARAM;
    } catch (const bm25b200::InvalidState &e) {
        error = e.what();
        return BM25_ERR_ILLEGAL_OPERATION;
    } catch (const bm25b200::DeviceError &e) {
        error = e.what();
        code = e.code;
        return BM25_ERR_INNER_ERROR;
    } catch (const std::exception &e) {
        error = e.what();
        return BM25_ERR_INNER_ERROR;
    } catch (...) {
        error = "Unknown BM25 failure";
        return BM25_ERR_INNER_ERROR;
    }
}

template <class Upload>
int Create(int64_t vocab, int64_t docs, int64_t postings, const bm25_options *options, bm25_handle **out,
           Upload &&upload)
{
    return Invoke(
        [&] {
            bm25b200::Check(out != nullptr, "Null handle output");
            *out = nullptr;
            bm25_options o;
            bm25_default_options(&o);
            if (options)
                o = *options;
            auto h = std::make_unique<bm25_handle>();
            h->engine = std::make_unique<bm25b200::Engine>(o, vocab, docs, postings);
            upload(*h->engine);
            *out = h.release();
        },
        g_create_error, g_create_code);
}
} // namespace

extern "C" {

void bm25_default_options(bm25_options *o)
{
    if (!o)
        return;
    std::memset(o, 0, sizeof(*o));
    o->device_id = 0;
    o->max_k = 10;
    o->query_capacity = 8;
    o->word_capacity = 24;
    o->kernel = BM25_KERNEL_WARP_TILE;
}

int bm25_create(const int64_t *indptr, const int32_t *indices, const float *data, int64_t vocab, int64_t num_docs,
                const bm25_options *options, bm25_handle **out)
{
    int64_t postings = 0;
    const int pre = Invoke(
        [&] {
            bm25b200::Check(indptr != nullptr && vocab >= 1 && vocab < INT32_MAX, "Empty or oversized index");
            postings = indptr[vocab];
            bm25b200::ValidateEager(indptr, indices, data, vocab, num_docs);
        },
        g_create_error, g_create_code);
    if (pre != BM25_OK) {
        if (out)
            *out = nullptr;
        return pre;
    }
    return Create(vocab, num_docs, postings, options, out,
                  [&](bm25b200::Engine &e) { e.UploadEager(indptr, indices, data); });
}

int bm25_create_lazy(const int64_t *term_offsets, const int32_t *posting_doc_ids, const float *posting_tf,
                     const float *doc_norm, const float *idf, int64_t vocab, int64_t num_docs, float k1,
                     const bm25_options *options, bm25_handle **out)
{
    int64_t postings = 0;
    const int pre = Invoke(
        [&] {
            bm25b200::Check(term_offsets != nullptr && vocab >= 1 && vocab < INT32_MAX, "Empty or oversized index");
            postings = term_offsets[vocab];
            bm25b200::ValidateLazy(term_offsets, posting_doc_ids, posting_tf, doc_norm, idf, vocab, num_docs);
        },
        g_create_error, g_create_code);
    if (pre != BM25_OK) {
        if (out)
            *out = nullptr;
        return pre;
    }
    return Create(vocab, num_docs, postings, options, out, [&](bm25b200::Engine &e) {
        e.UploadLazy(term_offsets, posting_doc_ids, posting_tf, doc_norm, idf, k1);
    });
}

int bm25_search(bm25_handle *h, const int64_t *qoffsets, const int32_t *words, int64_t q, int32_t k,
                float *out_scores, int32_t *out_ids)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            h->engine->Search(qoffsets, words, q, k, out_scores, out_ids);
        },
        h->error, h->code);
}

int bm25_search_device(bm25_handle *h, const int64_t *qoffsets, const int32_t *words, int64_t q, int32_t k,
                       float *out_scores, int32_t *out_ids, void *stream)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            h->engine->SearchDevice(qoffsets, words, q, k, out_scores, out_ids, static_cast<cudaStream_t>(stream));
        },
        h->error, h->code);
}

int bm25_search_pruned_device(bm25_handle *h, const int64_t *qoffsets, const int32_t *words, const float *tau,
                              int64_t q, int32_t k, float *out_scores, int32_t *out_ids, int32_t *out_exact,
                              void *stream)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            bm25b200::Check(tau != nullptr, "Null tau buffer");
            h->engine->SearchPrunedDevice(qoffsets, words, tau, q, k, out_scores, out_ids, out_exact,
                                          static_cast<cudaStream_t>(stream));
        },
        h->error, h->code);
}

int bm25_search_pruned(bm25_handle *h, const int64_t *qoffsets, const int32_t *words, const float *tau, int64_t q,
                       int32_t k, float *out_scores, int32_t *out_ids, int32_t *out_exact)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            bm25b200::Check(tau != nullptr, "Null tau buffer");
            h->engine->SearchPruned(qoffsets, words, tau, q, k, out_scores, out_ids, out_exact);
        },
        h->error, h->code);
}

int bm25_search_learned(bm25_handle *h, const int64_t *qoffsets, const int32_t *words, int64_t q, int32_t k,
                        float *out_scores, int32_t *out_ids, int32_t *out_exact)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            h->engine->SearchPruned(qoffsets, words, nullptr, q, k, out_scores, out_ids, out_exact);
        },
        h->error, h->code);
}

int bm25_search_learned_device(bm25_handle *h, const int64_t *qoffsets, const int32_t *words, int64_t q, int32_t k,
                               float *out_scores, int32_t *out_ids, int32_t *out_exact, void *stream)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            h->engine->SearchPrunedDevice(qoffsets, words, nullptr, q, k, out_scores, out_ids, out_exact,
                                          static_cast<cudaStream_t>(stream));
        },
        h->error, h->code);
}

int bm25_search_batch(bm25_handle *h, const int64_t *qoffsets, const int32_t *words, const int32_t *ks, int64_t q,
                      float *out_scores, int32_t *out_ids)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            h->engine->SearchBatch(qoffsets, words, ks, q, false, out_scores, out_ids, nullptr);
        },
        h->error, h->code);
}

int bm25_search_batch_learned(bm25_handle *h, const int64_t *qoffsets, const int32_t *words, const int32_t *ks,
                              int64_t q, float *out_scores, int32_t *out_ids, int32_t *out_exact)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            h->engine->SearchBatch(qoffsets, words, ks, q, true, out_scores, out_ids, out_exact);
        },
        h->error, h->code);
}

int bm25_search_batch_device(bm25_handle *h, const int64_t *qoffsets, const int32_t *words, const int32_t *ks,
                             const int64_t *kout, int64_t q, int32_t kmax, int32_t learned, float *out_scores,
                             int32_t *out_ids, int32_t *out_exact, void *stream)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            h->engine->SearchBatchDevice(qoffsets, words, ks, kout, q, kmax, learned != 0, out_scores, out_ids,
                                         out_exact, static_cast<cudaStream_t>(stream));
        },
        h->error, h->code);
}

int bm25_merge_topk(const float *scores, const int32_t *ids, const int32_t *bases, int64_t q, int32_t shards,
                    int32_t k, int64_t num_docs, int32_t shard_major, float *out_scores, int32_t *out_ids,
                    void *stream)
{
    return Invoke(
        [&] {
            bm25b200::Check(scores && ids && out_scores && out_ids, "Null device buffer");
            bm25b200::Check(q >= 1 && q <= INT32_MAX, "Query count outside [1, 2^31)");
            bm25b200::Check(shards >= 1 && k >= 1 && (int64_t)shards * k <= (int64_t(1) << 30),
                            "Shard count or K outside range");
            bm25b200::Check(num_docs >= 1 && num_docs <= INT32_MAX, "Document count outside [1, 2^31)");
            bm25k::MergeArgs a{scores, ids, bases, (int)q, shards, k, num_docs, out_scores, out_ids, shard_major != 0};
            bm25k::MergeShardsKernel<<<(unsigned)q, bm25k::kMergeThreads, 0, static_cast<cudaStream_t>(stream)>>>(a);
            bm25b200::Cuda(cudaGetLastError(), "merge kernel launch");
        },
        g_create_error, g_create_code);
}

int bm25_set_threshold_model(bm25_handle *h, const float *params, float margin)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            h->engine->SetThresholdModel(params, margin);
        },
        h->error, h->code);
}

int bm25_query_features_device(bm25_handle *h, const int64_t *qoffsets, const int32_t *words, int64_t q, int32_t k,
                               float *features, float *safe, void *stream)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            h->engine->QueryFeaturesDevice(qoffsets, words, q, k, features, safe, static_cast<cudaStream_t>(stream));
        },
        h->error, h->code);
}

int bm25_search_stats(bm25_handle *h, uint64_t *out, int32_t reset)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            h->engine->SearchStats(out, reset != 0);
        },
        h->error, h->code);
}

int bm25_device_status(bm25_handle *h, uint32_t *status)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            bm25b200::Check(status != nullptr, "Null status output");
            *status = h->engine->DeviceStatus();
        },
        h->error, h->code);
}

int bm25_kernel_timing(bm25_handle *h, int32_t enable)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            h->engine->KernelTiming(enable != 0);
        },
        h->error, h->code);
}

int bm25_kernel_times(bm25_handle *h, float *ms, int64_t capacity, int64_t *count)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            bm25b200::Check(count != nullptr, "Null count output");
            *count = h->engine->KernelTimes(ms, capacity);
        },
        h->error, h->code);
}

int bm25_close(bm25_handle *h)
{
    if (!h)
        return BM25_OK;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (h->engine) {
                h->engine->Close();
                h->engine.reset();
            }
        },
        h->error, h->code);
}

void bm25_destroy(bm25_handle *h)
{
    if (!h)
        return;
    bm25_close(h);
    delete h;
}

int bm25_get_tuning(bm25_handle *h, bm25_tuning *t)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            bm25b200::Check(t != nullptr, "Null tuning");
            h->engine->GetTuning(t);
        },
        h->error, h->code);
}

int bm25_set_tuning(bm25_handle *h, const bm25_tuning *t)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            bm25b200::Check(t != nullptr, "Null tuning");
            h->engine->SetTuning(*t);
        },
        h->error, h->code);
}

int bm25_prepare_batch_graphs(bm25_handle *h, int32_t max_batch, int32_t learned)
{
    if (!h)
        return BM25_ERR_ILLEGAL_OPERATION;
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 is not initialized");
            h->engine->PrepareBatchGraphs(max_batch, learned != 0);
        },
        h->error, h->code);
}

int bm25_test_inject(bm25_handle *h, int32_t what)
{
    if (!h) {
        if (what != BM25_INJECT_HOST_FAILURE)
            return BM25_ERR_INVALID_PARAM;
        bm25b200::g_fail_next.store(1);
        return BM25_OK;
    }
    std::lock_guard<std::mutex> guard(h->mutex);
    return Invoke(
        [&] {
            if (!h->engine)
                throw bm25b200::InvalidState("BM25 session is closed");
            h->engine->Inject(what);
        },
        h->error, h->code);
}

int bm25_last_error(const bm25_handle *h, char *buffer, size_t length, int64_t *code)
{
    const std::string &e = h ? h->error : g_create_error;
    if (code)
        *code = h ? h->code : g_create_code;
    if (buffer && length) {
        std::snprintf(buffer, length, "%s", e.c_str());
    }
    return BM25_OK;
}

int bm25_get_info(const bm25_handle *h, bm25_info *info)
{
    if (!h || !info)
        return BM25_ERR_INVALID_PARAM;
    if (!h->engine)
        return BM25_ERR_ILLEGAL_OPERATION;
    h->engine->Info(info);
    return BM25_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Search with no device allocation (bm25_search_csc_static).
//
// For callers that hold their CSC index in device memory they manage
// themselves and may not allocate: code running where cudaMalloc is not
// allowed or not wanted (inside a framework that owns every byte of device
// memory through its own pool, a serving loop that forbids allocation after
// start-up, or a process whose allocator is locked down).  All per-search
// scratch lives in the fixed array below; every GPU that loads this library
// holds it until the process exits.

namespace {
constexpr size_t kStaticScratchBytes = size_t(16) << 20;  // 16 MiB, the largest Search this path accepts
constexpr size_t kStaticHeadBytes = 256;                  // work counter + status word
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

struct StaticDevice {
    bool ready = false;
    unsigned char *scratch = nullptr;  // device address of g_static_scratch on this device
    int sms = 0;
    int grid[3] = {0, 0, 0};  // streaming-kernel CTAs for tile_docs 2048, 4096, 8192
};
std::mutex g_static_mutex;
StaticDevice g_static_devices[64];
// Host word each device's status is copied into: page-locked once per device at set-up
// (cudaHostRegister of this static array; nothing is allocated), so the copy is a plain DMA.
alignas(4096) unsigned g_static_status[64][1024];

// Puts the caller's current device back on every exit of the allocation-free Search.
struct DeviceRestore {
    int device = -1;
    DeviceRestore() { (void)cudaGetDevice(&device); }
    ~DeviceRestore()
    {
        if (device >= 0)
            (void)cudaSetDevice(device);
    }
};

size_t AlignUp(size_t n, size_t a) { return (n + a - 1) / a * a; }
size_t StaticSmem(int tile_docs)
{
    return (size_t)tile_docs * sizeof(float) + 2 * (size_t)4 * bm25k::kChunk * sizeof(int) +
           sizeof(bm25k::StreamShared);
}

void StaticRaiseSmem(size_t bytes)
{
    bm25b200::RaiseSmemCap(reinterpret_cast<const void *>(bm25k::StreamSearchKernel), bytes);
}

// Once per device, with that device current: the device address of the
// scratch array (its host-side name is only a stand-in), kernel attributes and
// occupancy.  Must not run inside a stream capture.
void StaticSetup(int device, StaticDevice &d)
{
    if (d.ready)
        return;
    void *ptr = nullptr;
    bm25b200::Cuda(cudaGetSymbolAddress(&ptr, g_static_scratch), "cudaGetSymbolAddress(static scratch)");
    bm25b200::Cuda(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, device), "SM count");
    StaticRaiseSmem(StaticSmem(8192));
    for (int i = 0; i < 3; ++i) {
        int per_sm = 0;
        bm25b200::Cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bm25k::StreamSearchKernel,
                                                                     bm25k::kStreamThreads, StaticSmem(2048 << i)),
                       "occupancy");
        d.grid[i] = std::max(1, per_sm) * d.sms;
    }
    const cudaError_t reg = cudaHostRegister(g_static_status[device], sizeof(g_static_status[device]),
                                             cudaHostRegisterDefault);
    if (reg != cudaSuccess && reg != cudaErrorHostMemoryAlreadyRegistered)
        bm25b200::Cuda(reg, "cudaHostRegister(static status word)");
    d.scratch = static_cast<unsigned char *>(ptr);
    d.ready = true;
}

// Scratch layout of one Search: head | threshold[q] | cand_count[q] | slots[q][32] |
// cand_scores[q][cap] | cand_ids[q][cap] | plan[num_words][tiles]; everything before cand_scores
// starts at zero.
struct StaticLayout {
    long long cand_cap;
    size_t off_thr, off_cnt, off_slots, off_cs, off_ci, off_plan, need;
};
StaticLayout StaticLayoutFor(int64_t q, int k, int64_t num_words, int64_t tiles)
{
    StaticLayout l;
    l.cand_cap = tiles * bm25k::kConsumerWarps * k;
    l.off_thr = kStaticHeadBytes;
    l.off_cnt = AlignUp(l.off_thr + (size_t)q * 4, 16);
    l.off_slots = AlignUp(l.off_cnt + (size_t)q * 4, 16);
    l.off_cs = AlignUp(l.off_slots + (size_t)q * 32 * 4, 16);
    l.off_ci = AlignUp(l.off_cs + (size_t)q * l.cand_cap * 4, 16);
    l.off_plan = AlignUp(l.off_ci + (size_t)q * l.cand_cap * 4, 16);
    l.need = l.off_plan + (size_t)std::max<int64_t>(1, num_words) * tiles * sizeof(bm25k::PlanEntry);
    return l;
}

// Tile of the streaming kernel for num_docs on `sms` SMs: the smallest power of two from 2048 that
// gives each SM at most one tile, capped at 8192.
int StaticTile(int64_t num_docs, int sms, int *index)
{
    int tile = 2048, ti = 0;
    const int64_t per_sm = (num_docs + sms - 1) / sms;
    while (tile < per_sm && tile < 8192) {
        tile <<= 1;
        ++ti;
    }
    *index = ti;
    return tile;
}
} // namespace

extern "C" int bm25_search_csc_static(const int64_t *indptr, const int32_t *indices, const float *data,
                                      int64_t vocab, int64_t num_docs, const int64_t *qoffsets,
                                      const int32_t *words, int64_t q, int64_t num_words, int32_t k,
                                      float *out_scores, int32_t *out_ids, void *stream, int32_t device_id)
{
    return Invoke(
        [&] {
            using bm25b200::Check;
            using bm25b200::Cuda;
            Check(indptr && indices && data && qoffsets && words && out_scores && out_ids, "Null device buffer");
            Check(reinterpret_cast<uintptr_t>(indices) % 16 == 0 && reinterpret_cast<uintptr_t>(data) % 16 == 0,
                  "indices and data must be 16-byte aligned");
            Check(vocab >= 1 && vocab < INT32_MAX && num_docs >= 1 && num_docs <= INT32_MAX,
                  "Empty or oversized index");
            Check(q >= 1 && q <= 65535 && num_words >= 0 && num_words <= 16777216, "Query batch out of range");
            Check(k >= 1 && k <= bm25k::kMaxSmallK && k <= num_docs, "K outside [1, min(32, N)]");
            Check(device_id >= 0 && device_id < 64, "device_id out of range");
            // The need falls as the tile grows: with the largest tile first, so a Search that can never
            // fit is rejected before any CUDA call, then with the device's own tile.
            const auto check_need = [&](int64_t tiles) {
                const StaticLayout l = StaticLayoutFor(q, k, num_words, tiles);
                if (l.need > kStaticScratchBytes)
                    throw bm25b200::InvalidArgument("Search needs " + std::to_string(l.need) +
                                                    " bytes of scratch; the allocation-free path holds " +
                                                    std::to_string(kStaticScratchBytes));
                return l;
            };
            check_need((num_docs + 8191) / 8192);
            const DeviceRestore restore;
            Cuda(cudaSetDevice(device_id), "cudaSetDevice");
            StaticDevice *dev;
            {
                std::lock_guard<std::mutex> guard(g_static_mutex);
                dev = &g_static_devices[device_id];
                StaticSetup(device_id, *dev);
            }
            int ti = 0;
            const int tile = StaticTile(num_docs, dev->sms, &ti);
            const int64_t tiles = (num_docs + tile - 1) / tile;
            const StaticLayout layout = check_need(tiles);
            const long long cand_cap = layout.cand_cap;
            const size_t off_thr = layout.off_thr, off_cnt = layout.off_cnt, off_slots = layout.off_slots,
                         off_cs = layout.off_cs, off_ci = layout.off_ci, off_plan = layout.off_plan;
            StaticRaiseSmem(StaticSmem(tile));
            unsigned char *base = dev->scratch;
            cudaStream_t s = static_cast<cudaStream_t>(stream);
            bm25k::StreamArgs sa{};
            sa.indptr = reinterpret_cast<const long long *>(indptr);
            sa.indices = indices;
            sa.data = data;
            sa.qoffsets = reinterpret_cast<const long long *>(qoffsets);
            sa.words = words;
            sa.vocab = (int)vocab;
            sa.num_docs = (int)num_docs;
            sa.tile_docs = tile;
            sa.tiles = (int)tiles;
            sa.k = k;
            sa.q = (int)q;
            sa.word_cap = std::max<int64_t>(1, num_words);
            sa.ctrl = reinterpret_cast<bm25k::StreamCtrl *>(base);
            sa.status = reinterpret_cast<unsigned *>(base + 64);
            sa.threshold = reinterpret_cast<unsigned *>(base + off_thr);
            sa.cand_count = reinterpret_cast<unsigned *>(base + off_cnt);
            sa.tslots = reinterpret_cast<unsigned *>(base + off_slots);
            sa.cand_scores = reinterpret_cast<float *>(base + off_cs);
            sa.cand_ids = reinterpret_cast<int *>(base + off_ci);
            sa.cand_cap = cand_cap;
            sa.plan = reinterpret_cast<bm25k::PlanEntry *>(base + off_plan);
            sa.stages = 4;
            sa.out_scores = out_scores;
            sa.out_ids = out_ids;
            // The array keeps the previous call's contents: clear what must start at zero.
            Cuda(cudaMemsetAsync(base, 0, off_cs, s), "clear static scratch");
            // no directory: every word takes the one-pass path of PlanKernel
            bm25k::PlanKernel<<<bm25k::PlanGrid(num_words, (int)tiles, dev->sms), bm25k::kPlanThreads, 0, s>>>(sa);
            Cuda(cudaGetLastError(), "plan kernel launch");
            const int grid = (int)std::min<long long>(dev->grid[ti], (q * tiles + bm25k::kTaskBatch - 1) /
                                                                         bm25k::kTaskBatch);
            bm25k::StreamSearchKernel<<<std::max(grid, 1), bm25k::kStreamThreads, StaticSmem(tile), s>>>(sa);
            Cuda(cudaGetLastError(), "stream kernel launch");
            bm25k::FinalSelectKernel<<<(int)q, bm25k::kFinalThreads, 0, s>>>(sa);
            Cuda(cudaGetLastError(), "final kernel launch");
            volatile unsigned *slot = g_static_status[device_id];
            Cuda(cudaMemcpyAsync(g_static_status[device_id], sa.status, sizeof(unsigned), cudaMemcpyDeviceToHost, s),
                 "status D2H");
            Cuda(cudaStreamSynchronize(s), "complete static Search");
            const unsigned status = *slot;
            if (status && !(status & ~(unsigned)(bm25k::kStatusBadWord | bm25k::kStatusBadQuery)))
                throw bm25b200::InvalidArgument("Invalid word ID or query offsets in the device query packet, status=" +
                                                std::to_string(status));
            if (status)
                throw bm25b200::DeviceError(0, "Device reported invalid Search state, status=" + std::to_string(status));
        },
        g_create_error, g_create_code);
}
