// C entry points around the reference's own CPU search sessions -- TEST INFRASTRUCTURE ONLY.
//
// Compiled (by oracle/Makefile) against the unmodified reference headers
//   feature_retrieval/src/ascendfaiss/test/ascendhost/bm25/reference/cpu_index_search.h
//   feature_retrieval/src/ascendfaiss/test/ascendhost/bm25/reference/cpu_directory_search.h
// into oracle/_ref/libref_cpu.so.  The reference code keeps its own limits
// (K <= 32, k1 = 1.2 hard-coded as 2.2F, Q * N <= INT32_MAX).  This file only
// converts flat arrays into the reference's Index / Queries types and back.
#include "test/ascendhost/bm25/reference/cpu_directory_search.h"
#include "test/ascendhost/bm25/reference/cpu_index_search.h"

#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>
#include <vector>

namespace {
struct RefSession {
    std::unique_ptr<bm25cpu::Index> index;
    std::unique_ptr<bm25cpu::CpuSearchSession> plain;
    std::unique_ptr<bm25cpu::DirectoryCpuSearchSession> directory;
    int64_t k = 0;
};

void SetError(char *err, size_t len, const char *what)
{
    if (err && len) {
        std::snprintf(err, len, "%s", what);
    }
}

bm25cpu::Queries Unpack(const int64_t *qoffsets, const int32_t *words, int64_t q)
{
    bm25cpu::Queries rows(static_cast<size_t>(q));
    for (int64_t i = 0; i < q; ++i)
        rows[i].assign(words + qoffsets[i], words + qoffsets[i + 1]);
    return rows;
}
} // namespace

extern "C" {

// Builds the reference Index (validated by its constructor) and one CPU session.
// mode 0: CpuSearchSession (lower_bound shards), mode 1: DirectoryCpuSearchSession.
void *ref_session_create(const int64_t *offsets, int64_t vocab, const int32_t *docs, const float *tf, int64_t postings,
                         const float *norm, int64_t num_docs, const float *idf, int threads, int64_t k,
                         int64_t shards, int64_t query_capacity, int64_t word_capacity, int mode, char *err,
                         size_t errlen)
{
    try {
        auto s = std::make_unique<RefSession>();
        s->index = std::make_unique<bm25cpu::Index>(
            std::vector<int64_t>(offsets, offsets + vocab + 1), std::vector<int32_t>(docs, docs + postings),
            std::vector<float>(tf, tf + postings), std::vector<float>(norm, norm + num_docs),
            std::vector<float>(idf, idf + vocab));
        s->k = k;
        if (mode == 0)
            s->plain = std::make_unique<bm25cpu::CpuSearchSession>(*s->index, threads, k, shards,
                                                                   static_cast<size_t>(query_capacity),
                                                                   static_cast<size_t>(word_capacity));
        else
            s->directory = std::make_unique<bm25cpu::DirectoryCpuSearchSession>(
                *s->index, threads, k, shards, static_cast<size_t>(query_capacity),
                static_cast<size_t>(word_capacity));
        return s.release();
    } catch (const std::exception &e) {
        SetError(err, errlen, e.what());
        return nullptr;
    }
}

// Runs Search; returns 0 on success.  ms receives the reference's own timer.
int ref_session_search(void *handle, const int64_t *qoffsets, const int32_t *words, int64_t q, float *out_scores,
                       int32_t *out_ids, double *ms, char *err, size_t errlen)
{
    try {
        auto *s = static_cast<RefSession *>(handle);
        const auto queries = Unpack(qoffsets, words, q);
        const auto result = s->plain ? s->plain->Search(queries) : s->directory->Search(queries);
        std::memcpy(out_scores, result.scores.data(), result.scores.size() * sizeof(float));
        std::memcpy(out_ids, result.ids.data(), result.ids.size() * sizeof(int32_t));
        if (ms)
            *ms = result.searchMs;
        return 0;
    } catch (const std::exception &e) {
        SetError(err, errlen, e.what());
        return 1;
    }
}

// Full per-document scores of the last Search (the reference's DebugScores).
int ref_session_debug_scores(void *handle, int64_t q, float *out, int64_t num_docs)
{
    try {
        auto *s = static_cast<RefSession *>(handle);
        const auto v = s->plain ? s->plain->DebugScores(static_cast<size_t>(q))
                                : s->directory->DebugScores(static_cast<size_t>(q));
        if (static_cast<int64_t>(v.size()) != q * num_docs)
            return 1;
        std::memcpy(out, v.data(), v.size() * sizeof(float));
        return 0;
    } catch (const std::exception &) {
        return 1;
    }
}

int ref_session_threads(void *handle)
{
    auto *s = static_cast<RefSession *>(handle);
    return s->plain ? s->plain->actualThreads : s->directory->actualThreads;
}

void ref_session_destroy(void *handle) { delete static_cast<RefSession *>(handle); }
}
