// C++ SDK facade (include/AscendIndexBm25.h) over the engine's C ABI.
//
// Follows the reference facade
//   feature_retrieval/src/ascendfaiss/ascendhost/src/bm25/AscendIndexBm25.cpp:14-84
// and its error adapter (ascendhost/include/impl/Bm25ErrorAdapter.h:11-45):
// each public call runs under the object's mutex, clears the last error, and
// maps InvalidArgument / InvalidState / DeviceError (or anything else) to
// INVALID_PARAM / ILLEGAL_OPERATION / INNER_ERROR.  The session itself is a
// bm25_handle; its status codes are turned back into those exception types.
#include "AscendIndexBm25.h"
#include "bm25_b200.h"

#include <climits>
#include <cmath>
#include <mutex>
#include <utility>

namespace ascend::bm25 {

static void CheckArgument(bool ok, const char *message)
{
    if (!ok)
        throw InvalidArgument(message);
}

// Validation rules and messages of common/bm25/index_data.h:18-40.
Index::Index(std::vector<int64_t> termOffsets, std::vector<int32_t> postingIds, std::vector<float> termFrequencies,
             std::vector<float> documentNorms, std::vector<float> inverseFrequencies)
    : offsets(std::move(termOffsets)), docs(std::move(postingIds)), tf(std::move(termFrequencies)),
      norm(std::move(documentNorms)), idf(std::move(inverseFrequencies))
{
    CheckArgument(!norm.empty() && !idf.empty() && norm.size() <= INT32_MAX && idf.size() < INT32_MAX &&
                      docs.size() <= INT32_MAX,
                  "Empty or oversized index");
    CheckArgument(offsets.size() == idf.size() + 1 && docs.size() == tf.size() && offsets.front() == 0 &&
                      offsets.back() == static_cast<int64_t>(docs.size()),
                  "Index dimensions/endpoints differ");
    for (float v : norm)
        CheckArgument(std::isfinite(v) && v > 0, "Invalid article norm");
    for (size_t t = 0; t < idf.size(); ++t) {
        CheckArgument(std::isfinite(idf[t]) && idf[t] >= 0, "Invalid IDF");
        const int64_t b = offsets[t], e = offsets[t + 1];
        CheckArgument(b >= 0 && b <= e && e <= static_cast<int64_t>(docs.size()), "Invalid posting bounds");
        for (int64_t p = b; p < e; ++p) {
            CheckArgument(docs[p] >= 0 && static_cast<size_t>(docs[p]) < norm.size() && (p == b || docs[p - 1] < docs[p]),
                          "Unsorted/duplicate/out-of-range posting ID");
            CheckArgument(std::isfinite(tf[p]) && tf[p] >= 1 && tf[p] <= 16777216.0F && std::floor(tf[p]) == tf[p],
                          "Invalid posting TF");
        }
    }
}

} // namespace ascend::bm25

namespace faiss::ascend {

namespace {
namespace err = ::ascend::bm25;

// Re-raises a non-OK C ABI status as the exception type it stands for.
void Raise(int status, const bm25_handle *handle)
{
    if (status == BM25_OK)
        return;
    char message[1024] = {0};
    int64_t code = 0;
    bm25_last_error(handle, message, sizeof(message), &code);
    switch (status) {
    case BM25_ERR_INVALID_PARAM:
        throw err::InvalidArgument(message);
    case BM25_ERR_ILLEGAL_OPERATION:
        throw err::InvalidState(message);
    default:
        throw err::DeviceError(message, code);
    }
}

template <class F> ::ascend::APP_ERROR InvokeSdkOperation(F &&operation, err::ErrorInfo &error) noexcept
{
    error.Set(nullptr);
    try {
        operation();
        return ::ascend::APP_ERR_OK;
    } catch (const err::InvalidArgument &e) {
        error.Set(e.what());
        return ::ascend::APP_ERR_INVALID_PARAM;
    } catch (const err::InvalidState &e) {
        error.Set(e.what());
        return ::ascend::APP_ERR_ILLEGAL_OPERATION;
    } catch (const err::DeviceError &e) {
        error.Set(e.what(), e.GetCode());
        return ::ascend::APP_ERR_INNER_ERROR;
    } catch (const std::exception &e) {
        error.Set(e.what());
        return ::ascend::APP_ERR_INNER_ERROR;
    } catch (...) {
        error.Set("Unknown BM25 failure");
        return ::ascend::APP_ERR_INNER_ERROR;
    }
}
} // namespace

class AscendIndexBm25::Impl {
  public:
    mutable std::mutex mutex;
    err::ErrorInfo error;
    bm25_handle *session = nullptr;
    Bm25Config config;
    std::vector<int64_t> offsets;  // packed query batch, reused
    std::vector<int32_t> words;
    std::vector<float> scores;
    std::vector<int32_t> ids;

    ~Impl()
    {
        if (session)
            bm25_destroy(session);
    }
};

AscendIndexBm25::AscendIndexBm25() : impl_(std::make_unique<Impl>()) {}
AscendIndexBm25::~AscendIndexBm25() = default;

::ascend::APP_ERROR AscendIndexBm25::Init(const ::ascend::bm25::Index &index, const Bm25Config &config)
{
    std::lock_guard<std::mutex> guard(impl_->mutex);
    return InvokeSdkOperation(
        [&] {
            if (impl_->session)
                throw err::InvalidState("BM25 is already initialized; Close before Init");
            err::CheckArgument(config.queryCount >= 1 && config.queryCount <= 65535 && config.topK >= 1 &&
                                   config.topK <= 32 && config.maxQueryWords <= 16777216,
                               "Invalid fixed packet capacity");
            // Index fields are public data: revalidate the caller's snapshot.
            err::Index checked(index.offsets, index.docs, index.tf, index.norm, index.idf);
            bm25_options o;
            bm25_default_options(&o);
            o.device_id = config.deviceId;
            o.max_k = static_cast<int32_t>(config.topK);
            o.query_capacity = static_cast<int64_t>(config.queryCount);
            o.word_capacity = static_cast<int64_t>(config.maxQueryWords);
            o.stream = config.stream;
            bm25_handle *h = nullptr;
            Raise(bm25_create_lazy(checked.offsets.data(), checked.docs.data(), checked.tf.data(), checked.norm.data(),
                                   checked.idf.data(), static_cast<int64_t>(checked.idf.size()),
                                   static_cast<int64_t>(checked.norm.size()), config.k1, &o, &h),
                  nullptr);
            impl_->session = h;
            impl_->config = config;
            impl_->offsets.assign(config.queryCount + 1, 0);
            impl_->scores.resize(config.queryCount * config.topK);
            impl_->ids.resize(config.queryCount * config.topK);
        },
        impl_->error);
}

::ascend::APP_ERROR AscendIndexBm25::Search(const ::bm25search::Queries &queries, Bm25SearchResult &result)
{
    std::lock_guard<std::mutex> guard(impl_->mutex);
    return InvokeSdkOperation(
        [&] {
            if (!impl_->session)
                throw err::InvalidState("BM25 is not initialized");
            const Bm25Config &c = impl_->config;
            // Packing rules of common/bm25/fixed_query_packet.h:29-37, checked before any work.
            err::CheckArgument(queries.size() == c.queryCount, "Fixed session requires its declared query count");
            size_t total = 0;
            for (const auto &row : queries) {
                err::CheckArgument(row.size() <= 64 && row.size() <= c.maxQueryWords - total,
                                   "Query exceeds fixed word/64-term capacity");
                total += row.size();
                for (int32_t w : row)
                    err::CheckArgument(w >= 0 && w < INT32_MAX, "Invalid public word ID");
            }
            impl_->words.clear();
            for (size_t r = 0; r < queries.size(); ++r) {
                impl_->words.insert(impl_->words.end(), queries[r].begin(), queries[r].end());
                impl_->offsets[r + 1] = static_cast<int64_t>(impl_->words.size());
            }
            if (impl_->words.empty())
                impl_->words.push_back(0);  // a valid pointer; qoffsets say there are no words
            Raise(bm25_search(impl_->session, impl_->offsets.data(), impl_->words.data(),
                              static_cast<int64_t>(c.queryCount), static_cast<int32_t>(c.topK), impl_->scores.data(),
                              impl_->ids.data()),
                  impl_->session);
            Bm25SearchResult next;
            next.scores = impl_->scores;
            next.labels.assign(impl_->ids.begin(), impl_->ids.end());
            result = std::move(next);
        },
        impl_->error);
}

::ascend::APP_ERROR AscendIndexBm25::Close()
{
    std::lock_guard<std::mutex> guard(impl_->mutex);
    return InvokeSdkOperation(
        [&] {
            if (impl_->session) {
                Raise(bm25_close(impl_->session), impl_->session);
                bm25_destroy(impl_->session);
                impl_->session = nullptr;
            }
        },
        impl_->error);
}

::ascend::bm25::ErrorInfo AscendIndexBm25::GetLastError() const
{
    std::lock_guard<std::mutex> guard(impl_->mutex);
    return impl_->error;
}

} // namespace faiss::ascend
