/*
 * AscendIndexBm25.h -- C++ Search facade over the B200 engine's C ABI (bm25_b200.h).
 *
 * Same class, namespaces, method names, argument meaning and error behaviour
 * as the reference's SDK facade
 *   feature_retrieval/src/ascendfaiss/ascendhost/include/index/AscendIndexBm25.h:37-57
 * so a caller switches by changing the include path and the library it links:
 *   - Init copies and validates the index; a failed Init leaves the object
 *     uninitialised; a second Init fails with ILLEGAL_OPERATION.
 *   - Search replaces `result` only on success; input errors return
 *     INVALID_PARAM and the object stays usable; a device error returns
 *     INNER_ERROR and poisons the session (later Searches: ILLEGAL_OPERATION).
 *   - Close is idempotent; on failure it keeps its state so it can be retried.
 *   - Every call on one object is serialised by its own mutex.
 * Differences, all from the platform: Bm25Config has no ACL context,
 * resources or operator vendor directory; it takes an optional CUDA stream and
 * the BM25 k1 used to turn the lazy index into posting scores (1.2 = the
 * reference's 2.2F literal).  Built into libbm25_facade.so (C++17).
 */
#ifndef BM25_B200_ASCEND_INDEX_BM25_H
#define BM25_B200_ASCEND_INDEX_BM25_H

#include <array>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace ascend {
/* IndexSDK keeps the numeric APP_ERR values in common/ErrorCode.h, which the
 * reference does not ship; these local values are unpinned. */
using APP_ERROR = int;
constexpr APP_ERROR APP_ERR_OK = 0;
constexpr APP_ERROR APP_ERR_INVALID_PARAM = 2001;
constexpr APP_ERROR APP_ERR_ILLEGAL_OPERATION = 2002;
constexpr APP_ERROR APP_ERR_INNER_ERROR = 2003;

namespace bm25 {
/* Exception types of common/bm25/error.h:8-31. */
struct InvalidArgument : std::runtime_error {
    explicit InvalidArgument(const std::string &m) : std::runtime_error(m) {}
};
struct InvalidState : std::runtime_error {
    explicit InvalidState(const std::string &m) : std::runtime_error(m) {}
};
struct DeviceError : std::runtime_error {
    DeviceError(const std::string &m, int64_t code) : std::runtime_error(m), code_(code) {}
    int64_t GetCode() const noexcept { return code_; }

  private:
    int64_t code_;
};

/* ErrorInfo of common/bm25/error_info.h:8-20; aclCode carries the CUDA error (or 0). */
struct ErrorInfo {
    int64_t aclCode = 0;
    std::array<char, 1024> message{};
    void Set(const char *text, int64_t code = 0) noexcept
    {
        aclCode = code;
        message.fill('\0');
        if (text)
            std::strncpy(message.data(), text, message.size() - 1);
    }
};

/* The resident lazy index of common/bm25/index_data.h:9-42, validated on
 * construction with the same rules and messages (throws InvalidArgument). */
struct Index {
    std::vector<int64_t> offsets;
    std::vector<int32_t> docs;
    std::vector<float> tf, norm, idf;
    Index(std::vector<int64_t> termOffsets, std::vector<int32_t> postingIds, std::vector<float> termFrequencies,
          std::vector<float> documentNorms, std::vector<float> inverseFrequencies);
};
} // namespace bm25
} // namespace ascend

namespace bm25search {
/* Word ids grouped by query (common/bm25/search_inputs.h:11). */
using Queries = std::vector<std::vector<int32_t>>;
} // namespace bm25search

namespace faiss::ascend {
struct Bm25Config {
    int deviceId = 0;
    uint64_t queryCount = 8;
    uint64_t maxQueryWords = 24;
    uint64_t topK = 10;
    float k1 = 1.2f;
    void *stream = nullptr;  // cudaStream_t; nullptr = the session's own stream
};

struct Bm25SearchResult {
    std::vector<float> scores;
    std::vector<int64_t> labels;
};

class AscendIndexBm25 {
  public:
    AscendIndexBm25();
    ~AscendIndexBm25();
    AscendIndexBm25(const AscendIndexBm25 &) = delete;
    AscendIndexBm25 &operator=(const AscendIndexBm25 &) = delete;
    AscendIndexBm25(AscendIndexBm25 &&) = delete;
    AscendIndexBm25 &operator=(AscendIndexBm25 &&) = delete;

    ::ascend::APP_ERROR Init(const ::ascend::bm25::Index &index, const Bm25Config &config);
    ::ascend::APP_ERROR Search(const ::bm25search::Queries &queries, Bm25SearchResult &result);
    ::ascend::APP_ERROR Close();
    ::ascend::bm25::ErrorInfo GetLastError() const;

  private:
    class Impl;
    std::unique_ptr<Impl> impl_;
};
} // namespace faiss::ascend

#endif
