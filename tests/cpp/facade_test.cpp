// Behaviour of the C++ facade (include/AscendIndexBm25.h), after the
// reference's SDK facade tests (ut/cases/bm25/sdk_facade_tests.cpp):
//   facade_test host               -- lifecycle and input errors, no device work
//   facade_test device DIR Q OUT   -- Init from the index files in DIR, Search the
//                                     packed queries in Q, write scores + labels to OUT,
//                                     checking the error behaviour around it
#include "AscendIndexBm25.h"
#include "bm25_b200.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

using faiss::ascend::AscendIndexBm25;
using faiss::ascend::Bm25Config;
using faiss::ascend::Bm25SearchResult;

static int failures = 0;
#define EXPECT(cond)                                                                                                   \
    do {                                                                                                               \
        if (!(cond)) {                                                                                                 \
            std::fprintf(stderr, "FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond);                                      \
            ++failures;                                                                                                \
        }                                                                                                              \
    } while (0)

template <class T> static std::vector<T> ReadAll(const std::string &path)
{
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f)
        throw std::runtime_error("cannot open " + path);
    const auto n = static_cast<size_t>(f.tellg());
    std::vector<T> v(n / sizeof(T));
    f.seekg(0);
    f.read(reinterpret_cast<char *>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(T)));
    return v;
}

static ascend::bm25::Index Tiny()
{
    // 2 terms, 3 documents
    return ascend::bm25::Index({0, 2, 3}, {0, 2, 1}, {1.f, 2.f, 1.f}, {1.f, 1.2f, 0.9f}, {0.5f, 1.5f});
}

static bool Throws(std::vector<int64_t> o, std::vector<int32_t> d, std::vector<float> tf, std::vector<float> n,
                   std::vector<float> idf, const char *message)
{
    try {
        ascend::bm25::Index bad(o, d, tf, n, idf);
    } catch (const ascend::bm25::InvalidArgument &e) {
        return std::string(e.what()) == message;
    }
    return false;
}

static void HostChecks()
{
    EXPECT(Throws({0, 1}, {0}, {1.f}, {}, {1.f}, "Empty or oversized index"));
    EXPECT(Throws({0, 2}, {0}, {1.f}, {1.f}, {1.f}, "Index dimensions/endpoints differ"));
    EXPECT(Throws({0, 1}, {0}, {1.f}, {0.f}, {1.f}, "Invalid article norm"));
    EXPECT(Throws({0, 1}, {0}, {1.f}, {1.f}, {-1.f}, "Invalid IDF"));
    EXPECT(Throws({0, 2}, {1, 0}, {1.f, 1.f}, {1.f, 1.f}, {1.f}, "Unsorted/duplicate/out-of-range posting ID"));
    EXPECT(Throws({0, 1}, {0}, {1.5f}, {1.f}, {1.f}, "Invalid posting TF"));
    (void)Tiny();

    AscendIndexBm25 index;
    Bm25SearchResult result;
    result.scores = {7.f};
    EXPECT(index.Search({{1}}, result) == ascend::APP_ERR_ILLEGAL_OPERATION);
    EXPECT(result.scores.size() == 1 && result.scores[0] == 7.f);  // untouched on failure
    EXPECT(std::string(index.GetLastError().message.data()) == "BM25 is not initialized");
    EXPECT(index.Close() == ascend::APP_ERR_OK);
    EXPECT(index.Close() == ascend::APP_ERR_OK);
    EXPECT(index.GetLastError().message[0] == '\0');
    Bm25Config bad;
    bad.topK = 33;
    EXPECT(index.Init(Tiny(), bad) == ascend::APP_ERR_INVALID_PARAM);
    bad.topK = 10;
    bad.queryCount = 0;
    EXPECT(index.Init(Tiny(), bad) == ascend::APP_ERR_INVALID_PARAM);
}

static int DeviceRun(const std::string &dir, const std::string &qfile, const std::string &out)
{
    ascend::bm25::Index idx(ReadAll<int64_t>(dir + "/term_offsets.bin"), ReadAll<int32_t>(dir + "/posting_doc_ids.bin"),
                            ReadAll<float>(dir + "/posting_tf.bin"), ReadAll<float>(dir + "/doc_norm.bin"),
                            ReadAll<float>(dir + "/idf.bin"));
    // query file: int64 q, int64 k, float k1 bits as int64, offsets int64[q+1], words int32[...]
    const auto bytes = ReadAll<char>(qfile);
    int64_t head[3];
    std::memcpy(head, bytes.data(), sizeof(head));
    const int64_t q = head[0], k = head[1];
    float k1;
    {
        const int32_t bits = static_cast<int32_t>(head[2]);
        std::memcpy(&k1, &bits, sizeof(k1));
    }
    std::vector<int64_t> offsets(static_cast<size_t>(q) + 1);
    std::memcpy(offsets.data(), bytes.data() + sizeof(head), offsets.size() * sizeof(int64_t));
    std::vector<int32_t> words(static_cast<size_t>(offsets[q]));
    std::memcpy(words.data(), bytes.data() + sizeof(head) + offsets.size() * sizeof(int64_t),
                words.size() * sizeof(int32_t));
    bm25search::Queries queries(static_cast<size_t>(q));
    for (int64_t r = 0; r < q; ++r)
        queries[r].assign(words.begin() + offsets[r], words.begin() + offsets[r + 1]);

    AscendIndexBm25 index;
    Bm25Config config;
    config.queryCount = static_cast<uint64_t>(q);
    config.maxQueryWords = static_cast<uint64_t>(offsets[q]) + 8;
    config.topK = static_cast<uint64_t>(k);
    config.k1 = k1;
    EXPECT(index.Init(idx, config) == ascend::APP_ERR_OK);
    EXPECT(index.Init(idx, config) == ascend::APP_ERR_ILLEGAL_OPERATION);

    Bm25SearchResult result;
    EXPECT(index.Search(queries, result) == ascend::APP_ERR_OK);
    const Bm25SearchResult first = result;
    // input errors leave the session usable and the output untouched
    bm25search::Queries wrong = queries;
    wrong.pop_back();
    EXPECT(index.Search(wrong, result) == ascend::APP_ERR_INVALID_PARAM);
    bm25search::Queries negative = queries;
    negative[0].push_back(-3);
    EXPECT(index.Search(negative, result) == ascend::APP_ERR_INVALID_PARAM);
    EXPECT(std::string(index.GetLastError().message.data()) == "Invalid public word ID");
    bm25search::Queries too_long = queries;
    too_long[0].assign(65, 1);
    EXPECT(index.Search(too_long, result) == ascend::APP_ERR_INVALID_PARAM);
    EXPECT(result.scores == first.scores && result.labels == first.labels);
    EXPECT(index.Search(queries, result) == ascend::APP_ERR_OK);
    EXPECT(result.scores == first.scores && result.labels == first.labels);
    EXPECT(index.Close() == ascend::APP_ERR_OK);
    EXPECT(index.Search(queries, result) == ascend::APP_ERR_ILLEGAL_OPERATION);
    EXPECT(index.Close() == ascend::APP_ERR_OK);

    // a device failure (injected on the host through the engine's test hook, as the reference's
    // facade test mocks a failing session): INNER_ERROR, the output untouched, the session poisoned
    // (later calls ILLEGAL_OPERATION), and Close still succeeds (sdk_facade_tests.cpp:47-56)
    AscendIndexBm25 failing;
    EXPECT(failing.Init(idx, config) == ascend::APP_ERR_OK);
    Bm25SearchResult kept;
    EXPECT(failing.Search(queries, kept) == ascend::APP_ERR_OK);
    const Bm25SearchResult before = kept;
    EXPECT(bm25_test_inject(nullptr, BM25_INJECT_HOST_FAILURE) == BM25_OK);
    EXPECT(failing.Search(queries, kept) == ascend::APP_ERR_INNER_ERROR);
    EXPECT(std::string(failing.GetLastError().message.data()).find("Injected device failure") != std::string::npos);
    EXPECT(kept.scores == before.scores && kept.labels == before.labels);
    EXPECT(failing.Search(queries, kept) == ascend::APP_ERR_ILLEGAL_OPERATION);
    EXPECT(failing.Close() == ascend::APP_ERR_OK);
    EXPECT(failing.Close() == ascend::APP_ERR_OK);

    std::ofstream f(out, std::ios::binary);
    f.write(reinterpret_cast<const char *>(first.scores.data()),
            static_cast<std::streamsize>(first.scores.size() * sizeof(float)));
    f.write(reinterpret_cast<const char *>(first.labels.data()),
            static_cast<std::streamsize>(first.labels.size() * sizeof(int64_t)));
    return 0;
}

int main(int argc, char **argv)
{
    const std::string mode = argc > 1 ? argv[1] : "host";
    if (mode == "host") {
        HostChecks();
    } else if (mode == "device" && argc == 5) {
        DeviceRun(argv[2], argv[3], argv[4]);
    } else {
        std::fprintf(stderr, "usage: facade_test host | device DIR QUERIES OUT\n");
        return 2;
    }
    if (failures)
        std::fprintf(stderr, "%d check(s) failed\n", failures);
    return failures ? 1 : 0;
}
