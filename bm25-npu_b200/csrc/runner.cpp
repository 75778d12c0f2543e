// bm25_runner: the benchmark runner process boundary of the reference
// (test/ascendhost/bm25/benchmark.cpp:31-110, benchmark_common.h:49-139) on this
// engine, for the Python entry points that drive a runner binary.
//
//   bm25_runner INDEX A_RAW B_RAW OUTPUT DEVICE VENDORS K Q WORDS WARMUP REPEATS REF_A REF_B
//   bm25_runner --memory DEVICE OUT
//
// INDEX holds the reference's index files (term_offsets.bin, posting_doc_ids.bin,
// posting_tf.bin, doc_norm.bin, idf.bin; standalone/resident_index.py:12-18), A_RAW
// and B_RAW raw query-ID files ("BM25_QUERY_IDS_V1 Q", then per query its word
// count and word ids), REF_A / REF_B the original-document oracle's full score rows
// (expected_scores.bin, Q x N FP32).  VENDORS is unused (no vendor libraries on
// this backend).  The session is built with the reference's contribution
// constant (k1 1.2, f32(k1 + 1) = 2.2F).
//
// As the reference runner: one checkpoint Search of A and of B before the
// measurement (before_A, before_B: top_scores.bin, top_ids.bin, check.json),
// WARMUP alternating A/B - B/A cycles whose top-K bits must equal the
// checkpoints, REPEATS measured cycles timed by the caller's steady clock around
// each bm25_search call (the same bit check, outside the timer), then the after_A
// and after_B checkpoints.  check.json compares the checkpoint with the strict
// top-K (score desc, id asc, zero fill by id) of the REF rows bit for bit.
// OUTPUT/benchmark_session.json records the samples and the engine's facts
// under this backend's own contract name.
#include "bm25_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

namespace fs = std::filesystem;
using Clock = std::chrono::steady_clock;

namespace {

void Check(bool ok, const std::string &message)
{
    if (!ok)
        throw std::runtime_error(message);
}

int64_t Number(const char *text, int64_t low, int64_t high)
{
    size_t used = 0;
    const long long value = std::stoll(text, &used);
    Check(used == std::strlen(text) && value >= low && value <= high, std::string("Invalid numeric argument: ") + text);
    return value;
}

template <class T> std::vector<T> ReadArray(const fs::path &path)
{
    std::ifstream f(path, std::ios::binary);
    Check(bool(f), "Cannot open " + path.string());
    const auto bytes = fs::file_size(path);
    Check(bytes % sizeof(T) == 0, "Truncated file " + path.string());
    std::vector<T> out(bytes / sizeof(T));
    Check(bool(f.read(reinterpret_cast<char *>(out.data()), (std::streamsize)bytes)), "Cannot read " + path.string());
    return out;
}

template <class T> void WriteArray(const fs::path &path, const std::vector<T> &v)
{
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char *>(v.data()), (std::streamsize)(v.size() * sizeof(T)));
    Check(bool(f), "Cannot write " + path.string());
}

using Queries = std::vector<std::vector<int32_t>>;

Queries LoadQueries(const std::string &path)
{
    std::ifstream f(path);
    std::string magic;
    int64_t q = 0;
    Check(bool(f >> magic >> q) && magic == "BM25_QUERY_IDS_V1" && q >= 1 && q <= 10000,
          "Invalid raw query ID file header: " + path);
    Queries out((size_t)q);
    size_t total = 0;
    for (auto &row : out) {
        int64_t n = 0;
        Check(bool(f >> n) && n >= 0 && n <= 16777216 && total + (size_t)n <= 16777216,
              "Invalid raw query length: " + path);
        total += (size_t)n;
        for (int64_t i = 0; i < n; ++i) {
            int64_t w = 0;
            Check(bool(f >> w) && w >= 0 && w < INT32_MAX, "Invalid raw query word ID: " + path);
            row.push_back((int32_t)w);
        }
    }
    f >> std::ws;
    Check(f.eof(), "Unexpected trailing raw query data: " + path);
    return out;
}

struct Result {
    std::vector<float> scores;
    std::vector<int32_t> ids;
};

struct Engine {
    bm25_handle *h = nullptr;
    int64_t q = 0, words = 0;
    int32_t k = 0;

    Result Search(const Queries &queries) const
    {
        Check((int64_t)queries.size() == q, "Query batch size differs from Q");
        std::vector<int64_t> offsets(1, 0);
        std::vector<int32_t> w;
        for (const auto &row : queries) {
            w.insert(w.end(), row.begin(), row.end());
            offsets.push_back((int64_t)w.size());
        }
        if (w.empty())
            w.push_back(0);
        Result r{std::vector<float>((size_t)q * k), std::vector<int32_t>((size_t)q * k)};
        const int st = bm25_search(h, offsets.data(), w.data(), q, k, r.scores.data(), r.ids.data());
        if (st != BM25_OK) {
            char buf[1024];
            int64_t code = 0;
            bm25_last_error(h, buf, sizeof(buf), &code);
            throw std::runtime_error(std::string("Search failed: ") + buf);
        }
        return r;
    }
};

bool Better(float as, int32_t ai, float bs, int32_t bi) { return as > bs || (as == bs && ai < bi); }

// Strict top-K of one full score row (score desc, id asc; zero scores fill by ascending id).
void StrictTopK(const float *row, int64_t n, int32_t k, float *out_s, int32_t *out_i)
{
    std::vector<int32_t> pos;
    for (int64_t d = 0; d < n; ++d)
        if (row[d] > 0.0f)
            pos.push_back((int32_t)d);
    const size_t take = std::min(pos.size(), (size_t)k);
    std::partial_sort(pos.begin(), pos.begin() + take, pos.end(),
                      [&](int32_t a, int32_t b) { return Better(row[a], a, row[b], b); });
    int32_t r = 0;
    for (; r < (int32_t)take; ++r) {
        out_s[r] = row[pos[r]];
        out_i[r] = pos[r];
    }
    for (int64_t d = 0; r < k && d < n; ++d)
        if (!(row[d] > 0.0f)) {
            out_s[r] = 0.0f;
            out_i[r] = (int32_t)d;
            ++r;
        }
}

bool SameBits(const Result &a, const Result &b)
{
    return a.scores.size() == b.scores.size() &&
           std::memcmp(a.scores.data(), b.scores.data(), a.scores.size() * sizeof(float)) == 0 && a.ids == b.ids;
}

void SaveCheckpoint(const fs::path &dir, const Result &r, const fs::path &ref, int64_t q, int32_t k, int64_t docs)
{
    Check(fs::create_directory(dir), "Cannot create checkpoint " + dir.string());
    WriteArray(dir / "top_scores.bin", r.scores);
    WriteArray(dir / "top_ids.bin", r.ids);
    Check(fs::file_size(ref) == (uintmax_t)(q * docs * 4), "Reference score rows size mismatch: " + ref.string());
    const auto rows = ReadArray<float>(ref);
    int64_t mismatched = 0;
    std::vector<float> s(k);
    std::vector<int32_t> id(k);
    for (int64_t i = 0; i < q; ++i) {
        StrictTopK(rows.data() + i * docs, docs, k, s.data(), id.data());
        if (std::memcmp(s.data(), r.scores.data() + i * k, (size_t)k * 4) != 0 ||
            std::memcmp(id.data(), r.ids.data() + i * k, (size_t)k * 4) != 0)
            ++mismatched;
    }
    std::ofstream f(dir / "check.json");
    f << "{\"status\":\"" << (mismatched ? "mismatch" : "strict_topk_bits_equal_original_document_oracle")
      << "\",\"queries\":" << q << ",\"mismatched_queries\":" << mismatched << "}\n";
    Check(bool(f), "Cannot write check.json");
    Check(mismatched == 0, "Top-K differs from the original-document oracle in " + dir.string());
}

int Memory(int argc, char **argv)
{
    Check(argc == 4, "Usage: --memory DEVICE OUT");
    const int device = (int)Number(argv[2], 0, INT32_MAX);
    Check(!fs::exists(argv[3]), "Memory output exists");
    Check(cudaSetDevice(device) == cudaSuccess, "cudaSetDevice failed");
    size_t free = 0, total = 0;
    Check(cudaMemGetInfo(&free, &total) == cudaSuccess && total > 0, "Device memory unavailable");
    std::ofstream f(argv[3]);
    f << "{\"free\":" << free << ",\"total\":" << total << "}\n";
    Check(bool(f), "Cannot write memory report");
    return 0;
}

} // namespace

int main(int argc, char **argv)
{
    try {
        if (argc >= 2 && std::string(argv[1]) == "--memory")
            return Memory(argc, argv);
        Check(argc == 14,
              "Usage: INDEX A_RAW B_RAW OUTPUT DEVICE VENDORS K Q WORDS WARMUP REPEATS REF_A REF_B");
        const fs::path index = fs::absolute(argv[1]), output = fs::absolute(argv[4]);
        Check(!fs::exists(output), "New output required");
        const Queries a = LoadQueries(argv[2]), b = LoadQueries(argv[3]);
        const int device = (int)Number(argv[5], 0, INT32_MAX);
        const int32_t k = (int32_t)Number(argv[7], 1, 1024);
        const int64_t q = Number(argv[8], 1, 10000);
        const int64_t words = Number(argv[9], 0, 16777216);
        const int warm = (int)Number(argv[10], 1, 10000);
        const int repeats = (int)Number(argv[11], 10, 100000);
        const fs::path ref_a = fs::absolute(argv[12]), ref_b = fs::absolute(argv[13]);
        Check(!a.empty() && a.size() == b.size() && a != b && (int64_t)a.size() == q,
              "A/B must be different raw query-ID batches of Q queries");

        const auto cold = Clock::now();
        const auto offsets = ReadArray<int64_t>(index / "term_offsets.bin");
        const auto docs = ReadArray<int32_t>(index / "posting_doc_ids.bin");
        const auto tf = ReadArray<float>(index / "posting_tf.bin");
        const auto norm = ReadArray<float>(index / "doc_norm.bin");
        const auto idf = ReadArray<float>(index / "idf.bin");
        Check(offsets.size() == idf.size() + 1 && !norm.empty(), "Index dimensions differ");
        bm25_options o;
        bm25_default_options(&o);
        o.device_id = device;
        o.max_k = k;
        o.query_capacity = (int32_t)q;
        o.word_capacity = (int32_t)words;
        Engine e;
        e.q = q;
        e.k = k;
        e.words = words;
        if (bm25_create_lazy(offsets.data(), docs.data(), tf.data(), norm.data(), idf.data(), (int64_t)idf.size(),
                             (int64_t)norm.size(), 1.2f, &o, &e.h) != BM25_OK) {
            char buf[1024];
            int64_t code = 0;
            bm25_last_error(nullptr, buf, sizeof(buf), &code);
            throw std::runtime_error(std::string("Session creation failed: ") + buf);
        }
        const double cold_ms = std::chrono::duration<double, std::milli>(Clock::now() - cold).count();
        const int64_t ndocs = (int64_t)norm.size();
        Check(fs::create_directories(output), "Cannot create output");

        std::cout << "stage=before_measurement_checkpoints" << std::endl;
        const Result gold_a = e.Search(a);
        SaveCheckpoint(output / "before_A", gold_a, ref_a, q, k, ndocs);
        const Result gold_b = e.Search(b);
        SaveCheckpoint(output / "before_B", gold_b, ref_b, q, k, ndocs);
        const Queries *sets[2] = {&a, &b};
        const Result *gold[2] = {&gold_a, &gold_b};
        std::cout << "stage=warmup_alternating_AB_BA" << std::endl;
        for (int c = 0; c < warm; ++c)
            for (int slot = 0; slot < 2; ++slot) {
                const int which = slot ^ (c & 1);
                Check(SameBits(e.Search(*sets[which]), *gold[which]), "Alternating Search Top-K bits changed");
            }
        struct Sample {
            int cycle, which;
            double ms;
        };
        std::vector<Sample> samples;
        std::cout << "stage=measure" << std::endl;
        for (int c = 0; c < repeats; ++c)
            for (int slot = 0; slot < 2; ++slot) {
                const int which = slot ^ (c & 1);
                const auto start = Clock::now();
                const Result r = e.Search(*sets[which]);
                const double ms = std::chrono::duration<double, std::milli>(Clock::now() - start).count();
                Check(SameBits(r, *gold[which]), "Alternating Search Top-K bits changed");
                samples.push_back({c, which, ms});
            }
        std::cout << "stage=after_measurement_checkpoints" << std::endl;
        const Result last_a = e.Search(a);
        Check(SameBits(last_a, gold_a), "Alternating Search Top-K bits changed");
        SaveCheckpoint(output / "after_A", last_a, ref_a, q, k, ndocs);
        const Result last_b = e.Search(b);
        Check(SameBits(last_b, gold_b), "Alternating Search Top-K bits changed");
        SaveCheckpoint(output / "after_B", last_b, ref_b, q, k, ndocs);

        bm25_info info{};
        bm25_get_info(e.h, &info);
        size_t words_a = 0;
        for (const auto &row : a)
            words_a += row.size();
        std::ofstream rec(output / "benchmark_session.json");
        rec << std::setprecision(17) << "{\n\"status\":\"search_benchmark_calls_completed_checks_passed\",\n"
            << "\"backend\":\"b200\",\"contract\":\"b200_tile_group_exact_v1\",\"docs\":" << ndocs
            << ",\"queries\":" << q << ",\"k\":" << k << ",\"partitions\":" << info.tiles
            << ",\"capacity_queries\":" << q << ",\"capacity_words\":" << words << ",\n"
            << "\"input_contract\":\"raw_grouped_INT32_word_IDs_in_CPU_memory\",\n"
            << "\"timer_policy\":\"caller steady_clock before Search through returned CPU Top-K\",\n"
            << "\"index_bytes\":" << info.index_bytes << ",\"device_bytes\":" << info.device_bytes
            << ",\"cold_init_ms\":" << cold_ms << ",\"checkpoint_search_calls\":4,\n"
            << "\"warmup_cycles\":" << warm << ",\"warmup_search_calls\":" << 2 * warm
            << ",\"measured_cycles\":" << repeats << ",\"measured_search_calls\":" << samples.size()
            << ",\"measured_topk_bit_checks\":" << samples.size() << ",\n"
            << "\"device\":" << device << ",\"tile_docs\":" << info.tile_docs << ",\"kernel\":" << info.kernel
            << ",\"graph_replays\":" << info.graph_replays << ",\"searches\":" << info.searches
            << ",\"example_query_words\":" << words_a << ",\n\"samples\":[";
        for (size_t i = 0; i < samples.size(); ++i)
            rec << (i ? "," : "") << "{\"cycle\":" << samples[i].cycle << ",\"case\":\""
                << (samples[i].which ? "B" : "A") << "\",\"call_wall_ms\":" << samples[i].ms << "}";
        rec << "]\n}\n";
        rec.close();
        Check(bool(rec), "Cannot save benchmark session");
        Check(bm25_close(e.h) == BM25_OK, "Close failed");
        bm25_destroy(e.h);
        return 0;
    } catch (const std::exception &error) {
        std::cerr << "FAILED: " << error.what() << std::endl;
        return 1;
    }
}
