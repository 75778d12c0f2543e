// Index builder on the GPU: token ids of every document -> the reference's lazy
// index (term_offsets, posting_doc_ids, posting_tf, doc_norm, idf), the layout of
// standalone/resident_index.py:12-18 built by standalone/large_corpus.py:95-297.
//
// The heavy part runs on the device: one 64-bit key (term << 32 | doc) per token,
// a radix sort (CUB), run-length counts -- each run is one posting, its length the
// term frequency, already in term-major, doc-ascending order -- and the per-term
// offsets.  The per-term idf and per-document norm are computed on the host in
// double precision with the C library's log1p and rounded to FP32 once, as the
// reference's Python does (math.log1p, k1 * (1 - b + b * len / avgdl)), so the
// arrays match the reference's bit for bit.  The eager FP32 scores then come
// from bm25_create_lazy (BuildContributionsKernel).
#include "bm25_b200.h"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_run_length_encode.cuh>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

namespace {

thread_local std::string g_build_error;

struct BuildFailure {
    int status;
    std::string message;
};

void Check(bool ok, int status, const char *message)
{
    if (!ok)
        throw BuildFailure{status, message};
}

void Cuda(cudaError_t e, const char *what)
{
    if (e != cudaSuccess)
        throw BuildFailure{BM25_ERR_INNER_ERROR, std::string(what) + ": " + cudaGetErrorString(e)};
}

// One key per token: term << 32 | document; a token outside [0, vocab) sets *bad.
__global__ void TokenKeysKernel(const long long *doc_offsets, const int *tokens, long long num_docs, long long vocab,
                                unsigned long long *keys, unsigned *bad)
{
    for (long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x; d < num_docs;
         d += (long long)gridDim.x * blockDim.x) {
        for (long long i = doc_offsets[d]; i < doc_offsets[d + 1]; ++i) {
            const int t = tokens[i];
            if (t < 0 || t >= vocab) {
                *bad = 1u;  // the build is refused before the sort
                keys[i] = 0ull;
                continue;
            }
            keys[i] = ((unsigned long long)t << 32) | (unsigned long long)d;
        }
    }
}

// Postings from the runs: document id, term frequency, and the per-term offsets (for every
// run whose term differs from the previous run's, offsets[prev term + 1 .. term] = run index).
__global__ void PostingsKernel(const unsigned long long *unique, const int *counts, long long runs, long long vocab,
                               int *docs, float *tf, long long *offsets)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < runs;
         i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long key = unique[i];
        const long long term = (long long)(key >> 32);
        docs[i] = (int)(key & 0xffffffffull);
        tf[i] = (float)counts[i];
        const long long prev = i == 0 ? -1 : (long long)(unique[i - 1] >> 32);
        for (long long t = prev + 1; t <= term; ++t)
            offsets[t] = i;
        if (i == runs - 1)
            for (long long t = term + 1; t <= vocab; ++t)
                offsets[t] = runs;
    }
}

template <class T> T *DeviceAlloc(std::vector<void *> &owned, size_t count, const char *what)
{
    void *p = nullptr;
    Cuda(cudaMalloc(&p, count * sizeof(T) + 16), what);
    owned.push_back(p);
    return static_cast<T *>(p);
}

} // namespace

extern "C" int bm25_build_index(const int64_t *doc_offsets, const int32_t *tokens, int64_t num_docs, int64_t vocab,
                                double k1, double b, int32_t device_id, int64_t *term_offsets,
                                int32_t *posting_doc_ids, float *posting_tf, float *doc_norm, float *idf,
                                int64_t *postings)
{
    std::vector<void *> owned;
    cudaStream_t s = nullptr;
    int status = BM25_OK;
    try {
        Check(doc_offsets && term_offsets && posting_doc_ids && posting_tf && doc_norm && idf && postings,
              BM25_ERR_INVALID_PARAM, "Null buffer");
        Check(num_docs >= 1 && num_docs < INT32_MAX && vocab >= 1 && vocab < INT32_MAX, BM25_ERR_INVALID_PARAM,
              "Document or vocabulary count outside [1, 2^31)");
        Check(doc_offsets[0] == 0, BM25_ERR_INVALID_PARAM, "Document offsets must start at 0");
        for (int64_t d = 0; d < num_docs; ++d)
            Check(doc_offsets[d + 1] >= doc_offsets[d], BM25_ERR_INVALID_PARAM, "Document offsets must not decrease");
        const int64_t total = doc_offsets[num_docs];
        Check(total >= 1 && total < INT32_MAX, BM25_ERR_INVALID_PARAM, "Token count outside [1, 2^31)");
        Check(tokens != nullptr, BM25_ERR_INVALID_PARAM, "Null token buffer");
        Check(std::isfinite(k1) && k1 >= 0 && std::isfinite(b) && b >= 0 && b <= 1, BM25_ERR_INVALID_PARAM,
              "Invalid k1 or b");
        Cuda(cudaSetDevice(device_id), "cudaSetDevice");
        Cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
        auto *d_off = DeviceAlloc<long long>(owned, num_docs + 1, "cudaMalloc offsets");
        auto *d_tok = DeviceAlloc<int>(owned, total, "cudaMalloc tokens");
        auto *d_keys = DeviceAlloc<unsigned long long>(owned, total, "cudaMalloc keys");
        auto *d_sorted = DeviceAlloc<unsigned long long>(owned, total, "cudaMalloc keys");
        auto *d_unique = DeviceAlloc<unsigned long long>(owned, total, "cudaMalloc runs");
        auto *d_counts = DeviceAlloc<int>(owned, total, "cudaMalloc runs");
        auto *d_runs = DeviceAlloc<long long>(owned, 1, "cudaMalloc run count");
        auto *d_bad = DeviceAlloc<unsigned>(owned, 1, "cudaMalloc status");
        Cuda(cudaMemcpyAsync(d_off, doc_offsets, (num_docs + 1) * sizeof(long long), cudaMemcpyHostToDevice, s),
             "H2D");
        Cuda(cudaMemcpyAsync(d_tok, tokens, total * sizeof(int), cudaMemcpyHostToDevice, s), "H2D");
        Cuda(cudaMemsetAsync(d_bad, 0, sizeof(unsigned), s), "memset");
        const int grid = (int)std::min<long long>((num_docs + 255) / 256, 148 * 32);
        TokenKeysKernel<<<grid, 256, 0, s>>>(d_off, d_tok, num_docs, vocab, d_keys, d_bad);
        Cuda(cudaGetLastError(), "token key kernel launch");
        int end_bit = 32;  // the document bits, then as many term bits as the vocabulary needs
        while (end_bit < 64 && ((unsigned long long)(vocab - 1) >> (end_bit - 32)) != 0)
            ++end_bit;
        size_t sort_bytes = 0, rle_bytes = 0;
        Cuda(cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, d_keys, d_sorted, (int)total, 0, end_bit, s),
             "radix sort size");
        Cuda(cub::DeviceRunLengthEncode::Encode(nullptr, rle_bytes, d_sorted, d_unique, d_counts, d_runs, (int)total,
                                                s),
             "run-length size");
        void *temp = DeviceAlloc<unsigned char>(owned, std::max(sort_bytes, rle_bytes), "cudaMalloc sort scratch");
        size_t temp_bytes = sort_bytes;
        unsigned bad = 0;
        Cuda(cudaMemcpyAsync(&bad, d_bad, sizeof(unsigned), cudaMemcpyDeviceToHost, s), "D2H");
        Cuda(cudaStreamSynchronize(s), "token keys");
        Check(bad == 0, BM25_ERR_INVALID_PARAM, "Token id outside [0, vocab)");
        Cuda(cub::DeviceRadixSort::SortKeys(temp, temp_bytes, d_keys, d_sorted, (int)total, 0, end_bit, s),
             "radix sort");
        temp_bytes = rle_bytes;
        Cuda(cub::DeviceRunLengthEncode::Encode(temp, temp_bytes, d_sorted, d_unique, d_counts, d_runs, (int)total, s),
             "run-length encode");
        long long runs = 0;
        Cuda(cudaMemcpyAsync(&runs, d_runs, sizeof(long long), cudaMemcpyDeviceToHost, s), "D2H");
        Cuda(cudaStreamSynchronize(s), "run-length encode");
        auto *d_docs = DeviceAlloc<int>(owned, runs, "cudaMalloc postings");
        auto *d_tf = DeviceAlloc<float>(owned, runs, "cudaMalloc postings");
        auto *d_toff = DeviceAlloc<long long>(owned, vocab + 1, "cudaMalloc term offsets");
        const int pgrid = (int)std::min<long long>((runs + 255) / 256, 148 * 32);
        PostingsKernel<<<pgrid, 256, 0, s>>>(d_unique, d_counts, runs, vocab, d_docs, d_tf, d_toff);
        Cuda(cudaGetLastError(), "postings kernel launch");
        Cuda(cudaMemcpyAsync(term_offsets, d_toff, (vocab + 1) * sizeof(long long), cudaMemcpyDeviceToHost, s), "D2H");
        Cuda(cudaMemcpyAsync(posting_doc_ids, d_docs, runs * sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
        Cuda(cudaMemcpyAsync(posting_tf, d_tf, runs * sizeof(float), cudaMemcpyDeviceToHost, s), "D2H");
        Cuda(cudaStreamSynchronize(s), "postings");
        *postings = runs;
        // idf per term and norm per document in double, rounded to FP32 once
        const double n = (double)num_docs;
        for (int64_t t = 0; t < vocab; ++t) {
            const double df = (double)(term_offsets[t + 1] - term_offsets[t]);
            idf[t] = (float)std::log1p((n - df + 0.5) / (df + 0.5));
        }
        const double average = (double)total / n;
        for (int64_t d = 0; d < num_docs; ++d) {
            const double len = (double)(doc_offsets[d + 1] - doc_offsets[d]);
            doc_norm[d] = (float)(k1 * (1.0 - b + b * len / average));
        }
    } catch (const BuildFailure &f) {
        g_build_error = f.message;
        status = f.status;
    } catch (const std::exception &e) {
        g_build_error = e.what();
        status = BM25_ERR_INNER_ERROR;
    }
    for (void *p : owned)
        cudaFree(p);
    if (s)
        cudaStreamDestroy(s);
    return status;
}

extern "C" int bm25_build_last_error(char *buffer, size_t length)
{
    if (buffer && length) {
        const size_t n = g_build_error.size() < length - 1 ? g_build_error.size() : length - 1;
        g_build_error.copy(buffer, n);
        buffer[n] = '\0';
    }
    return BM25_OK;
}
