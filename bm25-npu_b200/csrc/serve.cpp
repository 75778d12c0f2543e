// Continuous-batching Search server over one session (the serving loop; no
// counterpart in the reference, which serves one fixed batch per call).
//
// Callers submit single queries (words, K) from any thread and wait on a
// ticket.  One worker thread forms batches continuously: whenever the previous
// batch has returned, it takes the waiting queries in arrival order while the
// batch stays within the session's capacities (queries, words) and the
// candidate-memory budget (the sum of the batch's K: a query's candidate
// buffer and its final select grow with K), and runs them as one Search with a
// K per query (bm25_search_batch, or bm25_search_batch_learned: learned
// pruning, every result still exact).  Latency is measured from each query's
// arrival to the return of its batch.
//
// bm25_serve_poisson drives a server with an open-loop Poisson arrival process
// (seeded) from a pool of queries and reports every query's latency: the
// measurement of the serving configuration.
#include "bm25_b200.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <random>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

thread_local std::string g_server_error;

int Fail(int status, const std::string &m)
{
    g_server_error = m;
    return status;
}

} // namespace

struct bm25_server {
    struct Item {
        uint64_t ticket;
        std::vector<int32_t> words;
        int32_t k;
        Clock::time_point arrival;
    };
    struct Done {
        std::vector<float> scores;
        std::vector<int32_t> ids;
        int32_t exact = 1;
        int status = BM25_OK;
        double latency_us = 0;
    };

    bm25_handle *handle = nullptr;
    bm25_server_options opts{};
    int32_t query_capacity = 0, word_capacity = 0, max_k = 0;
    std::mutex m;
    std::condition_variable work_cv, done_cv;
    std::deque<Item> queue;
    std::unordered_map<uint64_t, Done> done;
    std::unordered_set<uint64_t> outstanding;  // submitted and not yet waited for
    uint64_t next_ticket = 1;
    bool stop = false;
    std::thread worker;
    int64_t batches = 0, served = 0;
    int first_error = BM25_OK;

    void Loop()
    {
        std::vector<int64_t> offsets;
        std::vector<int32_t> words, ks, exact;
        std::vector<float> scores;
        std::vector<int32_t> ids;
        std::vector<Item> batch;
        std::unique_lock<std::mutex> lk(m);
        for (;;) {
            work_cv.wait(lk, [&] { return stop || !queue.empty(); });
            if (queue.empty() && stop)
                return;
            if (opts.max_wait_us > 0 && (int32_t)queue.size() < opts.max_batch) {
                // a partial batch may wait a little for more arrivals
                const auto until = queue.front().arrival + std::chrono::microseconds(opts.max_wait_us);
                work_cv.wait_until(lk, until, [&] { return stop || (int32_t)queue.size() >= opts.max_batch; });
            }
            // admission: arrival order, within the query, word and candidate budgets (one at least)
            batch.clear();
            int64_t nwords = 0, ksum = 0;
            while (!queue.empty() && (int32_t)batch.size() < opts.max_batch) {
                const Item &it = queue.front();
                const int64_t w = (int64_t)it.words.size();
                if (!batch.empty() && (nwords + w > word_capacity ||
                                       (opts.candidate_budget > 0 && ksum + it.k > opts.candidate_budget)))
                    break;
                nwords += w;
                ksum += it.k;
                batch.push_back(std::move(queue.front()));
                queue.pop_front();
            }
            lk.unlock();
            const int64_t q = (int64_t)batch.size();
            offsets.assign(q + 1, 0);
            words.clear();
            ks.resize(q);
            for (int64_t i = 0; i < q; ++i) {
                words.insert(words.end(), batch[i].words.begin(), batch[i].words.end());
                offsets[i + 1] = (int64_t)words.size();
                ks[i] = batch[i].k;
            }
            if (words.empty())
                words.push_back(0);
            scores.resize(ksum);
            ids.resize(ksum);
            exact.assign(q, 1);
            const int status =
                opts.learned ? bm25_search_batch_learned(handle, offsets.data(), words.data(), ks.data(), q,
                                                         scores.data(), ids.data(), exact.data())
                             : bm25_search_batch(handle, offsets.data(), words.data(), ks.data(), q, scores.data(),
                                                 ids.data());
            const auto finished = Clock::now();
            lk.lock();
            int64_t at = 0;
            for (int64_t i = 0; i < q; ++i) {
                Done d;
                d.status = status;
                if (status == BM25_OK) {
                    d.scores.assign(scores.begin() + at, scores.begin() + at + ks[i]);
                    d.ids.assign(ids.begin() + at, ids.begin() + at + ks[i]);
                    d.exact = exact[i];
                }
                at += ks[i];
                d.latency_us = std::chrono::duration<double, std::micro>(finished - batch[i].arrival).count();
                done[batch[i].ticket] = std::move(d);
            }
            if (status != BM25_OK && first_error == BM25_OK)
                first_error = status;
            ++batches;
            served += q;
            done_cv.notify_all();
        }
    }

    int Submit(const int32_t *w, int32_t n, int32_t k, Clock::time_point arrival, uint64_t *ticket)
    {
        if (n < 0 || n > 64 || (n > 0 && !w) || !ticket)
            return Fail(BM25_ERR_INVALID_PARAM, "Query exceeds 64 words or null buffer");
        if (n > word_capacity)
            return Fail(BM25_ERR_INVALID_PARAM, "Query exceeds the session's word capacity");
        if (k < 1 || k > max_k)
            return Fail(BM25_ERR_INVALID_PARAM, "K outside [1, max_k]");
        for (int32_t i = 0; i < n; ++i)
            if (w[i] < 0 || w[i] == INT32_MAX)
                return Fail(BM25_ERR_INVALID_PARAM, "Invalid public word ID");
        Item it{0, std::vector<int32_t>(w, w + n), k, arrival};
        {
            std::lock_guard<std::mutex> lk(m);
            if (stop)
                return Fail(BM25_ERR_ILLEGAL_OPERATION, "Server is stopping");
            it.ticket = next_ticket++;
            *ticket = it.ticket;
            outstanding.insert(it.ticket);
            queue.push_back(std::move(it));
        }
        work_cv.notify_one();
        return BM25_OK;
    }

    int Wait(uint64_t ticket, float *s, int32_t *i, int32_t *exact, double *latency)
    {
        std::unique_lock<std::mutex> lk(m);
        if (!outstanding.count(ticket))
            return Fail(BM25_ERR_INVALID_PARAM, "Unknown ticket, or one already waited for");
        done_cv.wait(lk, [&] { return done.count(ticket) != 0; });
        Done d = std::move(done[ticket]);
        done.erase(ticket);
        outstanding.erase(ticket);
        lk.unlock();
        if (d.status != BM25_OK)
            return Fail(d.status, "The batch holding this query failed; see bm25_last_error of the session");
        if (s)
            std::memcpy(s, d.scores.data(), d.scores.size() * sizeof(float));
        if (i)
            std::memcpy(i, d.ids.data(), d.ids.size() * sizeof(int32_t));
        if (exact)
            *exact = d.exact;
        if (latency)
            *latency = d.latency_us;
        return BM25_OK;
    }

    void Shutdown()
    {
        {
            std::lock_guard<std::mutex> lk(m);
            stop = true;
        }
        work_cv.notify_all();
        if (worker.joinable())
            worker.join();
    }
};

extern "C" {

void bm25_default_server_options(bm25_server_options *o)
{
    if (!o)
        return;
    std::memset(o, 0, sizeof(*o));
    o->max_batch = 256;
}

int bm25_server_create(bm25_handle *h, const bm25_server_options *options, bm25_server **out)
{
    if (!out)
        return Fail(BM25_ERR_INVALID_PARAM, "Null server output");
    *out = nullptr;
    if (!h)
        return Fail(BM25_ERR_ILLEGAL_OPERATION, "Null session");
    bm25_info info{};
    const int st = bm25_get_info(h, &info);
    if (st != BM25_OK)
        return Fail(st, "Session is not usable");
    bm25_server_options o;
    bm25_default_server_options(&o);
    if (options)
        o = *options;
    if (o.max_batch < 1 || o.max_batch > info.query_capacity)
        return Fail(BM25_ERR_INVALID_PARAM, "max_batch must be in [1, query_capacity]");
    if (info.kernel != BM25_KERNEL_TILE_GROUP && info.kernel != BM25_KERNEL_WARP_TILE)
        return Fail(BM25_ERR_INVALID_PARAM, "The server needs a warp-tile or tile-group session (a K per query)");
    if (o.learned && !info.prune)
        return Fail(BM25_ERR_INVALID_PARAM, "Learned serving needs a session created with prune = 1");
    if (o.candidate_budget < 0 || o.max_wait_us < 0)
        return Fail(BM25_ERR_INVALID_PARAM, "Negative budget or wait");
    // every batch the worker can form replays an instantiated graph: none is built on the request path
    const int prep = bm25_prepare_batch_graphs(h, o.max_batch, o.learned);
    if (prep != BM25_OK) {
        char message[512] = {0};
        bm25_last_error(h, message, sizeof(message), nullptr);
        return Fail(prep, std::string("Preparing the batch graphs failed: ") + message);
    }
    auto s = new bm25_server();
    s->handle = h;
    s->opts = o;
    s->query_capacity = info.query_capacity;
    s->word_capacity = info.word_capacity;
    s->max_k = std::min<int64_t>(info.max_k, info.num_docs);
    s->worker = std::thread([s] { s->Loop(); });
    *out = s;
    return BM25_OK;
}

int bm25_server_submit(bm25_server *s, const int32_t *words, int32_t n, int32_t k, uint64_t *ticket)
{
    if (!s)
        return Fail(BM25_ERR_ILLEGAL_OPERATION, "Null server");
    return s->Submit(words, n, k, Clock::now(), ticket);
}

int bm25_server_wait(bm25_server *s, uint64_t ticket, float *scores, int32_t *ids, int32_t *exact, double *latency_us)
{
    if (!s)
        return Fail(BM25_ERR_ILLEGAL_OPERATION, "Null server");
    return s->Wait(ticket, scores, ids, exact, latency_us);
}

int bm25_server_stats(bm25_server *s, int64_t *batches, int64_t *served)
{
    if (!s)
        return Fail(BM25_ERR_ILLEGAL_OPERATION, "Null server");
    std::lock_guard<std::mutex> lk(s->m);
    if (batches)
        *batches = s->batches;
    if (served)
        *served = s->served;
    return BM25_OK;
}

int bm25_server_destroy(bm25_server *s)
{
    if (!s)
        return BM25_OK;
    s->Shutdown();
    delete s;
    return BM25_OK;
}

int bm25_server_last_error(char *buffer, size_t length)
{
    if (buffer && length) {
        const size_t n = std::min(g_server_error.size(), length - 1);
        g_server_error.copy(buffer, n);
        buffer[n] = '\0';
    }
    return BM25_OK;
}

int bm25_serve_poisson(bm25_handle *h, const bm25_server_options *options, const int64_t *qoffsets,
                       const int32_t *words, const int32_t *ks, int64_t pool, double rate_qps, int64_t total,
                       uint64_t seed, double *latency_us, double *elapsed_s, int64_t *batches)
{
    if (!qoffsets || !words || !ks || pool < 1 || total < 1 || !(rate_qps > 0) || !latency_us)
        return Fail(BM25_ERR_INVALID_PARAM, "Invalid Poisson run");
    bm25_server *s = nullptr;
    int st = bm25_server_create(h, options, &s);
    if (st != BM25_OK)
        return st;
    // arrival schedule: exponential gaps at rate_qps (seeded), queries cycled through the pool
    std::mt19937_64 rng(seed);
    std::exponential_distribution<double> gap(rate_qps);
    std::vector<double> at(total);
    double t = 0;
    for (int64_t i = 0; i < total; ++i) {
        t += gap(rng);
        at[i] = t;
    }
    std::vector<uint64_t> tickets(total, 0);
    std::atomic<int64_t> submitted{0};
    int wait_status = BM25_OK;
    const auto start = Clock::now();
    // collector: waits for the tickets in order
    std::thread collector([&] {
        for (int64_t i = 0; i < total; ++i) {
            while (submitted.load(std::memory_order_acquire) <= i)
                std::this_thread::yield();
            double lat = 0;
            const int r = s->Wait(tickets[i], nullptr, nullptr, nullptr, &lat);
            if (r != BM25_OK && wait_status == BM25_OK)
                wait_status = r;
            latency_us[i] = lat;
        }
    });
    int submit_status = BM25_OK;
    for (int64_t i = 0; i < total; ++i) {
        const auto arrival = start + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(at[i]));
        while (Clock::now() < arrival) {
            const auto left = arrival - Clock::now();
            if (left > std::chrono::microseconds(200))
                std::this_thread::sleep_for(left - std::chrono::microseconds(100));
        }
        const int64_t p = i % pool;
        const int r = s->Submit(words + qoffsets[p], (int32_t)(qoffsets[p + 1] - qoffsets[p]), ks[p], arrival,
                                &tickets[i]);
        if (r != BM25_OK) {
            submit_status = r;
            tickets[i] = 0;
            // let the collector skip the remaining tickets
            for (int64_t j = i; j < total; ++j)
                latency_us[j] = -1;
            submitted.store(total, std::memory_order_release);
            break;
        }
        submitted.store(i + 1, std::memory_order_release);
    }
    if (submit_status != BM25_OK) {
        collector.join();  // the worker completes the submitted queries
        bm25_server_destroy(s);
        return submit_status;
    }
    collector.join();
    const double elapsed = std::chrono::duration<double>(Clock::now() - start).count();
    if (elapsed_s)
        *elapsed_s = elapsed;
    bm25_server_stats(s, batches, nullptr);
    bm25_server_destroy(s);
    return wait_status;
}

} // extern "C"
