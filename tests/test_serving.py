"""Continuous-batching server: results equal the oracle's whatever the batch a query lands in.

CPU: argument checks that need no device.  GPU: queries with K from {5, 10, 100}
submitted from two threads are served in batches (plain and learned) with
results bit-exact against the oracle; an open-loop Poisson run completes every
query with a positive latency.
"""

import threading

import numpy as np
import pytest

from helpers import mixed_queries


def test_server_rejects_without_session(pkg):
    import ctypes
    lib = pkg._native.engine_library()
    out = ctypes.c_void_p()
    assert lib.bm25_server_create(None, None, ctypes.byref(out)) == pkg._native.BM25_ERR_ILLEGAL_OPERATION
    assert not out.value
    assert lib.bm25_server_destroy(None) == pkg._native.BM25_OK


@pytest.fixture(scope='module')
def corpus(pkg, oracle_mod):
    spec = pkg.CorpusSpec(docs=100_000, vocab=10_000, seed=19, k1=1.2)
    index = pkg.synthetic_index(spec)
    return index, oracle_mod.contributions(index, spec.k1)


@pytest.mark.gpu
@pytest.mark.parametrize('learned', [False, True])
def test_server_matches_oracle(pkg, oracle_mod, corpus, cuda_ok, learned):
    index, data = corpus
    rows = mixed_queries(index.vocab, np.random.default_rng(8), 60, 1, 10, oov=True)
    ks = np.random.default_rng(9).choice([5, 10, 100], len(rows))
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=16,
                                  word_capacity=256, max_k=100, prune=True) as s:
        with pkg.serving.Server(s, max_batch=16, learned=learned, candidate_budget=300) as srv:
            prepared = s.info()['graph_instantiations']
            assert prepared >= 5  # batch buckets 1, 2, 4, 8, 16 at least (x K buckets)
            tickets = [None] * len(rows)

            def submit(part):
                for i in range(part, len(rows), 2):
                    tickets[i] = srv.submit(rows[i], int(ks[i]))

            th = [threading.Thread(target=submit, args=(p,)) for p in range(2)]
            for t in th:
                t.start()
            for t in th:
                t.join()
            for i, row in enumerate(rows):
                got_s, got_i, exact, lat = srv.wait(tickets[i])
                o = np.array([0, len(row)], np.int64)
                want = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, o,
                                         np.array(row, np.int32), int(ks[i]))
                assert np.array_equal(got_i, want[1][0]) and np.array_equal(got_s.view(np.uint32),
                                                                             want[0][0].view(np.uint32)), i
                assert lat > 0
            st = srv.stats()
            assert st['served'] == len(rows) and 1 <= st['batches'] <= len(rows)
            # every batch replayed a graph instantiated when the server was created
            assert s.info()['graph_instantiations'] == prepared
            with pytest.raises(pkg.InvalidParam):
                srv.wait(tickets[0])  # already waited for


@pytest.mark.gpu
def test_poisson_run_completes(pkg, corpus, cuda_ok):
    index, data = corpus
    qo, w = pkg.synthetic_queries(index.offsets, 64, 1, 8, 3)
    ks = np.random.default_rng(1).choice([10, 100], 64).astype(np.int32)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=64,
                                  word_capacity=64 * 8, max_k=100) as s:
        lat, st = pkg.serving.serve_poisson(s, qo, w, ks, rate_qps=5000, total=2000, max_batch=64)
        assert lat.shape == (2000,) and np.all(lat > 0)
        assert st['batches'] >= 1 and st['achieved_qps'] > 1000


@pytest.mark.gpu
def test_batch_buckets_pad_exactly(pkg, oracle_mod, corpus, cuda_ok):
    """Batches of 1..13 queries with K up to 100 run in their bucket's graph (queries padded to a power
    of two, K to 32 or 128): results equal the oracle, and one graph serves every batch of a bucket."""
    index, data = corpus
    rng = np.random.default_rng(21)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=16,
                                  word_capacity=256, max_k=100) as s:
        for q in (1, 2, 3, 5, 8, 13):
            rows = mixed_queries(index.vocab, rng, q, 0, 6, oov=True)
            ks = rng.choice([1, 7, 32, 33, 100], q).astype(np.int32)
            qo = np.zeros(q + 1, np.int64)
            qo[1:] = np.cumsum([len(r) for r in rows])
            words = np.array([w for r in rows for w in r], np.int32)
            gs, gi, koff = s.search_batch((qo, words), ks)
            for i in range(q):
                want = oracle_mod.search(index.offsets, index.docs, data, index.num_docs,
                                         np.array([0, len(rows[i])], np.int64), np.array(rows[i], np.int32),
                                         int(ks[i]))
                assert np.array_equal(gi[koff[i]:koff[i + 1]], want[1][0]), (q, i)
                assert np.array_equal(gs[koff[i]:koff[i + 1]].view(np.uint32), want[0][0].view(np.uint32)), (q, i)
        made = s.info()['graph_instantiations']
        for q in (5, 6, 7):  # bucket 8, K bucket 128: the graph made above
            qo, w = pkg.synthetic_queries(index.offsets, q, 1, 4, q)
            s.search_batch((qo, w), np.full(q, 100, np.int32))
        assert s.info()['graph_instantiations'] == made
