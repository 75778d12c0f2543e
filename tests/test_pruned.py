"""Pruned Search (128-document block bounds + a starting bound per query) against the oracle.

Every row must equal the oracle's top-K bit for bit, and the exactness flag is
predictable from the oracle's full score rows: 1 exactly when at least K
documents score at or above the starting bound (or the bound is not positive);
the queries flagged 0 were answered by the call's retry pass on the plain path.
"""

import numpy as np
import pytest

from helpers import assert_same_topk, mixed_queries, pack


def block_bounds(indptr, indices, data, words, block_docs, blocks):
    """Per query word and block: the largest posting score of the word in the block (0 if none)."""
    out = np.zeros((len(words), blocks), dtype=np.float32)
    vocab = indptr.size - 1
    for w, term in enumerate(words):
        if 0 <= term < vocab:
            s, e = indptr[term], indptr[term + 1]
            np.maximum.at(out[w], indices[s:e] // block_docs, np.maximum(data[s:e], 0))
    return out


def round_up_fp16(x):
    """x rounded up to FP16 (as the engine stores its block maxima), back in FP32."""
    h = np.asarray(x, np.float32).astype(np.float16)
    low = h.astype(np.float32) < x
    h[low] = np.nextafter(h[low], np.float16(np.inf))
    return h.astype(np.float32)


def test_round_up_fp16_never_lowers():
    x = np.random.default_rng(3).random(10_000, dtype=np.float32) * np.float32(40.0)
    r = round_up_fp16(x)
    assert np.all(r >= x) and np.all(r <= x * np.float32(1.001))


@pytest.mark.parametrize('block_docs', [128, 1024])
@pytest.mark.parametrize('stored', ['fp32', 'fp16_up'])
def test_block_bound_covers_every_document(pkg, oracle_mod, block_docs, stored):
    """FP32 sums of per-block maxima in query-word order bound every document's FP32 sum in the block,
    with the maxima in FP32 or rounded up to FP16 (the engine's block index)."""
    spec = pkg.CorpusSpec(docs=20_000, vocab=3_000, seed=5, k1=1.2)
    index = pkg.synthetic_index(spec)
    data = oracle_mod.contributions(index, spec.k1)
    rows = mixed_queries(index.vocab, np.random.default_rng(1), 24, 1, 12, oov=True)
    offsets, words = pack(rows)
    _, _, full = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words, 10, full=True)
    blocks = (index.num_docs + block_docs - 1) // block_docs
    for q in range(len(rows)):
        wb = block_bounds(index.offsets, index.docs, data, words[offsets[q]:offsets[q + 1]], block_docs, blocks)
        if stored == 'fp16_up':
            wb = round_up_fp16(wb)
        bound = np.zeros(blocks, dtype=np.float32)
        for b in wb:  # query-word order, FP32 rounding at every step
            bound = (bound + b).astype(np.float32)
        per_doc = np.repeat(bound, block_docs)[:index.num_docs]
        assert np.all(full[q] <= per_doc)


def expected_exact(full, tau, k):
    """1 where K documents reach the positive bound tau (or tau is not positive)."""
    reach = (full >= tau[:, None]) & (full > 0)
    return np.where(~(tau > 0) | (reach.sum(axis=1) >= k), 1, 0)


def _kth(scores):
    return scores[:, -1].copy()


@pytest.fixture(scope='module')
def corpus(pkg, oracle_mod):
    spec = pkg.CorpusSpec(docs=150_000, vocab=20_000, seed=31, k1=1.2)
    index = pkg.synthetic_index(spec)
    data = oracle_mod.contributions(index, spec.k1)
    return index, data


@pytest.mark.gpu
@pytest.mark.parametrize('kernel,tile_docs', [(5, 1024), (4, 1024), (4, 2048)])
def test_pruned_matches_oracle(pkg, oracle_mod, corpus, cuda_ok, kernel, tile_docs):
    index, data = corpus
    rng = np.random.default_rng(tile_docs)
    # besides random rows: a duplicated word, an empty query, and 40 words (the block scorer
    # fetches word metadata 32 words at a time)
    rows = mixed_queries(index.vocab, rng, 40, 0, 14, oov=True) + [[0, 1, 2], [5] * 12, [],
                                                                   [int(x) for x in rng.integers(0, 2000, 40)]]
    offsets, words = pack(rows)
    q = len(rows)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=64,
                                  word_capacity=1024, max_k=32, tile_docs=tile_docs, prune=True,
                                  kernel=kernel) as s:
        for k in (10, 32):
            want_s, want_i, full = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words,
                                                     k, full=True)
            kth = _kth(want_s)
            guesses = {
                'exact kth': kth,
                'half kth': kth * np.float32(0.5),
                'zero': np.zeros(q, np.float32),
                'above kth': np.nextafter(kth, np.float32(np.inf)),
                'mixed': np.where(rng.random(q) < 0.5, kth * np.float32(0.9), kth * np.float32(1.5)).astype(np.float32),
            }
            for label, tau in guesses.items():
                tau = tau.astype(np.float32)
                got_s, got_i, exact = s.search_pruned((offsets, words), k, tau)
                assert np.array_equal(exact, expected_exact(full, tau, k)), label
                assert_same_topk(got_s, got_i, want_s, want_i, f'k={k} {label}')
            # the plain path still answers the same afterwards (thresholds were reset)
            assert_same_topk(*s.search((offsets, words), k), want_s, want_i, f'k={k} plain after pruned')


@pytest.mark.gpu
def test_pruned_device_flags_and_rows(pkg, oracle_mod, corpus, cuda_ok):
    import torch
    index, data = corpus
    rows = mixed_queries(index.vocab, np.random.default_rng(9), 32, 2, 10, oov=False)
    offsets, words = pack(rows)
    q, k = len(rows), 10
    want_s, want_i, full = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words, k,
                                             full=True)
    tau = np.where(np.arange(q) % 3 == 0, _kth(want_s) * np.float32(2), _kth(want_s)).astype(np.float32)
    dev = torch.device('cuda:0')
    d_off = torch.from_numpy(offsets).to(dev)
    d_words = torch.from_numpy(words).to(dev)
    d_tau = torch.from_numpy(tau).to(dev)
    d_s = torch.empty((q, k), dtype=torch.float32, device=dev)
    d_i = torch.empty((q, k), dtype=torch.int32, device=dev)
    d_x = torch.full((q,), -1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=q,
                                  word_capacity=int(offsets[-1]), max_k=k, prune=True) as s:
        for _ in range(2):
            s.search_pruned_device(d_off.data_ptr(), d_words.data_ptr(), d_tau.data_ptr(), q, k, d_s.data_ptr(),
                                   d_i.data_ptr(), d_x.data_ptr(), stream.cuda_stream)
            torch.cuda.synchronize()
            assert s.device_status() == 0
            exact = d_x.cpu().numpy()
            assert np.array_equal(exact, expected_exact(full, tau, k))
            assert 0 < (exact == 0).sum() < q  # both the pruned pass and the retry pass answered
            assert_same_topk(d_s.cpu().numpy(), d_i.cpu().numpy(), want_s, want_i, 'device')


@pytest.mark.gpu
def test_pruned_needs_prune_session(pkg, corpus, cuda_ok):
    index, data = corpus
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs) as s:
        with pytest.raises(pkg.IllegalOperation):
            s.search_pruned([[1, 2]], 10, np.zeros(1, np.float32))
    with pytest.raises(pkg.InvalidParam):
        pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, kernel=0, prune=True)


@pytest.mark.gpu
def test_routing_streams_broad_queries_exactly(pkg, oracle_mod, corpus, cuda_ok):
    """In a pruned batch of 32+ queries, the queries whose bounds keep more than prune_route of their
    blocks are streamed by the tile-group kernel from their starting bound: still exact."""
    index, data = corpus
    rng = np.random.default_rng(77)
    df = np.diff(index.offsets)
    common = np.argsort(-df)[:40]
    rows = [[int(x) for x in rng.choice(common, 6, replace=False)] for _ in range(12)]  # broad
    rows += mixed_queries(index.vocab, rng, 28, 1, 4, oov=False)
    offsets, words = pack(rows)
    q = len(rows)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=64,
                                  word_capacity=1024, max_k=32, prune=True, prune_route=0.2) as s:
        for k in (10, 32):
            want_s, want_i, full = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets,
                                                     words, k, full=True)
            tau = (want_s[:, -1] * np.float32(0.9)).astype(np.float32)
            s.search_stats(reset=True)
            got_s, got_i, exact = s.search_pruned((offsets, words), k, tau)
            st = s.search_stats(reset=True)
            assert_same_topk(got_s, got_i, want_s, want_i, f'k={k}')
            assert np.array_equal(exact, expected_exact(full, tau, k))
            assert 0 < st['queries_streamed'] < q, st
