"""K above 32 (up to 1024): tile appends at the running bound, radix final select, overflow retry.

Bit-exact against the oracle's unbounded strict top-K (score desc, id asc,
zero-score fill by id), on queries with duplicates, out-of-vocabulary words,
empty rows and fewer than K matching documents; through the plain path, the
pruned path and a session whose small candidate buffer overflows so that the
retry pass must answer from its final bound.
"""

import numpy as np
import pytest

from helpers import assert_same_topk, mixed_queries, pack


def test_large_k_options_checked(pkg):
    """max_k above 32 needs the tile-group kernel; 1024 is the largest K (no device needed)."""
    spec = pkg.CorpusSpec(docs=4096, vocab=500, seed=3)
    index = pkg.synthetic_index(spec)
    with pytest.raises(pkg.InvalidParam):
        pkg.Bm25Session.from_lazy(index.offsets, index.docs, index.tf, index.norm, index.idf, max_k=64, kernel=0)
    with pytest.raises(pkg.InvalidParam):
        pkg.Bm25Session.from_lazy(index.offsets, index.docs, index.tf, index.norm, index.idf, max_k=1025)


@pytest.fixture(scope='module')
def corpus(pkg, oracle_mod):
    spec = pkg.CorpusSpec(docs=200_000, vocab=20_000, seed=77, k1=1.2)
    index = pkg.synthetic_index(spec)
    data = oracle_mod.contributions(index, spec.k1)
    return index, data


def _queries(index, seed, count):
    rng = np.random.default_rng(seed)
    rows = mixed_queries(index.vocab, rng, count, 1, 12, oov=True)
    rows += [[], [index.vocab - 1], [0, 0, 0]]  # empty, a rare word (fewer than K matches), duplicates
    return pack(rows)


@pytest.mark.gpu
@pytest.mark.parametrize('kernel,tile_docs', [(5, 1024), (4, 1024), (4, 2048)])
def test_large_k_plain_matches_oracle(pkg, oracle_mod, corpus, cuda_ok, kernel, tile_docs):
    index, data = corpus
    offsets, words = _queries(index, tile_docs, 29)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=64,
                                  word_capacity=1024, max_k=1024, tile_docs=tile_docs, kernel=kernel) as s:
        for k in (33, 100, 1000, 1024, 10):
            want = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words, k)
            assert_same_topk(*s.search((offsets, words), k), *want, f'k={k}')
            assert s.device_status() == 0


@pytest.mark.gpu
def test_large_k_overflow_is_retried(pkg, oracle_mod, corpus, cuda_ok):
    """A candidate buffer of 2048 per query overflows on the first pass for common words; the
    retry pass searches those queries again from their final bound and still answers exactly."""
    index, data = corpus
    df = np.diff(index.offsets)
    common = [int(x) for x in np.argsort(-df)[:6]]
    rows = [common[:2], common[2:5], [common[0]], common[1:6]]
    offsets, words = pack(rows)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=8,
                                  word_capacity=64, max_k=256, candidate_capacity=2048) as s:
        for k in (100, 256):
            want = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words, k)
            assert_same_topk(*s.search((offsets, words), k), *want, f'k={k}')
            s.search_stats(reset=True)


@pytest.mark.gpu
def test_large_k_pruned_matches_oracle(pkg, oracle_mod, corpus, cuda_ok):
    index, data = corpus
    offsets, words = _queries(index, 5, 29)
    q = offsets.size - 1
    # a buffer that holds every document: no query overflows, so the flags follow tau alone
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=64,
                                  word_capacity=1024, max_k=1000, prune=True,
                                  candidate_capacity=index.num_docs + 2048) as s:
        for k in (100, 1000):
            want_s, want_i, full = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets,
                                                     words, k, full=True)
            kth = want_s[:, -1]
            for label, tau in (('kth', kth), ('0.8 kth', kth * np.float32(0.8)), ('2 kth', kth * np.float32(2)),
                               ('zero', np.zeros(q, np.float32))):
                got_s, got_i, exact = s.search_pruned((offsets, words), k, tau.astype(np.float32))
                assert_same_topk(got_s, got_i, want_s, want_i, f'k={k} {label}')
                reach = ((full >= tau[:, None]) & (full > 0)).sum(axis=1)
                assert np.array_equal(exact, np.where(~(tau > 0) | (reach >= k), 1, 0)), label
            s.set_threshold_model(None)  # safe bounds alone (term ranks 64..1024): proven, so nothing fails
            got_s, got_i, exact = s.search_learned((offsets, words), k)
            assert_same_topk(got_s, got_i, want_s, want_i, f'k={k} learned (no model)')
            assert exact.all()


def _by_k(oracle_mod, index, data, offsets, words, ks):
    """Oracle rows for a batch with a K per query, packed like bm25_search_batch."""
    out_s, out_i = [], []
    for i, k in enumerate(ks):
        o = np.array([0, offsets[i + 1] - offsets[i]], dtype=np.int64)
        w = words[offsets[i]:offsets[i + 1]]
        s, d = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, o, w, int(k))
        out_s.append(s[0])
        out_i.append(d[0])
    return np.concatenate(out_s), np.concatenate(out_i)


@pytest.mark.gpu
def test_batch_with_k_per_query(pkg, oracle_mod, corpus, cuda_ok):
    """One Search of 40 queries with K drawn from {1, 10, 32, 33, 100, 1000}: packed rows equal the
    oracle's per-query top-K, through the plain path, the learned path (safe bounds and a model of
    random weights whose bounds fall back often) and the device entry point."""
    import torch
    index, data = corpus
    offsets, words = _queries(index, 11, 37)
    q = offsets.size - 1
    rng = np.random.default_rng(4)
    ks = rng.choice([1, 10, 32, 33, 100, 1000], q).astype(np.int32)
    want_s, want_i = _by_k(oracle_mod, index, data, offsets, words, ks)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=64,
                                  word_capacity=1024, max_k=1000, prune=True) as s:
        got_s, got_i, koff = s.search_batch((offsets, words), ks)
        assert koff[-1] == ks.sum()
        assert_same_topk(got_s[None], got_i[None], want_s[None], want_i[None], 'batch plain')
        for model in (None, pkg.learned.ThresholdModel(pkg.learned.init_params(1, 3.0), -1.0)):
            s.set_threshold_model(model)
            got_s, got_i, koff, exact = s.search_batch((offsets, words), ks, learned=True)
            assert_same_topk(got_s[None], got_i[None], want_s[None], want_i[None], f'batch learned {model is None}')
        dev = torch.device('cuda:0')
        d = {name: torch.from_numpy(x).to(dev) for name, x in
             (('o', offsets), ('w', words), ('k', ks), ('ko', koff[:-1].copy()))}
        d_s = torch.empty(int(koff[-1]), dtype=torch.float32, device=dev)
        d_i = torch.empty(int(koff[-1]), dtype=torch.int32, device=dev)
        d_x = torch.empty(q, dtype=torch.int32, device=dev)
        for learned in (False, True):
            s.search_batch_device(d['o'].data_ptr(), d['w'].data_ptr(), d['k'].data_ptr(), d['ko'].data_ptr(), q,
                                  int(ks.max()), d_s.data_ptr(), d_i.data_ptr(), d_x.data_ptr(), learned,
                                  torch.cuda.current_stream(dev).cuda_stream)
            torch.cuda.synchronize()
            assert s.device_status() == 0
            assert_same_topk(d_s.cpu().numpy()[None], d_i.cpu().numpy()[None], want_s[None], want_i[None],
                             f'batch device learned={learned}')


@pytest.mark.gpu
def test_tune_batch_with_k_per_query_learned(pkg, oracle_mod, corpus, cuda_ok):
    """The live-session tuner on a learned batch with a K per query (as the benchmark tunes the routing
    cut): every cut answers the same bits, the fastest is kept, and the session still answers the
    oracle's rows afterwards."""
    index, data = corpus
    offsets, words = _queries(index, 11, 41)
    q = offsets.size - 1
    ks = np.random.default_rng(9).choice([10, 100, 1000], q).astype(np.int32)
    want_s, want_i = _by_k(oracle_mod, index, data, offsets, words, ks)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=64,
                                  word_capacity=1024, max_k=1000, prune=True) as s:
        s.set_threshold_model(pkg.learned.ThresholdModel(pkg.learned.init_params(1, 3.0), -1.0))
        best, table = pkg.autotune.tune(s, (offsets, words), int(ks.max()), space={'prune_route': (0.2, 1.0)},
                                        learned=True, ks=ks, reps=2)
        assert len(table) == 2 and best['prune_route'] in (0.2, 1.0) and s.tuning()['prune_route'] == best['prune_route']
        got_s, got_i, _, _ = s.search_batch((offsets, words), ks, learned=True)
        assert_same_topk(got_s[None], got_i[None], want_s[None], want_i[None], 'tuned learned batch')
