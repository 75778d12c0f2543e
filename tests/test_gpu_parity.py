"""Parity of the CUDA engine (through the C ABI) with the CPU oracle: bit-exact top-K ids and FP32 score bits."""

import numpy as np
import pytest

from helpers import EDGE_A, EDGE_B, assert_same_topk, mixed_queries, pack

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def corpus(pkg, oracle_mod):
    spec = pkg.CorpusSpec(docs=60_000, vocab=30_000, seed=11, k1=1.5)
    index = pkg.synthetic_index(spec)
    data = oracle_mod.contributions(index, spec.k1)
    return spec, index, data


def _oracle(oracle_mod, index, data, offsets, words, k):
    return oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words, k)


KERNELS = pytest.mark.parametrize('kernel', [0, 1, 4, 5], ids=['stream', 'per_tile', 'tile_group', 'warp_tile'])


def _tile(kernel, tile_docs):
    """The tile-group kernel takes 1024- or 2048-document tiles, the warp-tile kernel 1024 (0 = automatic)."""
    return 0 if kernel in (4, 5) else tile_docs


@KERNELS
def test_config_8192_docs_q8x3_k10(pkg, oracle_mod, cuda_ok, kernel):
    """8192 docs, V 30,000 Zipf(1.1), lognormal mean 60, k1 1.5, b 0.75, 8 x 3 df-sampled terms, K 10."""
    spec = pkg.CONFIG_SHAPES['synthetic_8192']
    index = pkg.synthetic_index(spec)
    data = oracle_mod.contributions(index, spec.k1)
    for seed in (1, 2, 3):
        offsets, words = pkg.synthetic_queries(index.offsets, 8, 3, 3, seed)
        ref = _oracle(oracle_mod, index, data, offsets, words, 10)
        with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, kernel=kernel) as s:
            assert_same_topk(*s.search((offsets, words), 10), *ref, 'eager')
        with pkg.Bm25Session.from_lazy(index.offsets, index.docs, index.tf, index.norm, index.idf, k1=spec.k1,
                                       kernel=kernel) as s:
            assert_same_topk(*s.search((offsets, words), 10), *ref, 'lazy')


@KERNELS
@pytest.mark.parametrize('tile_docs,fan_in,stages', [(2048, 2, 2), (2048, 4, 3), (4096, 32, 8), (0, 0, 0),
                                                     (32768, 8, 4)])
def test_tiles_and_merge_tree(pkg, oracle_mod, corpus, cuda_ok, tile_docs, fan_in, stages, kernel):
    spec, index, data = corpus
    if (kernel == 4 and tile_docs not in (0, 1024, 2048)) or (kernel == 5 and tile_docs not in (0, 1024)):
        with pytest.raises(pkg.InvalidParam):
            pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, tile_docs=tile_docs,
                                     kernel=kernel)
        tile_docs = 0
    rng = np.random.default_rng(tile_docs + fan_in)
    rows = mixed_queries(index.vocab, rng, 24, 0, 12)
    rows[0] = [0, 1, 2]          # densest terms: candidate list overflow, full-row selection
    rows[1] = [0, 0, 0, 0]       # the same dense term repeatedly
    rows[2] = []                 # zero fill only
    offsets, words = pack(rows)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=32,
                                  word_capacity=512, max_k=32, tile_docs=tile_docs, merge_fan_in=fan_in,
                                  kernel=kernel, ring_stages=stages) as s:
        info = s.info()
        assert info['tiles'] == -(-index.num_docs // info['tile_docs'])
        for k in (1, 7, 10, 32):
            got = s.search((offsets, words), k)
            assert_same_topk(*got, *_oracle(oracle_mod, index, data, offsets, words, k), f'k={k}')


@KERNELS
def test_directory_and_scan_paths_agree(pkg, oracle_mod, corpus, cuda_ok, kernel):
    spec, index, data = corpus
    rng = np.random.default_rng(5)
    offsets, words = pack(mixed_queries(index.vocab, rng, 16, 1, 10))
    ref = _oracle(oracle_mod, index, data, offsets, words, 10)
    for budget in (1, 1 << 30):  # 1 byte: every list is counted inside the CTA; 1 GiB: directory for long lists
        with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=16,
                                      word_capacity=256, tile_docs=_tile(kernel, 2048), directory_bytes=budget,
                                      kernel=kernel) as s:
            assert_same_topk(*s.search((offsets, words), 10), *ref, f'budget={budget}')


@KERNELS
def test_reference_edge_queries(pkg, oracle_mod, corpus, cuda_ok, kernel):
    spec, index, data = corpus
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=7,
                                  word_capacity=128, max_k=32, tile_docs=_tile(kernel, 4096), kernel=kernel) as s:
        for rows in (EDGE_A, EDGE_B, EDGE_A, [[]] * 3, EDGE_B):
            offsets, words = pack(rows)
            for k in (1, 3, 10, 32):
                assert_same_topk(*s.search((offsets, words), k), *_oracle(oracle_mod, index, data, offsets, words, k))


@KERNELS
def test_empty_bootstrap_is_zero_fill(pkg, corpus, cuda_ok, kernel):
    """Search(empty) returns score 0 and ids 0..K-1 (large_search.cpp:184-187)."""
    spec, index, data = corpus
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, max_k=10, kernel=kernel) as s:
        scores, ids = s.search([[]] * 8, 10)
        assert (scores == 0).all() and (ids == np.arange(10)[None, :]).all()


def test_input_errors_keep_session_usable(pkg, oracle_mod, corpus, cuda_ok):
    spec, index, data = corpus
    s = pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=4,
                                 word_capacity=8, max_k=10)
    good = [[0, 5], [7], [], [3]]
    offsets, words = pack(good)
    ref = _oracle(oracle_mod, index, data, offsets, words, 10)
    bad_inputs = [
        [[-1]], [[2**31 - 1]], [[1]] * 5, [list(range(9))], [[0] * 65],
    ]
    for bad in bad_inputs:
        with pytest.raises(pkg.InvalidParam):
            s.search(bad, 10)
        assert_same_topk(*s.search(good, 10), *ref)
    for k in (0, 11):
        with pytest.raises(pkg.InvalidParam):
            s.search(good, k)
    s.close()
    with pytest.raises((pkg.IllegalOperation, AttributeError, TypeError)):
        s.search(good, 10)


def test_invalid_index_rejected(pkg, cuda_ok):
    indptr = np.array([0, 2, 3], dtype=np.int64)
    with pytest.raises(pkg.InvalidParam):
        pkg.Bm25Session.from_csc(indptr, np.array([1, 0, 2], dtype=np.int32), np.ones(3, np.float32), 4)
    with pytest.raises(pkg.InvalidParam):
        pkg.Bm25Session.from_csc(indptr, np.array([0, 1, 4], dtype=np.int32), np.ones(3, np.float32), 4)
    with pytest.raises(pkg.InvalidParam):
        pkg.Bm25Session.from_csc(indptr, np.array([0, 1, 2], dtype=np.int32),
                                 np.array([1, np.nan, 1], np.float32), 4)


@KERNELS
def test_device_resident_search_matches_host(pkg, oracle_mod, corpus, cuda_ok, kernel):
    import torch
    spec, index, data = corpus
    rng = np.random.default_rng(9)
    offsets, words = pack(mixed_queries(index.vocab, rng, 8, 1, 6, oov=False))
    ref = _oracle(oracle_mod, index, data, offsets, words, 10)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, word_capacity=64,
                                  kernel=kernel) as s:
        d_off = torch.from_numpy(offsets).cuda()
        d_words = torch.from_numpy(words).cuda()
        d_scores = torch.empty((8, 10), dtype=torch.float32, device='cuda')
        d_ids = torch.empty((8, 10), dtype=torch.int32, device='cuda')
        stream = torch.cuda.current_stream()
        s.search_device(d_off.data_ptr(), d_words.data_ptr(), 8, 10, d_scores.data_ptr(), d_ids.data_ptr(),
                        stream.cuda_stream)
        assert s.device_status() == 0
        stream.synchronize()
        assert_same_topk(d_scores.cpu().numpy(), d_ids.cpu().numpy(), *ref, 'device')
        assert_same_topk(*s.search((offsets, words), 10), *ref, 'host after device')


@KERNELS
def test_alternating_batches_replay(pkg, oracle_mod, corpus, cuda_ok, kernel):
    """A/B alternation through cached graphs, as the reference's benchmark does (benchmark_common.h:51-107)."""
    spec, index, data = corpus
    a = pkg.synthetic_queries(index.offsets, 8, 3, 3, 101)
    b = pkg.synthetic_queries(index.offsets, 8, 3, 3, 102)
    ra = _oracle(oracle_mod, index, data, *a, 10)
    rb = _oracle(oracle_mod, index, data, *b, 10)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, kernel=kernel) as s:
        for _ in range(5):
            assert_same_topk(*s.search(a, 10), *ra, 'A')
            assert_same_topk(*s.search(b, 10), *rb, 'B')
        assert s.info()['graph_replays'] == 10


def test_sessions_with_different_tiles_coexist(pkg, oracle_mod, corpus, cuda_ok):
    """The kernels' shared-memory cap is process-wide: a later session with small tiles must not break a
    live session with large tiles."""
    spec, index, data = corpus
    offsets, words = pkg.synthetic_queries(index.offsets, 8, 3, 3, 55)
    ref = _oracle(oracle_mod, index, data, offsets, words, 10)
    big = pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, tile_docs=32768, kernel=0)
    small = pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, tile_docs=2048, kernel=0)
    try:
        for s in (big, small, big):
            assert_same_topk(*s.search((offsets, words), 10), *ref)
    finally:
        small.close()
        big.close()


@KERNELS
def test_kernel_timing_hook(pkg, corpus, cuda_ok, kernel):
    import torch
    spec, index, data = corpus
    offsets, words = pkg.synthetic_queries(index.offsets, 8, 3, 3, 77)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, kernel=kernel) as s:
        with pytest.raises(pkg.InvalidParam):
            s.kernel_times()
        d_off = torch.from_numpy(offsets).cuda()
        d_words = torch.from_numpy(words).cuda()
        d_scores = torch.empty((8, 10), dtype=torch.float32, device='cuda')
        d_ids = torch.empty((8, 10), dtype=torch.int32, device='cuda')
        stream = torch.cuda.current_stream()
        s.kernel_timing(True)
        for _ in range(5):
            s.search_device(d_off.data_ptr(), d_words.data_ptr(), 8, 10, d_scores.data_ptr(), d_ids.data_ptr(),
                            stream.cuda_stream)
        s.search((offsets, words), 10)  # graph replay: not timed
        ms = s.kernel_times()
        assert ms.size == 5 and (ms > 0).all() and (ms < 1000).all()
        assert s.kernel_times().size == 0
        s.kernel_timing(False)
        assert s.device_status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize('density', [-1.0, 0.0, 0.02, 1.0])
def test_warp_tile_dense_rows(pkg, oracle_mod, corpus, cuda_ok, density):
    """The warp-tile kernel adds the terms kept as dense rows (df >= density * N) from those rows and
    the others from their postings, in query-word order: same bits as the oracle with no dense rows
    (-1), the default (0: a quarter of the documents), nearly every term dense (0.02), and only terms in every
    document (1.0).  Queries mix dense and sparse words in every order, repeats and unknown words."""
    spec, index, data = corpus
    df = np.diff(index.offsets)
    order = np.argsort(-df)
    dense_words = [int(x) for x in order[:6]]
    rng = np.random.default_rng(11)
    rows = mixed_queries(index.vocab, rng, 20, 0, 10)
    rows += [dense_words[:3], [dense_words[0], 5, dense_words[1], 7], [9, dense_words[2], dense_words[2], 9],
             dense_words + [index.vocab + 3], [int(order[-1]), dense_words[4]]]
    offsets, words = pack(rows)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=32,
                                  word_capacity=512, max_k=32, kernel=5, dense_density=density) as s:
        info = s.info()
        if density < 0:
            assert info['dense_rows'] == 0
        else:
            d = 0.25 if density == 0 else density
            fit = min(16 << 30, info['index_bytes']) // (info['tiles'] * 1024 * 4)  # the rows' byte budget
            assert info['dense_rows'] == min(fit, int(np.sum(df >= np.ceil(d * index.num_docs))))
        for k in (1, 10, 32):
            assert_same_topk(*s.search((offsets, words), k), *_oracle(oracle_mod, index, data, offsets, words, k),
                             f'density={density} k={k}')
