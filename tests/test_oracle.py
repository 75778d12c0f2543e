"""The CPU oracle against the reference's own CPU search (oracle/_ref) -- no GPU needed."""

import subprocess

import numpy as np
import pytest

from helpers import EDGE_A, EDGE_B, assert_same_topk, bits, mixed_queries, pack


def _need_reference(oracle_mod):
    if not oracle_mod.reference_available():
        pytest.skip('oracle/_ref not built (the reference sources are not on this machine)')


def test_reference_unit_test_binary_passes(oracle_mod):
    """The reference's own ut/cases/bm25/cpu_index_search_tests.cpp, compiled unmodified."""
    if not oracle_mod.REF_TEST.exists():
        pytest.skip('reference unit test binary not built')
    out = subprocess.run([str(oracle_mod.REF_TEST)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert 'CPU indexed Search passed 180' in out.stdout


@pytest.mark.parametrize('docs,vocab,seed', [(300, 50, 1), (5000, 2000, 2), (20000, 30000, 3)])
def test_oracle_matches_reference_session(pkg, oracle_mod, docs, vocab, seed):
    """Restated loop (eager and lazy) == reference CpuSearchSession at k1 = 1.2, K <= 32, bit for bit."""
    _need_reference(oracle_mod)
    spec = pkg.CorpusSpec(docs=docs, vocab=vocab, seed=seed, k1=1.2, len_mean=30.0)
    index = pkg.synthetic_index(spec)
    data = oracle_mod.contributions(index, 1.2)
    rng = np.random.default_rng(seed)
    for k in sorted({1, 3, 10, min(32, docs)}):
        for threads in (1, 4):
            ref = oracle_mod.ReferenceCpuSession(index, k, threads, query_capacity=16, word_capacity=256)
            for rows in (EDGE_A, EDGE_B, mixed_queries(vocab, rng, 16, 0, 12), [[]] * 4):
                offsets, words = pack(rows)
                rs, ri, _ = ref.search(offsets, words)
                es, ei, full = oracle_mod.search(index.offsets, index.docs, data, docs, offsets, words, k, full=True)
                assert_same_topk(es, ei, rs, ri, 'eager')
                ls, li = oracle_mod.search(index.offsets, index.docs, None, docs, offsets, words, k,
                                           lazy=(index.tf, index.norm, index.idf), k1=1.2)
                assert_same_topk(ls, li, rs, ri, 'lazy')
                ref_full = ref.debug_scores(len(rows))
                assert np.array_equal(bits(full), bits(ref_full)), 'full score rows differ'
            ref.close()


def test_directory_session_agrees(pkg, oracle_mod):
    _need_reference(oracle_mod)
    spec = pkg.CorpusSpec(docs=9000, vocab=4000, seed=4, k1=1.2)
    index = pkg.synthetic_index(spec)
    data = oracle_mod.contributions(index, 1.2)
    offsets, words = pkg.synthetic_queries(index.offsets, 8, 3, 3, 5)
    ref = oracle_mod.ReferenceCpuSession(index, 10, 4, mode=1)
    rs, ri, _ = ref.search(offsets, words)
    assert_same_topk(*oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words, 10), rs, ri)


def test_oracle_zero_fill_and_ties():
    """Hand-made ties: equal scores rank by id, zero scores fill by ascending id."""
    from oracle import oracle
    indptr = np.array([0, 3, 5], dtype=np.int64)
    indices = np.array([1, 4, 6, 2, 4], dtype=np.int32)
    data = np.array([1.0, 2.0, 1.0, 1.0, 0.0], dtype=np.float32)
    offsets, words = pack([[0], [1], [0, 1], []])
    s, i = oracle.search(indptr, indices, data, 8, offsets, words, 5)
    assert i.tolist() == [[4, 1, 6, 0, 2], [2, 0, 1, 3, 4], [4, 1, 2, 6, 0], [0, 1, 2, 3, 4]]
    assert s[0].tolist() == [2.0, 1.0, 1.0, 0.0, 0.0]


def test_oracle_rejects_invalid_words(oracle_mod):
    indptr = np.array([0, 1], dtype=np.int64)
    for bad in ([-1], [2**31 - 1]):
        offsets, words = pack([bad])
        with pytest.raises(ValueError):
            oracle_mod.search(indptr, np.array([0], np.int32), np.ones(1, np.float32), 2, offsets, words, 1)


def test_merge_of_document_shards(pkg, oracle_mod):
    """Per-shard top-K lists merge to the global top-K (topk_document_shards.h:4)."""
    spec = pkg.CorpusSpec(docs=7000, vocab=3000, seed=8)
    index = pkg.synthetic_index(spec)
    data = oracle_mod.contributions(index, spec.k1)
    offsets, words = pkg.synthetic_queries(index.offsets, 4, 2, 5, 9)
    gs, gi = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words, 10)
    cuts = [0, 1500, 4000, 7000]
    parts = []
    for lo, hi in zip(cuts, cuts[1:]):
        # shard = documents [lo, hi) with global ids, as a doc-sharded engine holds them
        keep = (index.docs >= lo) & (index.docs < hi)
        c = np.concatenate([[0], np.cumsum(keep, dtype=np.int64)])
        indptr = c[index.offsets]
        parts.append((indptr, index.docs[keep], data[keep], lo, hi))
    for qi in range(4):
        lists_s, lists_i = [], []
        for indptr, docs, d, lo, hi in parts:
            s, i = oracle_mod.search(indptr, docs, d, index.num_docs, offsets[qi:qi + 2] - offsets[qi],
                                     words[offsets[qi]:offsets[qi + 1]], 10)
            # a shard only knows its own documents: replace out-of-shard zero fill by in-shard zero fill
            zs = [x for x in range(lo, hi) if x not in set(i[0][s[0] > 0].tolist())]
            pos = int((s[0] > 0).sum())
            s[0][pos:] = 0
            i[0][pos:] = zs[:10 - pos]
            lists_s.append(s[0])
            lists_i.append(i[0])
        ms, mi = oracle_mod.merge(np.stack(lists_s), np.stack(lists_i), 10)
        assert_same_topk(ms[None], mi[None], gs[qi:qi + 1], gi[qi:qi + 1])


def test_bm25s_port_scores_equal_oracle(pkg, oracle_mod):
    """The numba restatement of bm25s's retrieve (the timed bm25s CPU baseline) returns the oracle's top-K
    scores for every query (its ids may differ only among tied scores: bm25s does not rank ties)."""
    from oracle import bm25s_port
    if not bm25s_port.available():
        pytest.skip('numba not installed')
    spec = pkg.CorpusSpec(docs=20_000, vocab=4_000, seed=12, k1=1.2)
    index = pkg.synthetic_index(spec)
    data = oracle_mod.contributions(index, spec.k1)
    qo, w = pkg.synthetic_queries(index.offsets, 12, 1, 6, 9)
    for k in (1, 10, 50):
        bs, bi = bm25s_port.retrieve(index.offsets, index.docs, data, index.num_docs, qo, w, k, 2)
        rs, ri = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, qo, w, k)
        assert np.array_equal(np.sort(bs, axis=1), np.sort(rs, axis=1)), k
        untied = np.array([len(set(r)) == r.size for r in rs])
        assert np.array_equal(np.sort(bi[untied], axis=1), np.sort(ri[untied], axis=1)), k
