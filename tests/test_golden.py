"""Committed golden vectors made by the reference's own Python code (tests/golden/make_golden.py).

large_corpus_n2048.npz pins the lazy-index formula and the strict top-K against the
reference's index builder and original-document FP32 oracle
(standalone/large_corpus.py:95-297); bm25s_tiny.npz pins the eager CSC query step against
the vendored bm25s (scoring.py:345-368) and the reference's strict adapter
(standalone/run_bm25s_reference.py:93-101).  Both are checked bit for bit.
"""

from pathlib import Path

import numpy as np
import pytest

from helpers import assert_same_topk, bits

GOLDEN = Path(__file__).resolve().parent / 'golden'


@pytest.fixture(scope='module')
def large(pkg):
    z = np.load(GOLDEN / 'large_corpus_n2048.npz')
    index = pkg.LazyIndex(z['offsets'], z['docs'], z['tf'], z['norm'], z['idf'])
    return index, {k: z[k] for k in z.files}


@pytest.fixture(scope='module')
def tiny():
    z = np.load(GOLDEN / 'bm25s_tiny.npz')
    return {k: z[k] for k in z.files}


@pytest.mark.parametrize('case', ['A', 'B'])
def test_oracle_matches_reference_builder(oracle_mod, large, case):
    index, g = large
    data = oracle_mod.contributions(index, 1.2)  # the reference's 2.2F literal
    scores, ids, rows = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, g[f'{case}_offsets'],
                                          g[f'{case}_words'], 10, full=True)
    assert np.array_equal(bits(rows), bits(g[f'{case}_expected_scores']))
    assert_same_topk(scores, ids, g[f'{case}_top_scores'], g[f'{case}_top_ids'], case)
    lazy = oracle_mod.search(index.offsets, index.docs, None, index.num_docs, g[f'{case}_offsets'],
                             g[f'{case}_words'], 10, lazy=(index.tf, index.norm, index.idf), k1=1.2)
    assert_same_topk(*lazy, g[f'{case}_top_scores'], g[f'{case}_top_ids'], case + ' lazy')


def test_oracle_matches_bm25s_query_step(oracle_mod, tiny):
    n = int(tiny['num_docs'][0])
    scores, ids, rows = oracle_mod.search(tiny['indptr'], tiny['indices'], tiny['data'], n, tiny['q_offsets'],
                                          tiny['q_words'], 10, full=True)
    assert np.array_equal(bits(rows), bits(tiny['rows']))
    assert_same_topk(scores, ids, tiny['top_scores'], tiny['top_ids'], 'bm25s strict')


def test_bm25s_files_round_trip(pkg, tiny, tmp_path):
    n = int(tiny['num_docs'][0])
    pkg.write_bm25s_dir(tiny['indptr'], tiny['indices'], tiny['data'], n, tmp_path)
    indptr, indices, data, num_docs = pkg.read_bm25s_dir(tmp_path)
    assert num_docs == n
    assert np.array_equal(indptr, tiny['indptr']) and np.array_equal(indices, tiny['indices'])
    assert np.array_equal(bits(data), bits(tiny['data']))


def test_query_files_round_trip(pkg, large, tmp_path):
    _, g = large
    pkg.write_queries_dir(g['A_offsets'], g['A_words'], tmp_path)
    offsets, words = pkg.read_queries_dir(tmp_path)
    assert np.array_equal(offsets, g['A_offsets']) and np.array_equal(words, g['A_words'])
    (tmp_path / 'query_offsets.bin').write_bytes(np.array([0, 5], dtype='<i8').tobytes())
    with pytest.raises(ValueError):
        pkg.read_queries_dir(tmp_path)


@pytest.mark.gpu
@pytest.mark.parametrize('kernel', [0, 1, 4], ids=['stream', 'per_tile', 'tile_group'])
def test_engine_matches_reference_builder(pkg, large, cuda_ok, kernel):
    index, g = large
    with pkg.Bm25Session.from_lazy(index.offsets, index.docs, index.tf, index.norm, index.idf, k1=1.2,
                                   kernel=kernel) as s:
        for case in ('A', 'B', 'A'):
            got = s.search((g[f'{case}_offsets'], g[f'{case}_words']), 10)
            assert_same_topk(*got, g[f'{case}_top_scores'], g[f'{case}_top_ids'], case)


@pytest.mark.gpu
@pytest.mark.parametrize('kernel', [0, 1, 4], ids=['stream', 'per_tile', 'tile_group'])
def test_engine_matches_bm25s(pkg, tiny, cuda_ok, kernel):
    n = int(tiny['num_docs'][0])
    with pkg.Bm25Session.from_csc(tiny['indptr'], tiny['indices'], tiny['data'], n, query_capacity=16,
                                  word_capacity=64, kernel=kernel) as s:
        got = s.search((tiny['q_offsets'], tiny['q_words']), 10)
        assert_same_topk(*got, tiny['top_scores'], tiny['top_ids'], 'bm25s')
