"""GPU index builder (bm25_build_index) against the reference's own builder output.

tests/golden/large_corpus_n2048.npz holds the documents the reference's generator
made (standalone/large_corpus.documents) and the lazy index its builder wrote
(standalone/large_corpus.py:95-190).  CPU: the oracle's restatement reproduces
that index bit for bit.  GPU: the device builder does too, a larger token corpus
matches the restatement, the built index searches like the reference, and
invalid tokens are refused.
"""

from pathlib import Path

import numpy as np
import pytest

from helpers import assert_same_topk, bits

GOLDEN = Path(__file__).resolve().parent / 'golden'


@pytest.fixture(scope='module')
def golden():
    z = np.load(GOLDEN / 'large_corpus_n2048.npz')
    return {k: z[k] for k in z.files}


def _same_index(got, g, label):
    offsets, docs, tf, norm, idf = got
    assert np.array_equal(offsets, g['offsets']), label
    assert np.array_equal(docs, g['docs']), label
    assert np.array_equal(bits(tf), bits(g['tf'])), label
    assert np.array_equal(bits(norm), bits(g['norm'])), label
    assert np.array_equal(bits(idf), bits(g['idf'])), label


def test_restatement_matches_reference_builder(golden):
    from oracle import build_oracle
    vocab = int(golden['meta'][1])
    _same_index(build_oracle.build(golden['doc_offsets'], golden['tokens'], vocab), golden, 'restatement')


def _random_tokens(seed, docs, vocab):
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 80, docs)
    p = np.arange(1, vocab + 1, dtype=np.float64) ** -1.1
    p /= p.sum()
    tokens = rng.choice(vocab, size=int(lens.sum()), p=p).astype(np.int32)
    return np.concatenate([[0], np.cumsum(lens)]).astype(np.int64), tokens


@pytest.mark.gpu
def test_gpu_builder_matches_reference_and_restatement(pkg, oracle_mod, golden, cuda_ok):
    from oracle import build_oracle
    vocab = int(golden['meta'][1])
    idx = pkg.build_index(golden['doc_offsets'], golden['tokens'], vocab)
    _same_index((idx.offsets, idx.docs, idx.tf, idx.norm, idx.idf), golden, 'gpu builder')
    with pkg.Bm25Session.from_lazy(idx.offsets, idx.docs, idx.tf, idx.norm, idx.idf, k1=1.2) as s:
        for case in ('A', 'B'):
            got = s.search((golden[f'{case}_offsets'], golden[f'{case}_words']), 10)
            assert_same_topk(*got, golden[f'{case}_top_scores'], golden[f'{case}_top_ids'], case)
    doc_offsets, tokens = _random_tokens(5, 50_000, 70_000)  # empty documents and unused terms included
    idx = pkg.build_index(doc_offsets, tokens, 70_000, k1=1.5, b=0.75)
    want = build_oracle.build(doc_offsets, tokens, 70_000, k1=1.5, b=0.75)
    for got, exp, name in zip((idx.offsets, idx.docs, idx.tf, idx.norm, idx.idf), want,
                              ('offsets', 'docs', 'tf', 'norm', 'idf')):
        assert np.array_equal(np.asarray(got).view(np.uint8), np.asarray(exp).view(np.uint8)), name
    bad = tokens.copy()
    bad[17] = 70_000
    with pytest.raises(ValueError):
        pkg.build_index(doc_offsets, bad, 70_000)
