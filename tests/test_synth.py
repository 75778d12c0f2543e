"""Seeded synthetic corpus generator: determinism and the reference's index formulas."""

import math

import numpy as np


def test_deterministic_for_any_thread_count(pkg):
    spec = pkg.CorpusSpec(docs=12345, vocab=5000, seed=3)
    a = pkg.synthetic_index(spec, threads=1)
    b = pkg.synthetic_index(spec, threads=7)
    for f in ('offsets', 'docs', 'tf', 'norm', 'idf', 'doc_len'):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


def test_index_invariants_and_formulas(pkg):
    spec = pkg.CorpusSpec(docs=4000, vocab=3000, seed=5, k1=1.5, b=0.75)
    idx = pkg.synthetic_index(spec)
    df = idx.df()
    assert idx.offsets[0] == 0 and idx.offsets[-1] == idx.postings and (df >= 0).all()
    for t in np.flatnonzero(df)[:200]:
        d = idx.docs[idx.offsets[t]:idx.offsets[t + 1]]
        assert (np.diff(d) > 0).all() and d.min() >= 0 and d.max() < spec.docs
    assert (idx.tf >= 1).all() and (idx.tf == np.floor(idx.tf)).all()
    # per-document tf sums to the document length
    assert np.array_equal(np.bincount(idx.docs, weights=idx.tf, minlength=spec.docs).astype(np.int64),
                          idx.doc_len.astype(np.int64))
    avg = idx.doc_len.sum() / spec.docs
    for d in (0, 17, 3999):  # large_corpus.py:174 with k1 = 1.5
        assert idx.norm[d] == np.float32(1.5 * (1 - 0.75 + 0.75 * idx.doc_len[d] / avg))
    for t in (0, 5, 2999):   # large_corpus.py:148
        assert idx.idf[t] == np.float32(math.log1p((spec.docs - df[t] + 0.5) / (df[t] + 0.5)))


def test_zipf_and_length_shape(pkg):
    spec = pkg.CorpusSpec(docs=20000, vocab=30000, seed=1)
    idx = pkg.synthetic_index(spec)
    assert abs(idx.doc_len.mean() - 60) < 1.5
    df = idx.df()
    assert df[0] > df[10] > df[1000] > 0  # rank order by frequency


def test_queries_distinct_and_df_weighted(pkg):
    spec = pkg.CorpusSpec(docs=5000, vocab=30000, seed=2)
    idx = pkg.synthetic_index(spec)
    qo, w = pkg.synthetic_queries(idx.offsets, 64, 3, 3, 7)
    assert qo.tolist() == list(range(0, 193, 3))
    rows = w.reshape(64, 3)
    assert all(len(set(r)) == 3 for r in rows.tolist())
    assert np.median(idx.df()[w]) > np.median(idx.df()[idx.df() > 0])
    qo2, w2 = pkg.synthetic_queries(idx.offsets, 64, 3, 3, 7)
    assert np.array_equal(w, w2)


def test_index_files_round_trip(pkg, tmp_path):
    spec = pkg.CorpusSpec(docs=1000, vocab=500, seed=9)
    idx = pkg.synthetic_index(spec)
    pkg.write_index_dir(idx, tmp_path)
    back = pkg.read_index_dir(tmp_path)
    for f in ('offsets', 'docs', 'tf', 'norm', 'idf'):
        assert np.array_equal(getattr(idx, f), getattr(back, f))


def test_reference_shaped_corpus(pkg):
    """The reference's benchmark corpus shape (standalone/large_corpus.py:58-62): tokens uniform over
    1024 terms, lengths uniform in 16..48, k1 1.2; deterministic for any thread count."""
    import dataclasses
    spec = dataclasses.replace(pkg.CONFIG_SHAPES['reference_10m'], docs=40_000)
    assert (spec.vocab, spec.zipf_s, spec.k1, spec.b, spec.seed) == (1024, 0.0, 1.2, 0.75, 20261014)
    a = pkg.synthetic_index(spec, threads=1)
    b = pkg.synthetic_index(spec, threads=4)
    assert np.array_equal(a.offsets, b.offsets) and np.array_equal(a.docs, b.docs)
    assert a.doc_len.min() == 16 and a.doc_len.max() == 48
    assert abs(a.doc_len.mean() - 32.0) < 0.3
    counts = np.bincount(a.doc_len - 16, minlength=33)
    assert counts.min() > 0.8 * counts.mean()  # every length in 16..48 about equally often
    df = np.diff(a.offsets)
    assert df.min() > 0.85 * df.mean() and df.max() < 1.15 * df.mean()  # no term favoured
