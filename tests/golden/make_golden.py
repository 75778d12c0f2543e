"""Generates the golden fixtures in this folder by running the reference's own Python code.

Run once, in a checkout that has the reference tree (default location below or
REFERENCE_ROOT); the fixtures are committed so tests never need the reference.

  large_corpus_n2048.npz  standalone/large_corpus.prepare (the reference's index builder and
                          original-document FP32 oracle) on 2048 docs, vocab 1024, seed 2026,
                          with the reference's query sets fixtures/A.txt and fixtures/B.txt, K 10:
                          the lazy index arrays, both query batches, expected_scores rows and
                          expected top-K ids / scores, and the generated documents' token ids
                          (doc_offsets, tokens: the input of the GPU index builder).
  bm25s_tiny.npz          the vendored bm25s (reference_only/bm25s_original, pinned commit
                          03eac5a8) eager index of a seeded 2000-doc token-id corpus (vocab 1500) (k1 1.5,
                          b 0.75, lucene): its CSC arrays, 16 queries, the query step's full score
                          rows (get_scores_from_ids) and the strict top-10 of the reference's
                          adapter (standalone/run_bm25s_reference.strict_select).
"""

import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = Path(os.environ.get('REFERENCE_ROOT', '/root/reference'))


def large_corpus():
    sys.path.insert(0, str(REF / 'standalone'))
    import large_corpus as lc
    cases = {'A': lc.load_raw(REF / 'fixtures' / 'A.txt'), 'B': lc.load_raw(REF / 'fixtures' / 'B.txt')}
    n, vocab, seed, k = 2048, 1024, 2026, 10
    with tempfile.TemporaryDirectory() as tmp:
        out = Path(tmp) / 'prepared'
        lc.prepare(out, n, vocab, seed, cases, k=k)
        idx = out / 'index'
        arrays = {
            'offsets': np.fromfile(idx / 'term_offsets.bin', dtype='<i8'),
            'docs': np.fromfile(idx / 'posting_doc_ids.bin', dtype='<i4'),
            'tf': np.fromfile(idx / 'posting_tf.bin', dtype='<f4'),
            'norm': np.fromfile(idx / 'doc_norm.bin', dtype='<f4'),
            'idf': np.fromfile(idx / 'idf.bin', dtype='<f4'),
        }
        for case, rows in cases.items():
            q = len(rows)
            arrays[f'{case}_offsets'] = np.cumsum([0] + [len(r) for r in rows]).astype(np.int64)
            arrays[f'{case}_words'] = np.array([w for r in rows for w in r], dtype=np.int32)
            arrays[f'{case}_expected_scores'] = np.fromfile(out / case / 'expected_scores.bin',
                                                            dtype='<f4').reshape(q, n)
            arrays[f'{case}_top_ids'] = np.fromfile(out / case / 'expected_top_ids.bin', dtype='<i4').reshape(q, k)
            arrays[f'{case}_top_scores'] = np.fromfile(out / case / 'expected_top_scores.bin',
                                                       dtype='<f4').reshape(q, k)
    # the documents themselves (the reference's generator), for the GPU index builder
    docs = list(lc.documents(n, vocab, seed, None))
    arrays['doc_offsets'] = np.cumsum([0] + [len(d) for d in docs]).astype(np.int64)
    arrays['tokens'] = np.array([t for d in docs for t in d], dtype=np.int32)
    arrays['meta'] = np.array([n, vocab, seed, k], dtype=np.int64)
    np.savez_compressed(HERE / 'large_corpus_n2048.npz', **arrays)


def bm25s_tiny():
    sys.path.insert(0, str(REF / 'standalone'))
    import run_bm25s_reference as rb
    bm25s, _, _ = rb.load_reference()
    rng = np.random.default_rng(20261203)
    n_docs, vocab = 2000, 1500
    ranks = np.arange(1, vocab + 1, dtype=np.float64)
    p = ranks ** -1.1
    p /= p.sum()
    docs = [rng.choice(vocab, size=int(rng.integers(5, 60)), p=p).tolist() for _ in range(n_docs)]
    vocab_dict = {str(t): t for t in range(vocab)}
    model = bm25s.BM25(k1=1.5, b=0.75)
    model.index((docs, vocab_dict), create_empty_token=False, show_progress=False)
    queries = []
    for i in range(16):
        terms = rng.choice(vocab, size=int(rng.integers(1, 7)), p=p).tolist()
        if i % 5 == 0:
            terms.append(terms[0])  # duplicate term: added twice
        queries.append(terms)
    rows = np.stack([model.get_scores_from_ids(q) for q in queries]).astype(np.float32)
    sel = [rb.strict_select(np, row, 10) for row in rows]
    np.savez_compressed(
        HERE / 'bm25s_tiny.npz',
        indptr=np.asarray(model.scores['indptr'], dtype=np.int64),
        indices=np.asarray(model.scores['indices'], dtype=np.int32),
        data=np.asarray(model.scores['data'], dtype=np.float32),
        num_docs=np.array([model.scores['num_docs']], dtype=np.int64),
        q_offsets=np.cumsum([0] + [len(q) for q in queries]).astype(np.int64),
        q_words=np.array([w for q in queries for w in q], dtype=np.int32),
        rows=rows,
        top_scores=np.stack([s for s, _ in sel]).astype(np.float32),
        top_ids=np.stack([i for _, i in sel]).astype(np.int32),
    )


if __name__ == '__main__':
    large_corpus()
    bm25s_tiny()
