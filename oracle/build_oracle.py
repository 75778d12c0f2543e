"""CPU restatement of the reference's index builder (test infrastructure only).

Follows standalone/large_corpus.py:95-190: per document, term frequencies
(Counter); df per term; offsets by prefix sum; postings of a term in document
order; idf = f32(math.log1p((N - df + 0.5) / (df + 0.5))); norm =
f32(k1 * (1 - b + b * len / average)) with average = total tokens / N, both in
double (the reference hard-codes k1 1.2, b 0.75).  Pinned against the
reference's own output in tests/golden/large_corpus_n2048.npz.
"""

import math

import numpy as np


def build(doc_offsets, tokens, vocab, k1=1.2, b=0.75):
    doc_offsets = np.asarray(doc_offsets, dtype=np.int64)
    tokens = np.asarray(tokens, dtype=np.int64)
    n = doc_offsets.size - 1
    doc_of = np.repeat(np.arange(n, dtype=np.int64), np.diff(doc_offsets))
    keys = tokens * (1 << 32) + doc_of
    uniq, counts = np.unique(keys, return_counts=True)  # term-major, document-ascending
    terms = uniq >> 32
    offsets = np.zeros(vocab + 1, dtype=np.int64)
    np.add.at(offsets, terms + 1, 1)
    offsets = np.cumsum(offsets)
    df = np.diff(offsets)
    idf = np.array([math.log1p((n - c + 0.5) / (c + 0.5)) for c in df.tolist()], dtype=np.float32)
    total = int(doc_offsets[-1])
    average = total / n
    lens = np.diff(doc_offsets).tolist()
    norm = np.array([k1 * (1 - b + b * length / average) for length in lens], dtype=np.float32)
    return offsets, (uniq & 0xffffffff).astype(np.int32), counts.astype(np.float32), norm, idf
