"""Shared test helpers: seeded corpora, queries and bit-exact comparison."""

import numpy as np

# Query sets of the reference's CPU unit test (ut/cases/bm25/cpu_index_search_tests.cpp:100-102):
# duplicated terms, an empty query, out-of-vocabulary ids and 2147483646.
EDGE_A = [[0, 0], [], [6], [7], [4, 5, 0], [2147483646, 2], [0, 1, 2, 3]]
EDGE_B = [[4], [0], [], [7], [2, 2, 1]]


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def assert_same_topk(scores, ids, ref_scores, ref_ids, label=''):
    """Bit-exact: identical ids and identical FP32 score bits, rank by rank."""
    scores = np.asarray(scores).reshape(np.shape(ref_scores))
    ids = np.asarray(ids).reshape(np.shape(ref_ids))
    if not np.array_equal(ids, ref_ids) or not np.array_equal(bits(scores), bits(ref_scores)):
        bad = np.argwhere((ids != ref_ids) | (bits(scores) != bits(ref_scores)))
        q, r = bad[0]
        raise AssertionError(f'{label} top-K differs at query {q} rank {r}: got ({scores[q, r]!r}, {ids[q, r]}) '
                             f'expected ({ref_scores[q, r]!r}, {ref_ids[q, r]}); {len(bad)} mismatching slots')


def mixed_queries(vocab, rng, count, lo=0, hi=8, oov=True):
    """Random query rows with duplicates, empty rows and out-of-vocabulary ids."""
    rows = []
    for _ in range(count):
        n = int(rng.integers(lo, hi + 1))
        row = [int(x) for x in rng.integers(0, vocab, size=n)]
        if n and rng.random() < 0.3:
            row.append(row[0])  # duplicate term, added again in order
        if oov and rng.random() < 0.2:
            row.insert(int(rng.integers(0, len(row) + 1)), int(vocab + rng.integers(0, 1000)))
        rows.append(row[:64])
    return rows


def pack(rows):
    offsets = np.zeros(len(rows) + 1, dtype=np.int64)
    for i, r in enumerate(rows):
        offsets[i + 1] = offsets[i] + len(r)
    words = np.array([w for r in rows for w in r], dtype=np.int32)
    return offsets, words
