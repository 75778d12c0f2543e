"""Final selection with many exactly tied scores: bit-exact, ties ranked by ascending id.

Equal-score postings spread over many tiles give the final select anything from a
few to hundreds of candidates at its floor, so its pairwise rank (a few
survivors), its sort in shared memory (up to 512) and its re-filtered path (more)
all have to order ties by document id as the oracle does; the same corpus goes
through the plain path, the block-pruned path with the safe bounds, and K above 32.
"""

import numpy as np
import pytest

from helpers import assert_same_topk, pack

N = 65536  # 64 tiles of 1024 documents


def tied_corpus():
    """Eager CSC of four terms whose posting scores repeat exactly."""
    rng = np.random.default_rng(12)
    every7 = np.arange(0, N, 7)
    lists = [
        (every7, np.full(every7.size, 1.0)),  # every tile, one score
        (np.arange(3, 20 * 1024, 7), 0.5),  # the first 20 tiles, one score
        (np.sort(rng.choice(N, 300, replace=False)), rng.choice([0.25, 0.5, 0.75], 300)),  # three scores
        (np.sort(np.concatenate([np.arange(5, N, 1024), np.arange(900, N, 1024)])), 2.0),  # two per tile
    ]
    indptr, ids, vals = [0], [], []
    for docs, score in lists:
        docs = np.asarray(docs, np.int32)
        ids.append(docs)
        vals.append(np.broadcast_to(np.asarray(score, np.float32), docs.shape))
        indptr.append(indptr[-1] + docs.size)
    return (np.array(indptr, np.int64), np.concatenate(ids).astype(np.int32),
            np.concatenate(vals).astype(np.float32))


ROWS = [[0], [1], [2], [3], [0, 1], [1, 0], [0, 3], [2, 3, 1], [3, 3], [0, 2]]


def test_tied_corpus_shape():
    indptr, indices, data = tied_corpus()
    assert indptr[-1] == indices.size == data.size
    for t in range(indptr.size - 1):
        d = indices[indptr[t]:indptr[t + 1]]
        assert np.all(np.diff(d) > 0) and d[0] >= 0 and d[-1] < N
    assert np.unique(data).size == 5  # 0.25, 0.5, 0.75, 1.0 and 2.0: every score repeats


@pytest.mark.gpu
@pytest.mark.parametrize('prune', [False, True])
def test_tied_scores_rank_by_id(pkg, oracle_mod, cuda_ok, prune):
    indptr, indices, data = tied_corpus()
    offsets, words = pack(ROWS)
    with pkg.Bm25Session.from_csc(indptr, indices, data, N, query_capacity=16, word_capacity=64, max_k=32,
                                  prune=prune) as s:
        if prune:
            s.set_threshold_model(None)  # the safe bounds: K-th posting scores, themselves tied
        for k in (1, 10, 32):
            want = oracle_mod.search(indptr, indices, data, N, offsets, words, k)
            assert_same_topk(*s.search((offsets, words), k), *want, f'plain k={k}')
            if prune:
                got_s, got_i, exact = s.search_learned((offsets, words), k)
                assert_same_topk(got_s, got_i, *want, f'safe bounds k={k}')
                assert exact.all(), 'the safe bounds never fall back'
            assert s.device_status() == 0


@pytest.mark.gpu
def test_tied_scores_large_k(pkg, oracle_mod, cuda_ok):
    indptr, indices, data = tied_corpus()
    offsets, words = pack(ROWS)
    with pkg.Bm25Session.from_csc(indptr, indices, data, N, query_capacity=16, word_capacity=64,
                                  max_k=1000) as s:
        for k in (33, 100, 1000):
            want = oracle_mod.search(indptr, indices, data, N, offsets, words, k)
            assert_same_topk(*s.search((offsets, words), k), *want, f'k={k}')
            assert s.device_status() == 0


@pytest.mark.gpu
def test_ties_beyond_the_candidate_buffer_are_reported(pkg, cuda_ok):
    """K > 32 keeps every document at or above the running bound in a buffer of candidate_capacity per
    query.  When more documents than that tie at the K-th score (term 0: 9,363 documents, all 1.0; K =
    1000, 2,048 slots), every retry pass starts from that score and overflows again: the Search reports a
    device error (candidate overflow, status bit 32) instead of a wrong answer, as bm25_b200.h states."""
    indptr, indices, data = tied_corpus()
    offsets, words = pack([[0]])
    with pkg.Bm25Session.from_csc(indptr, indices, data, N, query_capacity=1, word_capacity=4, max_k=1000,
                                  candidate_capacity=2048) as s:
        with pytest.raises(pkg.InnerError) as err:
            s.search((offsets, words), 1000)
        status = int(str(err.value).split('status=')[1].split()[0].rstrip('.,;'))
        assert status & 32, str(err.value)
