"""Autotuner: the search space, and on the GPU a tuning run whose every configuration answers
the same bits and whose best configuration is one of those timed."""

import numpy as np
import pytest


def test_candidates_cover_the_space(pkg):
    c = pkg.autotune.candidates()
    assert len(c) == 2 * 3 * 3 and {'tile_docs', 'ring_chunk', 'ring_stages'} == set(c[0])
    big = pkg.autotune.candidates(max_k=1000)
    assert len(big) == 2 * len(c) and all('candidate_capacity' in o for o in big)
    small = pkg.autotune.candidates({'tile_docs': (1024,), 'ring_chunk': (1536,)})
    assert small == [{'ring_chunk': 1536, 'tile_docs': 1024}]


@pytest.mark.gpu
def test_autotune_picks_a_timed_configuration(pkg, oracle_mod, cuda_ok):
    spec = pkg.CorpusSpec(docs=200_000, vocab=20_000, seed=12, k1=1.2)
    index = pkg.synthetic_index(spec)
    data = oracle_mod.contributions(index, spec.k1)
    qo, w = pkg.synthetic_queries(index.offsets, 8, 3, 3, 4)
    space = {'tile_docs': (1024, 2048), 'ring_chunk': (1024, 1536), 'ring_stages': (3,)}
    best, table = pkg.autotune.autotune(index.offsets, index.docs, data, index.num_docs, (qo, w), 10, space=space,
                                        reps=5)
    assert len(table) == 4 and best in [opts for opts, _ in table]
    assert all(ms > 0 for _, ms in table)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=8,
                                  word_capacity=24, **best) as s:
        got = s.search((qo, w), 10)
    want = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, qo, w, 10)
    assert np.array_equal(got[1], want[1]) and np.array_equal(got[0].view(np.uint32), want[0].view(np.uint32))
