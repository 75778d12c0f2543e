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


def test_tuning_struct_and_null_handle(pkg):
    """bm25_tuning's layout (five 4-byte fields around one 8-byte one: 32 bytes) and the
    handle check of its entries, without a device."""
    import ctypes
    n = pkg._native
    assert ctypes.sizeof(n.Tuning) == 32 and n.Tuning.candidate_cap.offset == 16
    lib = n.engine_library()
    t = n.Tuning()
    assert lib.bm25_get_tuning(None, ctypes.byref(t)) == n.BM25_ERR_ILLEGAL_OPERATION
    assert lib.bm25_set_tuning(None, ctypes.byref(t)) == n.BM25_ERR_ILLEGAL_OPERATION


class _FakeSession:
    def __init__(self, kernel, max_k):
        self._info = {'kernel': kernel, 'max_k': max_k}

    def info(self):
        return self._info


def test_tuning_space_follows_the_kernel(pkg):
    space = pkg.autotune.tuning_space(_FakeSession(5, 10), 10)
    assert set(space) == {'claim_tiles', 'tail_claims', 'ring_stages', 'ring_chunk'}
    space = pkg.autotune.tuning_space(_FakeSession(4, 1000), 100, learned=True)
    assert set(space) == {'ring_stages', 'ring_chunk', 'candidate_cap', 'prune_route'}
    assert space['candidate_cap'] == (0, 8000)
    assert pkg.autotune.tuning_space(_FakeSession(0, 10), 10) == {}


@pytest.mark.gpu
def test_set_tuning_checks_and_keeps_results(pkg, oracle_mod, cuda_ok):
    """Every accepted tuning answers the oracle's bits; invalid fields are refused without
    changing the session; a change drops the instantiated graphs."""
    spec = pkg.CorpusSpec(docs=300_000, vocab=20_000, seed=31, k1=1.2)
    index = pkg.synthetic_index(spec)
    data = oracle_mod.contributions(index, spec.k1)
    qo, w = pkg.synthetic_queries(index.offsets, 16, 2, 4, 8)
    want10 = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, qo, w, 10)
    want100 = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, qo, w, 100)

    def same(got, want, what):
        assert np.array_equal(got[1], want[1]), what
        assert np.array_equal(got[0].view(np.uint32), want[0].view(np.uint32)), what

    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=16,
                                  word_capacity=64, max_k=100) as s:
        start = s.tuning()
        assert start['claim_tiles'] == 4 and start['tail_claims'] == 2 and start['candidate_cap'] == 0
        for bad in ({'claim_tiles': 3}, {'tail_claims': 9}, {'ring_stages': 1}, {'ring_chunk': 1002},
                    {'ring_chunk': 256}, {'candidate_cap': 50}, {'candidate_cap': 2044},
                    {'prune_route': float('nan')}):
            with pytest.raises(pkg.InvalidParam):
                s.set_tuning(**bad)
            assert s.tuning() == start, bad
        s.search_batch((qo, w), np.full(16, 10, np.int32))
        assert s.info()['graphs_cached'] >= 1
        for changes in ({'claim_tiles': 2, 'tail_claims': 0}, {'claim_tiles': 8, 'tail_claims': 4},
                        {'ring_stages': 2, 'ring_chunk': 1024}, {'candidate_cap': 2048},
                        {'candidate_cap': 2050}):
            s.set_tuning(**changes)
            assert s.info()['graphs_cached'] == 0
            got = s.tuning()
            for key, value in changes.items():
                assert got[key] == (value + 3) // 4 * 4 if key == 'candidate_cap' else got[key] == value
            same(s.search((qo, w), 10), want10, f'{changes} K=10')
            same(s.search((qo, w), 100), want100, f'{changes} K=100')  # a narrow capacity retries
        assert s.info()['ring_stages'] == 2 and s.info()['ring_chunk'] == 1024


@pytest.mark.gpu
def test_tune_on_a_live_session(pkg, oracle_mod, cuda_ok):
    spec = pkg.CorpusSpec(docs=300_000, vocab=20_000, seed=32, k1=1.2)
    index = pkg.synthetic_index(spec)
    data = oracle_mod.contributions(index, spec.k1)
    qo, w = pkg.synthetic_queries(index.offsets, 16, 2, 4, 9)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=16,
                                  word_capacity=64) as s:
        space = {'claim_tiles': (2, 4), 'tail_claims': (1, 2)}
        best, table = pkg.autotune.tune(s, (qo, w), 10, space=space, reps=3)
        assert len(table) == 4 and all(ms > 0 for _, ms in table)
        assert {k: best[k] for k in space} in [c for c, _ in table]
        assert s.tuning() == best
        got = s.search((qo, w), 10)
    want = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, qo, w, 10)
    assert np.array_equal(got[1], want[1]) and np.array_equal(got[0].view(np.uint32), want[0].view(np.uint32))
