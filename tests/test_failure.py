"""The device-error contract, tested without faulting a GPU.

The reference's session reports a device failure as INNER_ERROR, poisons itself,
and answers every later call with ILLEGAL_OPERATION until it is closed
(large_search.cpp:193-210; tested with a mocked failing session in
ut/cases/bm25/sdk_facade_tests.cpp:47-56).  Here the failure is made in two ways:
on the host (bm25_test_inject, BM25_INJECT_HOST_FAILURE), and on the device by a
ring producer that issues nothing, so that its consumers' bounded mbarrier waits
run out after a short budget and the kernel reports kStatusTimeout (16) in the
Search's status word.  No wait is endless and nothing faults: the context stays
usable, as the last session of each test shows.
"""

import numpy as np
import pytest

from helpers import assert_same_topk

TIMEOUT_BIT = 16  # kStatusTimeout


@pytest.fixture(scope='module')
def corpus(pkg, oracle_mod):
    spec = pkg.CONFIG_SHAPES['synthetic_8192']
    index = pkg.synthetic_index(spec)
    return spec, index, oracle_mod.contributions(index, spec.k1)


def test_inject_arguments_are_checked(pkg):
    """A handle-less injection can only be a host failure (no device needed)."""
    n = pkg._native
    lib = n.engine_library()
    assert lib.bm25_test_inject(None, n.BM25_INJECT_STALL) == n.BM25_ERR_INVALID_PARAM
    assert lib.bm25_test_inject(None, 99) == n.BM25_ERR_INVALID_PARAM


@pytest.mark.gpu
def test_host_injected_failure_poisons_the_session(pkg, oracle_mod, corpus, cuda_ok):
    spec, index, data = corpus
    offsets, words = pkg.synthetic_queries(index.offsets, 8, 3, 3, 2)
    want = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words, 10)
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs) as s:
        assert_same_topk(*s.search((offsets, words), 10), *want, 'before the failure')
        s.inject(pkg._native.BM25_INJECT_HOST_FAILURE)
        with pytest.raises(pkg.InnerError, match='Injected device failure'):
            s.search((offsets, words), 10)
        with pytest.raises(pkg.IllegalOperation):
            s.search((offsets, words), 10)
        with pytest.raises(pkg.IllegalOperation):
            s.inject(pkg._native.BM25_INJECT_HOST_FAILURE)
    # a fresh session on the same device works
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs) as s:
        assert_same_topk(*s.search((offsets, words), 10), *want, 'new session')


@pytest.mark.gpu
def test_bounded_wait_runs_out(pkg, oracle_mod, corpus, cuda_ok):
    """The tile-group kernel with a wait budget of 10^6 cycles (about 0.5 ms): a normal Search is
    unaffected; with its producer stalled, every consumer's wait gives up, the kernel reports the
    timeout, the call fails with INNER_ERROR and the session is poisoned."""
    spec, index, data = corpus
    offsets, words = pkg.synthetic_queries(index.offsets, 8, 3, 3, 3)
    want = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words, 10)
    s = pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, kernel=4,
                                 wait_budget_cycles=1_000_000)
    try:
        assert_same_topk(*s.search((offsets, words), 10), *want, 'short budget, no stall')
        s.inject(pkg._native.BM25_INJECT_STALL)
        with pytest.raises(pkg.InnerError) as err:
            s.search((offsets, words), 10)
        status = int(str(err.value).split('status=')[1].split()[0].rstrip('.,;'))
        assert status & TIMEOUT_BIT, str(err.value)
        with pytest.raises(pkg.IllegalOperation):
            s.search((offsets, words), 10)
    finally:
        s.close()
    # the warp-tile kernel has no wait to stall: the hook leaves its Search exact
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, kernel=5) as w:
        w.inject(pkg._native.BM25_INJECT_STALL)
        assert_same_topk(*w.search((offsets, words), 10), *want, 'warp tile ignores the stall')
        assert_same_topk(*w.search((offsets, words), 10), *want, 'warp tile after the stall')
