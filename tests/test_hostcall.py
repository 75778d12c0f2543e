"""The Python entry points of the host-buffer Searches (_hostcall, over the buffer protocol): they
check their arrays before the C ABI sees them, and pass the ABI's status through.  No device is
needed: without a handle the ABI answers ILLEGAL_OPERATION."""

import numpy as np
import pytest


@pytest.fixture(scope='module')
def hc(pkg):
    return pkg._native.hostcall()


def _batch():
    offsets = np.array([0, 3, 5], dtype=np.int64)
    words = np.array([1, 2, 3, 4, 5], dtype=np.int32)
    return offsets, words, np.empty((2, 10), np.float32), np.empty((2, 10), np.int32), np.empty(2, np.int32)


def test_status_passes_through_without_a_handle(pkg, hc):
    o, w, s, i, e = _batch()
    assert hc.search(0, o, w, 2, 10, s, i) == pkg._native.BM25_ERR_ILLEGAL_OPERATION
    assert hc.search_learned(0, o, w, 2, 10, s, i, e) == pkg._native.BM25_ERR_ILLEGAL_OPERATION


@pytest.mark.parametrize('bad', ['short_words', 'float64_scores', 'int64_ids', 'short_ids', 'strided', 'q0', 'k0',
                                 'readonly_out'])
def test_arrays_are_checked(hc, bad):
    o, w, s, i, e = _batch()
    q, k = 2, 10
    if bad == 'short_words':
        w = w[:4]
    elif bad == 'float64_scores':
        s = s.astype(np.float64)
    elif bad == 'int64_ids':
        i = i.astype(np.int64)
    elif bad == 'short_ids':
        i = i[:1]
    elif bad == 'strided':
        s = np.empty((2, 20), np.float32)[:, ::2]
    elif bad == 'q0':
        q = 0
    elif bad == 'k0':
        k = 0
    elif bad == 'readonly_out':
        s.flags.writeable = False
    with pytest.raises((ValueError, BufferError)):
        hc.search(0, o, w, q, k, s, i)


def test_session_maps_check_failures_to_invalid_param(pkg):
    """A session call whose arrays fail the checks raises InvalidParam (the handle is never used)."""
    s = pkg.Bm25Session.__new__(pkg.Bm25Session)
    s._lib = pkg._native.engine_library()
    s._call = pkg._native.hostcall()
    s._handle = None
    s._handle_int = 0
    o, w, sc, ids, _ = _batch()
    with pytest.raises(pkg.InvalidParam):
        s.search((o, w), 10, out=(sc.astype(np.float64), ids))
