"""bm25_search_csc_static: Search over a caller-held device CSC index with no device allocation.

Checked against the session entry point (bm25_create + bm25_search) on the same
index and queries: top-K ids and FP32 score bits must be identical, on two
calls in a row (the scratch array keeps the previous call's contents).
"""

import ctypes
from ctypes import c_void_p

import numpy as np
import pytest

from helpers import assert_same_topk, mixed_queries, pack

STATIC_SCRATCH_BYTES = 16 << 20


def _call(lib, indptr, indices, data, vocab, num_docs, qoffsets, words, q, num_words, k, scores, ids, stream=None,
          device=0):
    return lib.bm25_search_csc_static(c_void_p(indptr), c_void_p(indices), c_void_p(data), vocab, num_docs,
                                      c_void_p(qoffsets), c_void_p(words), q, num_words, k, c_void_p(scores),
                                      c_void_p(ids), c_void_p(stream), device)


def _error(lib):
    buf = ctypes.create_string_buffer(512)
    code = ctypes.c_int64(0)
    lib.bm25_last_error(None, buf, len(buf), ctypes.byref(code))
    return buf.value.decode()


def test_static_rejects_before_touching_the_device(pkg):
    """Argument and size checks run on the host before any CUDA call (no device needed)."""
    from importlib import import_module
    n = import_module('bm25-npu_b200._native')
    lib = n.engine_library()
    fake = 1 << 12  # aligned, never dereferenced: every case below is rejected first
    assert _call(lib, 0, fake, fake, 10, 100, fake, fake, 1, 1, 5, fake, fake) == n.BM25_ERR_INVALID_PARAM
    assert 'Null' in _error(lib)
    assert _call(lib, fake, fake + 4, fake, 10, 100, fake, fake, 1, 1, 5, fake, fake) == n.BM25_ERR_INVALID_PARAM
    assert 'aligned' in _error(lib)
    assert _call(lib, fake, fake, fake, 10, 100, fake, fake, 1, 1, 33, fake, fake) == n.BM25_ERR_INVALID_PARAM
    # 10M docs -> 1221 tiles of 8192; 64 queries x 32 x 8 warps x 1221 tiles x 8 B >> 16 MiB
    assert _call(lib, fake, fake, fake, 10, 10_000_000, fake, fake, 64, 64, 32, fake, fake) == \
        n.BM25_ERR_INVALID_PARAM
    assert str(STATIC_SCRATCH_BYTES) in _error(lib)


@pytest.mark.gpu
def test_static_matches_session_twice(pkg, oracle_mod, cuda_ok):
    import torch
    from importlib import import_module
    n = import_module('bm25-npu_b200._native')
    lib = n.engine_library()
    spec = pkg.CorpusSpec(docs=120_000, vocab=40_000, seed=23, k1=1.2)
    index = pkg.synthetic_index(spec)
    data = oracle_mod.contributions(index, spec.k1)
    m = int(index.offsets[-1])
    padded = (m + 3) // 4 * 4  # the kernel reads postings in 16-byte units
    dev = torch.device('cuda:0')
    d_indptr = torch.from_numpy(np.ascontiguousarray(index.offsets, dtype=np.int64)).to(dev)
    d_indices = torch.zeros(padded, dtype=torch.int32, device=dev)
    d_indices[:m] = torch.from_numpy(np.ascontiguousarray(index.docs, dtype=np.int32)).to(dev)
    d_data = torch.zeros(padded, dtype=torch.float32, device=dev)
    d_data[:m] = torch.from_numpy(data).to(dev)
    stream = torch.cuda.current_stream(dev)

    batches = [
        (pkg.synthetic_queries(index.offsets, 8, 3, 3, 7), 10),
        (pack(mixed_queries(index.vocab, np.random.default_rng(3), 16, 0, 12, oov=True) + [[0, 1, 2], []]), 32),
    ]
    with pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=32,
                                  word_capacity=512, max_k=32) as session:
        for (offsets, words), k in batches:
            q = offsets.size - 1
            nw = int(offsets[-1])
            want = session.search((offsets, words), k)
            assert_same_topk(*want, *oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets,
                                                      words, k), 'session')
            d_off = torch.from_numpy(offsets).to(dev)
            d_words = torch.from_numpy(words if words.size else np.zeros(1, np.int32)).to(dev)
            d_scores = torch.full((q, k), -1.0, dtype=torch.float32, device=dev)
            d_ids = torch.full((q, k), -1, dtype=torch.int32, device=dev)
            status = _call(lib, d_indptr.data_ptr(), d_indices.data_ptr(), d_data.data_ptr(), index.vocab,
                           index.num_docs, d_off.data_ptr(), d_words.data_ptr(), q, nw, k, d_scores.data_ptr(),
                           d_ids.data_ptr(), stream.cuda_stream)
            assert status == n.BM25_OK, _error(lib)
            assert_same_topk(d_scores.cpu().numpy(), d_ids.cpu().numpy(), *want, f'static k={k}')

        # an invalid word in the device packet is reported as a parameter error; the next call still works
        offsets, words = pack([[1, -5]])
        d_off = torch.from_numpy(offsets).to(dev)
        d_words = torch.from_numpy(words).to(dev)
        d_scores = torch.empty((1, 10), dtype=torch.float32, device=dev)
        d_ids = torch.empty((1, 10), dtype=torch.int32, device=dev)
        status = _call(lib, d_indptr.data_ptr(), d_indices.data_ptr(), d_data.data_ptr(), index.vocab,
                       index.num_docs, d_off.data_ptr(), d_words.data_ptr(), 1, 2, 10, d_scores.data_ptr(),
                       d_ids.data_ptr(), stream.cuda_stream)
        assert status == n.BM25_ERR_INVALID_PARAM
        (offsets, words), k = batches[0]
        want = session.search((offsets, words), k)
        d_off = torch.from_numpy(offsets).to(dev)
        d_words = torch.from_numpy(words).to(dev)
        d_scores = torch.empty((offsets.size - 1, k), dtype=torch.float32, device=dev)
        d_ids = torch.empty((offsets.size - 1, k), dtype=torch.int32, device=dev)
        status = _call(lib, d_indptr.data_ptr(), d_indices.data_ptr(), d_data.data_ptr(), index.vocab,
                       index.num_docs, d_off.data_ptr(), d_words.data_ptr(), offsets.size - 1, int(offsets[-1]), k,
                       d_scores.data_ptr(), d_ids.data_ptr(), stream.cuda_stream)
        assert status == n.BM25_OK, _error(lib)
        assert_same_topk(d_scores.cpu().numpy(), d_ids.cpu().numpy(), *want, 'static after error')


@pytest.mark.gpu
def test_static_exact_scratch_boundary(pkg, oracle_mod, cuda_ok):
    """A Search that needs exactly the 16 MiB of the array runs; one word more (16 bytes more) is
    rejected before any device work.  2048 documents make one 2048-document tile on any SM count, so
    the need is 256 + 2 a16(4 q) + 128 q + 64 q k + 16 num_words: q = 7680, k = 32 and 240 words
    come to 16,777,216 bytes."""
    import torch
    from importlib import import_module
    n = import_module('bm25-npu_b200._native')
    lib = n.engine_library()
    spec = pkg.CorpusSpec(docs=2048, vocab=3000, seed=31, k1=1.2)
    index = pkg.synthetic_index(spec)
    data = oracle_mod.contributions(index, spec.k1)
    m = int(index.offsets[-1])
    dev = torch.device('cuda:0')
    d_indptr = torch.from_numpy(np.ascontiguousarray(index.offsets, dtype=np.int64)).to(dev)
    d_indices = torch.zeros((m + 3) // 4 * 4, dtype=torch.int32, device=dev)
    d_indices[:m] = torch.from_numpy(np.ascontiguousarray(index.docs, dtype=np.int32)).to(dev)
    d_data = torch.zeros((m + 3) // 4 * 4, dtype=torch.float32, device=dev)
    d_data[:m] = torch.from_numpy(data).to(dev)
    stream = torch.cuda.current_stream(dev)
    q, k = 7680, 32
    a16 = lambda x: (x + 15) // 16 * 16  # noqa: E731
    need = lambda nw: 256 + 2 * a16(4 * q) + 128 * q + 64 * q * k + 16 * max(1, nw)  # noqa: E731
    assert need(240) == STATIC_SCRATCH_BYTES
    rng = np.random.default_rng(8)
    for nw, ok in ((240, True), (241, False)):
        rows = [[] for _ in range(q)]
        for i in range(nw):  # 80 queries of 3 words, the 241st word on a query of its own
            rows[i // 3 if i < 240 else 100].append(int(rng.integers(0, index.vocab)))
        offsets, words = pack(rows)
        assert int(offsets[-1]) == nw
        d_off = torch.from_numpy(offsets).to(dev)
        d_words = torch.from_numpy(words).to(dev)
        d_scores = torch.full((q, k), -1.0, dtype=torch.float32, device=dev)
        d_ids = torch.full((q, k), -1, dtype=torch.int32, device=dev)
        status = _call(lib, d_indptr.data_ptr(), d_indices.data_ptr(), d_data.data_ptr(), index.vocab,
                       index.num_docs, d_off.data_ptr(), d_words.data_ptr(), q, nw, k, d_scores.data_ptr(),
                       d_ids.data_ptr(), stream.cuda_stream)
        if ok:
            assert status == n.BM25_OK, _error(lib)
            want = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words, k)
            assert_same_topk(d_scores.cpu().numpy(), d_ids.cpu().numpy(), *want, f'static at {need(nw)} bytes')
        else:
            assert status == n.BM25_ERR_INVALID_PARAM
            assert str(need(nw)) in _error(lib) and str(STATIC_SCRATCH_BYTES) in _error(lib)
            assert (d_ids == -1).all().item(), 'a rejected Search wrote its output'
