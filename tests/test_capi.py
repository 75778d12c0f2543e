"""The C-ABI library loads and exports every declared symbol; host-side validation needs no GPU."""

import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT


def _declared(header):
    text = (ROOT / 'include' / header).read_text()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(bm25_[a-z_]+)\s*\(', text)))


def test_engine_exports_every_declared_symbol(pkg):
    lib = pkg._native.engine_library()
    declared = _declared('bm25_b200.h')
    assert 'bm25_search' in declared and 'bm25_create' in declared
    for name in declared:
        assert hasattr(lib, name), f'{name} declared in include/bm25_b200.h but not exported'
    assert set(declared) == set(pkg._native.SIGNATURES), 'ctypes signature table out of sync with the header'


def test_default_options_match_reference_config(pkg):
    """Bm25Config defaults (AscendIndexBm25.h:17-25): device 0, 8 queries, 24 words, topK 10."""
    o = pkg._native.Options()
    pkg._native.engine_library().bm25_default_options(ctypes.byref(o))
    assert (o.device_id, o.query_capacity, o.word_capacity, o.max_k) == (0, 8, 24, 10)
    assert o.kernel == 5  # the warp-tile kernel


@pytest.mark.parametrize('case', ['unsorted', 'range', 'nan', 'negative', 'bounds'])
def test_invalid_eager_index_rejected_before_device(pkg, case):
    indptr = np.array([0, 2, 3], dtype=np.int64)
    indices = np.array([0, 1, 2], dtype=np.int32)
    data = np.ones(3, dtype=np.float32)
    if case == 'unsorted':
        indices[:2] = [1, 0]
    elif case == 'range':
        indices[2] = 9
    elif case == 'nan':
        data[1] = np.nan
    elif case == 'negative':
        data[0] = -1.0
    elif case == 'bounds':
        indptr[1] = 4
    with pytest.raises(pkg.InvalidParam):
        pkg.Bm25Session.from_csc(indptr, indices, data, 4)


@pytest.mark.parametrize('case', ['tf', 'norm', 'idf'])
def test_invalid_lazy_index_rejected_before_device(pkg, case):
    """The reference's Index rules (index_data.h:18-40)."""
    offsets = np.array([0, 2, 3], dtype=np.int64)
    docs = np.array([0, 1, 2], dtype=np.int32)
    tf = np.ones(3, dtype=np.float32)
    norm = np.ones(4, dtype=np.float32)
    idf = np.ones(2, dtype=np.float32)
    if case == 'tf':
        tf[0] = 1.5
    elif case == 'norm':
        norm[3] = 0.0
    else:
        idf[1] = -1.0
    with pytest.raises(pkg.InvalidParam):
        pkg.Bm25Session.from_lazy(offsets, docs, tf, norm, idf)


def test_closed_handle_is_illegal_operation(pkg):
    lib = pkg._native.engine_library()
    assert lib.bm25_search(None, None, None, 1, 1, None, None) == pkg._native.BM25_ERR_ILLEGAL_OPERATION
    assert lib.bm25_close(None) == pkg._native.BM25_OK
