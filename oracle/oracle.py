"""CPU oracle bindings -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs
import this module, and only as the checker or the timed CPU baseline; the
product library never loads it.

  liboracle.so          plain-C restatement of the reference CPU search (bm25_oracle.c)
  _ref/libref_cpu.so    the reference's own CpuSearchSession compiled from its sources
                        (oracle/Makefile, target `ref`); present only where it was built
"""

import ctypes
import os
import subprocess
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_int64, c_size_t, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / 'liboracle.so'
REF_SO = HERE / '_ref' / 'libref_cpu.so'
REF_TEST = HERE / '_ref' / 'cpu_index_search_tests'
# where the reference's sources are read from when its CPU search is compiled (override: REFERENCE_ROOT)
REFERENCE_ROOT = Path(os.environ.get('REFERENCE_ROOT', '/root/reference'))


def build(with_reference=None):
    """make -C oracle [ref]; the reference part only where its sources exist."""
    subprocess.run(['make', '-s', '-C', str(HERE), 'all'], check=True)
    if with_reference is None:
        with_reference = REFERENCE_ROOT.exists()
    if with_reference:
        subprocess.run(['make', '-s', '-C', str(HERE), 'ref', f'REF_ROOT={REFERENCE_ROOT}'], check=True)


def _p(a, t):
    return a.ctypes.data_as(POINTER(t))


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            build(with_reference=False)
        L = ctypes.CDLL(str(ORACLE_SO))
        L.oracle_contributions.restype = c_int
        L.oracle_contributions.argtypes = [POINTER(c_int64), c_int64, POINTER(c_int32), POINTER(c_float),
                                           POINTER(c_float), c_int64, POINTER(c_float), c_float, POINTER(c_float)]
        L.oracle_search.restype = c_int
        L.oracle_search.argtypes = [POINTER(c_int64), c_int64, POINTER(c_int32), POINTER(c_float), POINTER(c_float),
                                    POINTER(c_float), POINTER(c_float), c_float, c_int64, POINTER(c_int64),
                                    POINTER(c_int32), c_int64, c_int64, POINTER(c_float), POINTER(c_int32),
                                    POINTER(c_float), c_int]
        L.oracle_merge.restype = c_int
        L.oracle_merge.argtypes = [POINTER(c_float), POINTER(c_int32), c_int64, c_int64, POINTER(c_float),
                                   POINTER(c_int32)]
        L.oracle_max_threads.restype = c_int
        _lib = L
    return _lib


def k1p1(k1):
    """f32(k1 + 1) with the sum in double: k1 = 1.2 gives the reference's 2.2F literal."""
    return float(np.float32(np.float64(k1) + 1.0))


def contributions(index, k1):
    """Eager FP32 posting scores of a lazy index (reference formula, cpu_index_search.h:185-186)."""
    data = np.empty(index.docs.size, dtype=np.float32)
    rc = lib().oracle_contributions(_p(index.offsets, c_int64), index.idf.size, _p(index.docs, c_int32),
                                    _p(index.tf, c_float), _p(index.norm, c_float), index.norm.size,
                                    _p(index.idf, c_float), k1p1(k1), _p(data, c_float))
    if rc:
        raise ValueError(f'oracle_contributions failed ({rc})')
    return data


def search(indptr, indices, data, num_docs, qoffsets, words, k, threads=0, full=False, lazy=None, k1=1.2):
    """Strict top-k (scores, ids) [Q, k]; data=None with lazy=(tf, norm, idf) uses the lazy formula."""
    indptr = np.ascontiguousarray(indptr, dtype=np.int64)
    indices = np.ascontiguousarray(indices, dtype=np.int32)
    qoffsets = np.ascontiguousarray(qoffsets, dtype=np.int64)
    words = np.ascontiguousarray(words if len(words) else np.zeros(1), dtype=np.int32)
    q = qoffsets.size - 1
    scores = np.empty((q, k), dtype=np.float32)
    ids = np.empty((q, k), dtype=np.int32)
    fullbuf = np.empty((q, num_docs), dtype=np.float32) if full else None
    null_f = ctypes.cast(None, POINTER(c_float))
    if data is not None:
        data = np.ascontiguousarray(data, dtype=np.float32)
        tf = norm = idf = None
    else:
        tf, norm, idf = (np.ascontiguousarray(x, dtype=np.float32) for x in lazy)
    rc = lib().oracle_search(
        _p(indptr, c_int64), indptr.size - 1, _p(indices, c_int32),
        _p(data, c_float) if data is not None else null_f,
        _p(tf, c_float) if tf is not None else null_f, _p(norm, c_float) if norm is not None else null_f,
        _p(idf, c_float) if idf is not None else null_f, k1p1(k1), int(num_docs), _p(qoffsets, c_int64),
        _p(words, c_int32), q, k, _p(scores, c_float), _p(ids, c_int32),
        _p(fullbuf, c_float) if full else null_f, threads)
    if rc:
        raise ValueError(f'oracle_search failed ({rc})')
    return (scores, ids, fullbuf) if full else (scores, ids)


def merge(scores, ids, k):
    """Exact merge of per-shard lists [S, k] (global ids, -1 = empty) into the strict top-k."""
    scores = np.ascontiguousarray(scores, dtype=np.float32)
    ids = np.ascontiguousarray(ids, dtype=np.int32)
    out_s = np.empty(k, dtype=np.float32)
    out_i = np.empty(k, dtype=np.int32)
    rc = lib().oracle_merge(_p(scores, c_float), _p(ids, c_int32), scores.size // k, k, _p(out_s, c_float),
                            _p(out_i, c_int32))
    if rc:
        raise ValueError('oracle_merge failed')
    return out_s, out_i


def max_threads():
    return lib().oracle_max_threads()


# --- the reference's own CPU search (oracle/_ref) ---------------------------------

_ref = None


def reference_available():
    return REF_SO.exists()


def ref_lib():
    global _ref
    if _ref is None:
        L = ctypes.CDLL(str(REF_SO))
        L.ref_session_create.restype = c_void_p
        L.ref_session_create.argtypes = [POINTER(c_int64), c_int64, POINTER(c_int32), POINTER(c_float), c_int64,
                                         POINTER(c_float), c_int64, POINTER(c_float), c_int, c_int64, c_int64, c_int64,
                                         c_int64, c_int, c_char_p, c_size_t]
        L.ref_session_search.restype = c_int
        L.ref_session_search.argtypes = [c_void_p, POINTER(c_int64), POINTER(c_int32), c_int64, POINTER(c_float),
                                         POINTER(c_int32), POINTER(c_double), c_char_p, c_size_t]
        L.ref_session_debug_scores.restype = c_int
        L.ref_session_debug_scores.argtypes = [c_void_p, c_int64, POINTER(c_float), c_int64]
        L.ref_session_threads.restype = c_int
        L.ref_session_threads.argtypes = [c_void_p]
        L.ref_session_destroy.restype = None
        L.ref_session_destroy.argtypes = [c_void_p]
        _ref = L
    return _ref


class ReferenceCpuSession:
    """bm25cpu::CpuSearchSession (mode 0) or DirectoryCpuSearchSession (mode 1), unmodified."""

    def __init__(self, index, k, threads, shards=None, query_capacity=8, word_capacity=24, mode=0):
        L = ref_lib()
        self._keep = [np.ascontiguousarray(x) for x in (index.offsets, index.docs, index.tf, index.norm, index.idf)]
        offsets, docs, tf, norm, idf = self._keep
        err = ctypes.create_string_buffer(1024)
        self.k = k
        self.num_docs = norm.size
        self._h = L.ref_session_create(_p(offsets, c_int64), idf.size, _p(docs, c_int32), _p(tf, c_float),
                                       docs.size, _p(norm, c_float), norm.size, _p(idf, c_float), threads, k,
                                       shards or threads, query_capacity, word_capacity, mode, err, len(err))
        if not self._h:
            raise ValueError('reference session: ' + err.value.decode())
        self.threads = L.ref_session_threads(self._h)

    def search(self, qoffsets, words):
        L = ref_lib()
        qoffsets = np.ascontiguousarray(qoffsets, dtype=np.int64)
        words = np.ascontiguousarray(words if len(words) else np.zeros(1), dtype=np.int32)
        q = qoffsets.size - 1
        scores = np.empty((q, self.k), dtype=np.float32)
        ids = np.empty((q, self.k), dtype=np.int32)
        ms = c_double(0)
        err = ctypes.create_string_buffer(1024)
        rc = L.ref_session_search(self._h, _p(qoffsets, c_int64), _p(words, c_int32), q, _p(scores, c_float),
                                  _p(ids, c_int32), ctypes.byref(ms), err, len(err))
        if rc:
            raise ValueError('reference search: ' + err.value.decode())
        return scores, ids, ms.value

    def debug_scores(self, q):
        out = np.empty((q, self.num_docs), dtype=np.float32)
        if ref_lib().ref_session_debug_scores(self._h, q, _p(out, c_float), self.num_docs):
            raise ValueError('reference debug scores failed')
        return out

    def close(self):
        if self._h:
            ref_lib().ref_session_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
