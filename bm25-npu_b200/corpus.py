"""Resident-index arrays: seeded synthetic corpora and the reference's on-disk index files.

``LazyIndex`` holds the reference's index layout (common/bm25/index_data.h:9-42,
files of standalone/resident_index.py:12-18).  ``synthetic_index`` builds one
with the native two-pass generator (csrc/synth.c, the counterpart of
standalone/large_corpus.py:95-297); ``read_index_dir`` / ``write_index_dir`` use
the reference's file names and little-endian dtypes.
"""

import ctypes
from ctypes import c_float, c_int32, c_int64
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _native as n

INDEX_FILES = {
    'term_offsets.bin': np.dtype('<i8'),
    'posting_doc_ids.bin': np.dtype('<i4'),
    'posting_tf.bin': np.dtype('<f4'),
    'doc_norm.bin': np.dtype('<f4'),
    'idf.bin': np.dtype('<f4'),
}


@dataclass
class LazyIndex:
    offsets: np.ndarray  # int64 [V+1]
    docs: np.ndarray     # int32 [M]
    tf: np.ndarray       # float32 [M]
    norm: np.ndarray     # float32 [N]
    idf: np.ndarray      # float32 [V]
    doc_len: np.ndarray = None  # int32 [N] (synthetic corpora only)

    @property
    def num_docs(self):
        return int(self.norm.size)

    @property
    def vocab(self):
        return int(self.idf.size)

    @property
    def postings(self):
        return int(self.docs.size)

    def df(self):
        return np.diff(self.offsets)


@dataclass
class CorpusSpec:
    """Seeded synthetic corpus shape: Zipf(s) token ranks (s = 0: uniform), lognormal lengths (mean,
    sigma), or uniform integer lengths in [mean - |sigma|, mean + |sigma|] when sigma < 0."""

    docs: int
    vocab: int
    zipf_s: float = 1.1
    len_mean: float = 60.0
    len_sigma: float = 0.5
    seed: int = 20261203
    k1: float = 1.5
    b: float = 0.75


# Workload shapes: 8192 docs / V 30k; 10M docs / V 1M; 8.8M passages / V 2.5M; 4.2M docs / V 1M; and
# the reference's own benchmark corpus shape (standalone/large_corpus.py:58-62: tokens uniform over
# 1024 terms, lengths uniform in 16..48, seed 20261014, its builder's k1 1.2 and b 0.75) at 10M docs.
CONFIG_SHAPES = {
    'synthetic_8192': CorpusSpec(docs=8192, vocab=30000),
    'synthetic_10m': CorpusSpec(docs=10_000_000, vocab=1_000_000),
    'passages_8p8m': CorpusSpec(docs=8_800_000, vocab=2_500_000, zipf_s=1.05, len_mean=56.0),
    'blockmax_4p2m': CorpusSpec(docs=4_200_000, vocab=1_000_000, len_mean=80.0),
    'reference_10m': CorpusSpec(docs=10_000_000, vocab=1024, zipf_s=0.0, len_mean=32.0, len_sigma=-16.0,
                                seed=20261014, k1=1.2, b=0.75),
}


def synthetic_index(spec, threads=0):
    """Builds the lazy index of a seeded synthetic corpus (deterministic for any thread count)."""
    lib = n.synth_library()
    h = lib.synth_create(spec.docs, spec.vocab, spec.zipf_s, spec.len_mean, spec.len_sigma, spec.seed, threads)
    if not h:
        raise ValueError('synthetic corpus: invalid shape or out of memory')
    try:
        m = lib.synth_postings(h)
        offsets = np.empty(spec.vocab + 1, dtype=np.int64)
        docs = np.empty(m, dtype=np.int32)
        tf = np.empty(m, dtype=np.float32)
        norm = np.empty(spec.docs, dtype=np.float32)
        idf = np.empty(spec.vocab, dtype=np.float32)
        doc_len = np.empty(spec.docs, dtype=np.int32)
        rc = lib.synth_fill(h, spec.k1, spec.b, n.ptr(offsets, c_int64), n.ptr(docs, c_int32), n.ptr(tf, c_float),
                            n.ptr(norm, c_float), n.ptr(idf, c_float), n.ptr(doc_len, c_int32))
        if rc != 0:
            raise MemoryError('synthetic corpus: pass 2 failed')
    finally:
        lib.synth_destroy(h)
    return LazyIndex(offsets, docs, tf, norm, idf, doc_len)


def synthetic_queries(offsets, count, lo, hi, seed, distinct=True):
    """Seeded query batch, terms drawn with probability df / M; returns (offsets int64, words int32)."""
    lib = n.synth_library()
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    qoff = np.empty(count + 1, dtype=np.int64)
    words = np.empty(max(1, count * hi), dtype=np.int32)
    w = lib.synth_queries(n.ptr(offsets, c_int64), offsets.size - 1, count, lo, hi, int(distinct), seed,
                          n.ptr(qoff, c_int64), n.ptr(words, c_int32))
    if w < 0:
        raise ValueError('synthetic queries: invalid arguments')
    return qoff, words[:w].copy()


def unpack_queries(qoffsets, words):
    return [words[qoffsets[i]:qoffsets[i + 1]].tolist() for i in range(qoffsets.size - 1)]


def read_index_dir(path):
    """Reads the reference's index directory (term_offsets.bin, posting_doc_ids.bin, posting_tf.bin, ...)."""
    path = Path(path)
    arrays = {name: np.fromfile(path / name, dtype=dt) for name, dt in INDEX_FILES.items()}
    return LazyIndex(arrays['term_offsets.bin'].astype(np.int64), arrays['posting_doc_ids.bin'].astype(np.int32),
                     arrays['posting_tf.bin'].astype(np.float32), arrays['doc_norm.bin'].astype(np.float32),
                     arrays['idf.bin'].astype(np.float32))


def write_index_dir(index, path):
    path = Path(path)
    path.mkdir(parents=True, exist_ok=True)
    for (name, dt), values in zip(INDEX_FILES.items(), (index.offsets, index.docs, index.tf, index.norm, index.idf)):
        np.ascontiguousarray(values, dtype=dt).tofile(path / name)


QUERY_FILES = {'query_offsets.bin': np.dtype('<i8'), 'query_term_ids.bin': np.dtype('<i4')}


def read_queries_dir(path):
    """The reference's packed query files (standalone/resident_index.py:19): (offsets int64, words int32)."""
    path = Path(path)
    offsets = np.fromfile(path / 'query_offsets.bin', dtype=QUERY_FILES['query_offsets.bin']).astype(np.int64)
    words = np.fromfile(path / 'query_term_ids.bin', dtype=QUERY_FILES['query_term_ids.bin']).astype(np.int32)
    if offsets.size < 2 or offsets[0] != 0 or offsets[-1] != words.size or (np.diff(offsets) < 0).any():
        raise ValueError('query offsets and word ids differ')
    return offsets, words


def write_queries_dir(offsets, words, path):
    path = Path(path)
    path.mkdir(parents=True, exist_ok=True)
    np.ascontiguousarray(offsets, dtype=QUERY_FILES['query_offsets.bin']).tofile(path / 'query_offsets.bin')
    np.ascontiguousarray(words, dtype=QUERY_FILES['query_term_ids.bin']).tofile(path / 'query_term_ids.bin')


BM25S_FILES = ('data.csc.index.npy', 'indices.csc.index.npy', 'indptr.csc.index.npy', 'params.index.json')


def read_bm25s_dir(path):
    """Eager CSC saved by bm25s ``BM25.save`` (reference_only/bm25s_original/bm25s/__init__.py:941-1040):
    returns (indptr int64, indices int32, data float32, num_docs) for ``Bm25Session.from_csc``."""
    import json
    path = Path(path)
    data = np.load(path / 'data.csc.index.npy', allow_pickle=False)
    indices = np.load(path / 'indices.csc.index.npy', allow_pickle=False)
    indptr = np.load(path / 'indptr.csc.index.npy', allow_pickle=False)
    num_docs = int(json.loads((path / 'params.index.json').read_text())['num_docs'])
    return indptr.astype(np.int64), indices.astype(np.int32), data.astype(np.float32), num_docs


def write_bm25s_dir(indptr, indices, data, num_docs, path, k1=1.5, b=0.75):
    """Writes the CSC part of the bm25s layout (arrays + params.index.json; no vocabulary)."""
    import json
    path = Path(path)
    path.mkdir(parents=True, exist_ok=True)
    np.save(path / 'data.csc.index.npy', np.ascontiguousarray(data, dtype=np.float32))
    np.save(path / 'indices.csc.index.npy', np.ascontiguousarray(indices, dtype=np.int32))
    np.save(path / 'indptr.csc.index.npy', np.ascontiguousarray(indptr, dtype=np.int64))
    (path / 'params.index.json').write_text(json.dumps({'k1': k1, 'b': b, 'method': 'lucene', 'num_docs': int(num_docs)},
                                                       indent=4))


def build_index(doc_offsets, tokens, vocab, k1=1.2, b=0.75, device_id=0):
    """The reference's lazy index from documents given as token ids, built on the GPU
    (bm25_build_index: key sort and run-length counts on the device, idf and norms in double
    on the host, as standalone/large_corpus.py:95-190 does in Python)."""
    lib = n.engine_library()
    doc_offsets = np.ascontiguousarray(doc_offsets, dtype=np.int64)
    tokens = np.ascontiguousarray(tokens, dtype=np.int32)
    num_docs = doc_offsets.size - 1
    cap = max(1, int(doc_offsets[-1]))
    offsets = np.empty(vocab + 1, dtype=np.int64)
    docs = np.empty(cap, dtype=np.int32)
    tf = np.empty(cap, dtype=np.float32)
    norm = np.empty(num_docs, dtype=np.float32)
    idf = np.empty(vocab, dtype=np.float32)
    m = ctypes.c_int64(0)
    status = lib.bm25_build_index(n.ptr(doc_offsets, c_int64), n.ptr(tokens, c_int32) if tokens.size else None,
                                  num_docs, vocab, ctypes.c_double(k1), ctypes.c_double(b), device_id,
                                  n.ptr(offsets, c_int64), n.ptr(docs, c_int32), n.ptr(tf, c_float),
                                  n.ptr(norm, c_float), n.ptr(idf, c_float), ctypes.byref(m))
    if status != n.BM25_OK:
        buf = ctypes.create_string_buffer(512)
        lib.bm25_build_last_error(buf, len(buf))
        raise ValueError(f'index build failed ({status}): {buf.value.decode()}')
    k = m.value
    return LazyIndex(offsets, docs[:k].copy(), tf[:k].copy(), norm, idf,
                     np.diff(doc_offsets).astype(np.int32))
