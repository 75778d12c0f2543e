"""Python mirror of the engine's Search session (C ABI in include/bm25_b200.h).

``Bm25Session`` corresponds to the reference's ``bm25large::Session``
(feature_retrieval/src/ascendfaiss/ascendhost/src/bm25/large_search.h:35-86) and
``AscendIndexBm25`` to the SDK facade
(feature_retrieval/src/ascendfaiss/ascendhost/include/index/AscendIndexBm25.h:37-57):
same method names, argument meaning and error behaviour (input errors leave the
session usable, device errors poison it, Close is idempotent).
"""

import ctypes
from ctypes import c_float, c_int32, c_int64, c_void_p

import numpy as np

from . import _native as n


class Bm25Error(RuntimeError):
    """Raised for a non-OK status; ``status`` is the C ABI code, ``code`` the CUDA error (or 0)."""

    def __init__(self, status, message, code=0):
        super().__init__(message)
        self.status = status
        self.code = code


class InvalidParam(Bm25Error, ValueError):
    pass


class IllegalOperation(Bm25Error):
    pass


class InnerError(Bm25Error):
    pass


_ERRORS = {
    n.BM25_ERR_INVALID_PARAM: InvalidParam,
    n.BM25_ERR_ILLEGAL_OPERATION: IllegalOperation,
    n.BM25_ERR_INNER_ERROR: InnerError,
}


def _last_error(lib, handle):
    buf = ctypes.create_string_buffer(1024)
    code = c_int64(0)
    lib.bm25_last_error(handle, buf, len(buf), ctypes.byref(code))
    return buf.value.decode('utf-8', 'replace'), code.value


def _raise(lib, status, handle):
    if status == n.BM25_OK:
        return
    message, code = _last_error(lib, handle)
    raise _ERRORS.get(status, Bm25Error)(status, message or f'BM25 status {status}', code)


def _outputs(q, k, out):
    """(scores [q, k] f32, ids [q, k] i32, exact [q] i32): new arrays, or `out` checked."""
    if out is None:
        return np.empty((q, k), dtype=np.float32), np.empty((q, k), dtype=np.int32), np.empty(q, dtype=np.int32)
    scores, ids, exact = out
    for a, dt, size in ((scores, np.float32, q * k), (ids, np.int32, q * k), (exact, np.int32, q)):
        if not (a.flags.c_contiguous and a.dtype == dt and a.size >= size):
            raise InvalidParam(n.BM25_ERR_INVALID_PARAM, 'out must be C-contiguous float32/int32 arrays of q*k, q*k, q')
    return scores, ids, exact


def pack_queries(queries):
    """List of word-id lists -> (offsets int64 [Q+1], words int32), common/bm25/search_inputs.h:23-42."""
    offsets = np.zeros(len(queries) + 1, dtype=np.int64)
    for i, row in enumerate(queries):
        offsets[i + 1] = offsets[i] + len(row)
    words = np.fromiter((w for row in queries for w in row), dtype=np.int64, count=int(offsets[-1]))
    if words.size and (words.min() < 0 or words.max() >= 2**31 - 1):
        raise InvalidParam(n.BM25_ERR_INVALID_PARAM, 'Invalid public word ID')
    return offsets, words.astype(np.int32)


def _options(query_capacity, word_capacity, max_k, device_id, tile_docs, merge_fan_in, directory_bytes, stream,
             kernel=5, ring_stages=0, ring_chunk=0, prune=False, candidate_capacity=0, prune_route=0.0,
             wait_budget_cycles=0, dense_density=0.0):
    o = n.Options()
    n.engine_library().bm25_default_options(ctypes.byref(o))
    o.device_id = device_id
    o.max_k = max_k
    o.query_capacity = query_capacity
    o.word_capacity = word_capacity
    o.tile_docs = tile_docs
    o.merge_fan_in = merge_fan_in
    o.directory_bytes = directory_bytes
    o.stream = stream
    o.kernel = kernel
    o.ring_stages = ring_stages
    o.ring_chunk = ring_chunk
    o.prune = int(bool(prune))
    o.candidate_capacity = candidate_capacity
    o.prune_route = prune_route
    o.wait_budget_cycles = wait_budget_cycles
    o.dense_density = dense_density
    return o


class Bm25Session:
    """A resident index on one GPU plus its fixed-capacity Search plan."""

    def __init__(self, handle, num_docs, max_k):
        self._lib = n.engine_library()
        self._call = n.hostcall()
        self._handle = handle
        self._handle_int = (handle.value if isinstance(handle, c_void_p) else handle) or 0
        self.num_docs = num_docs
        self.max_k = max_k

    @classmethod
    def from_csc(cls, indptr, indices, data, num_docs, *, query_capacity=8, word_capacity=24, max_k=10,
                 device_id=0, tile_docs=0, merge_fan_in=0, directory_bytes=0, stream=None, kernel=5, ring_stages=0,
                 ring_chunk=0, prune=False, candidate_capacity=0, prune_route=0.0, wait_budget_cycles=0,
                 dense_density=0.0):
        """Eager CSC index (bm25s layout): indptr int64 [V+1], indices int32 [M], data float32 [M]."""
        lib = n.engine_library()
        indptr = np.ascontiguousarray(indptr, dtype=np.int64)
        indices = np.ascontiguousarray(indices, dtype=np.int32)
        data = np.ascontiguousarray(data, dtype=np.float32)
        vocab = indptr.size - 1
        if vocab < 1 or indices.size != indptr[-1] or data.size != indices.size:
            raise InvalidParam(n.BM25_ERR_INVALID_PARAM, 'Index dimensions/endpoints differ')
        o = _options(query_capacity, word_capacity, max_k, device_id, tile_docs, merge_fan_in, directory_bytes,
                     stream, kernel, ring_stages, ring_chunk, prune, candidate_capacity, prune_route,
                     wait_budget_cycles, dense_density)
        h = c_void_p()
        status = lib.bm25_create(n.ptr(indptr, c_int64), n.ptr(indices, c_int32), n.ptr(data, c_float), vocab,
                                 int(num_docs), ctypes.byref(o), ctypes.byref(h))
        _raise(lib, status, None)
        return cls(h, int(num_docs), max_k)

    @classmethod
    def from_lazy(cls, term_offsets, posting_doc_ids, posting_tf, doc_norm, idf, *, k1=1.2, query_capacity=8,
                  word_capacity=24, max_k=10, device_id=0, tile_docs=0, merge_fan_in=0, directory_bytes=0,
                  stream=None, kernel=5, ring_stages=0, ring_chunk=0, prune=False, candidate_capacity=0,
                  prune_route=0.0, wait_budget_cycles=0, dense_density=0.0):
        """The reference's resident index (common/bm25/index_data.h:9-42); posting scores built on the GPU."""
        lib = n.engine_library()
        offsets = np.ascontiguousarray(term_offsets, dtype=np.int64)
        docs = np.ascontiguousarray(posting_doc_ids, dtype=np.int32)
        tf = np.ascontiguousarray(posting_tf, dtype=np.float32)
        norm = np.ascontiguousarray(doc_norm, dtype=np.float32)
        idf = np.ascontiguousarray(idf, dtype=np.float32)
        vocab = idf.size
        if offsets.size != vocab + 1 or docs.size != tf.size or offsets[-1] != docs.size:
            raise InvalidParam(n.BM25_ERR_INVALID_PARAM, 'Index dimensions/endpoints differ')
        o = _options(query_capacity, word_capacity, max_k, device_id, tile_docs, merge_fan_in, directory_bytes,
                     stream, kernel, ring_stages, ring_chunk, prune, candidate_capacity, prune_route,
                     wait_budget_cycles, dense_density)
        h = c_void_p()
        status = lib.bm25_create_lazy(n.ptr(offsets, c_int64), n.ptr(docs, c_int32), n.ptr(tf, c_float),
                                      n.ptr(norm, c_float), n.ptr(idf, c_float), vocab, norm.size, float(k1),
                                      ctypes.byref(o), ctypes.byref(h))
        _raise(lib, status, None)
        return cls(h, norm.size, max_k)

    def search(self, queries, k, *, out=None):
        """Top-k per query; queries = list of word lists or (offsets, words).  Returns (scores, ids) [Q, k]."""
        if isinstance(queries, tuple):
            offsets, words = queries
            offsets = np.ascontiguousarray(offsets, dtype=np.int64)
            words = np.ascontiguousarray(words, dtype=np.int32)
        else:
            offsets, words = pack_queries(queries)
        q = offsets.size - 1
        if out is None:
            scores = np.empty((q, k), dtype=np.float32)
            ids = np.empty((q, k), dtype=np.int32)
        else:
            scores, ids = out
        if words.size == 0:
            words = np.zeros(1, dtype=np.int32)
        try:  # type and length checks of the arrays, then bm25_search with the GIL released
            status = self._call.search(self._handle_int, offsets, words, q, k, scores, ids)
        except ValueError as e:
            raise InvalidParam(n.BM25_ERR_INVALID_PARAM, str(e)) from None
        if status:
            _raise(self._lib, status, self._handle)
        return scores, ids

    def search_pruned(self, queries, k, tau):
        """Exact top-k with tile pruning from starting bounds tau [Q] (a guess of each query's k-th score).

        Returns (scores, ids, exact): exact[i] is 1 where the pruned pass stood and 0 where the
        guess was too high and the call's retry pass searched the query on the plain path."""
        if isinstance(queries, tuple):
            offsets = np.ascontiguousarray(queries[0], dtype=np.int64)
            words = np.ascontiguousarray(queries[1], dtype=np.int32)
        else:
            offsets, words = pack_queries(queries)
        q = offsets.size - 1
        tau = np.ascontiguousarray(tau, dtype=np.float32)
        if tau.shape != (q,):
            raise InvalidParam(n.BM25_ERR_INVALID_PARAM, 'tau must hold one bound per query')
        scores, ids, exact = _outputs(q, k, None)
        if words.size == 0:
            words = np.zeros(1, dtype=np.int32)
        status = self._lib.bm25_search_pruned(self._handle, offsets.ctypes.data, words.ctypes.data, tau.ctypes.data,
                                              q, k, scores.ctypes.data, ids.ctypes.data, exact.ctypes.data)
        if status:
            _raise(self._lib, status, self._handle)
        return scores, ids, exact

    def search_pruned_device(self, qoffsets_ptr, words_ptr, tau_ptr, q, k, scores_ptr, ids_ptr, exact_ptr,
                             stream_ptr=None):
        """Device-resident pruned Search; every row exact, exact[i] = 0 where the retry pass answered."""
        status = self._lib.bm25_search_pruned_device(self._handle, c_void_p(qoffsets_ptr), c_void_p(words_ptr),
                                                     c_void_p(tau_ptr), q, k, c_void_p(scores_ptr),
                                                     c_void_p(ids_ptr), c_void_p(exact_ptr), c_void_p(stream_ptr))
        _raise(self._lib, status, self._handle)

    def search_batch(self, queries, ks, *, learned=False):
        """A batch with a K per query (one graph replay).  Returns (scores, ids, koff[, exact]):
        query i's results are scores[koff[i]:koff[i + 1]] and ids[...] (packed rows); exact is
        returned when learned is set (learned bounds, as search_learned)."""
        if isinstance(queries, tuple):
            offsets = np.ascontiguousarray(queries[0], dtype=np.int64)
            words = np.ascontiguousarray(queries[1], dtype=np.int32)
        else:
            offsets, words = pack_queries(queries)
        q = offsets.size - 1
        ks = np.ascontiguousarray(ks, dtype=np.int32)
        if ks.shape != (q,):
            raise InvalidParam(n.BM25_ERR_INVALID_PARAM, 'ks must hold one K per query')
        koff = np.zeros(q + 1, dtype=np.int64)
        np.cumsum(ks, out=koff[1:])
        scores = np.empty(int(koff[-1]), dtype=np.float32)
        ids = np.empty(int(koff[-1]), dtype=np.int32)
        if words.size == 0:
            words = np.zeros(1, dtype=np.int32)
        if learned:
            exact = np.empty(q, dtype=np.int32)
            status = self._lib.bm25_search_batch_learned(self._handle, offsets.ctypes.data, words.ctypes.data,
                                                         ks.ctypes.data, q, scores.ctypes.data, ids.ctypes.data,
                                                         exact.ctypes.data)
            if status:
                _raise(self._lib, status, self._handle)
            return scores, ids, koff, exact
        status = self._lib.bm25_search_batch(self._handle, offsets.ctypes.data, words.ctypes.data, ks.ctypes.data,
                                             q, scores.ctypes.data, ids.ctypes.data)
        if status:
            _raise(self._lib, status, self._handle)
        return scores, ids, koff

    def search_batch_device(self, qoffsets_ptr, words_ptr, ks_ptr, kout_ptr, q, kmax, scores_ptr, ids_ptr,
                            exact_ptr=None, learned=False, stream_ptr=None):
        """Device-resident batch with a K per query (see bm25_search_batch_device); asynchronous."""
        status = self._lib.bm25_search_batch_device(self._handle, c_void_p(qoffsets_ptr), c_void_p(words_ptr),
                                                    c_void_p(ks_ptr), c_void_p(kout_ptr), q, kmax, int(bool(learned)),
                                                    c_void_p(scores_ptr), c_void_p(ids_ptr), c_void_p(exact_ptr),
                                                    c_void_p(stream_ptr))
        _raise(self._lib, status, self._handle)

    def set_threshold_model(self, model):
        """Threshold model of the learned bounds (a ThresholdModel, or None for the safe bounds alone)."""
        if model is None:
            status = self._lib.bm25_set_threshold_model(self._handle, None, c_float(0.0))
        else:
            params = np.ascontiguousarray(model.params, dtype=np.float32)
            status = self._lib.bm25_set_threshold_model(self._handle, n.ptr(params, c_float), c_float(model.margin))
        _raise(self._lib, status, self._handle)

    def search_learned(self, queries, k, *, out=None):
        """Exact top-k with learned starting bounds; returns (scores, ids, exact) as search_pruned.
        out: optional (scores, ids, exact) arrays to write (C-contiguous, q*k, q*k and q)."""
        if isinstance(queries, tuple):
            offsets = np.ascontiguousarray(queries[0], dtype=np.int64)
            words = np.ascontiguousarray(queries[1], dtype=np.int32)
        else:
            offsets, words = pack_queries(queries)
        q = offsets.size - 1
        scores, ids, exact = _outputs(q, k, out)
        if words.size == 0:
            words = np.zeros(1, dtype=np.int32)
        try:
            status = self._call.search_learned(self._handle_int, offsets, words, q, k, scores, ids, exact)
        except ValueError as e:
            raise InvalidParam(n.BM25_ERR_INVALID_PARAM, str(e)) from None
        if status:
            _raise(self._lib, status, self._handle)
        return scores, ids, exact

    def search_learned_device(self, qoffsets_ptr, words_ptr, q, k, scores_ptr, ids_ptr, exact_ptr, stream_ptr=None):
        """Device-resident learned pruned Search (rows as search_pruned_device)."""
        status = self._lib.bm25_search_learned_device(self._handle, c_void_p(qoffsets_ptr), c_void_p(words_ptr), q,
                                                      k, c_void_p(scores_ptr), c_void_p(ids_ptr),
                                                      c_void_p(exact_ptr), c_void_p(stream_ptr))
        _raise(self._lib, status, self._handle)

    def query_features_device(self, qoffsets_ptr, words_ptr, q, k, features_ptr, safe_ptr=None, stream_ptr=None):
        """Features [q][32] and safe bounds [q] of a device query batch (asynchronous)."""
        status = self._lib.bm25_query_features_device(self._handle, c_void_p(qoffsets_ptr), c_void_p(words_ptr), q,
                                                      k, c_void_p(features_ptr), c_void_p(safe_ptr),
                                                      c_void_p(stream_ptr))
        _raise(self._lib, status, self._handle)

    def search_stats(self, reset=True):
        """Search counters since the last reset (tile-group kernel: claims, tiles scanned, postings
        copied; block-max pruned pass: tiles scored, blocks kept, postings read)."""
        out = (ctypes.c_uint64 * 7)()
        _raise(self._lib, self._lib.bm25_search_stats(self._handle, out, int(bool(reset))), self._handle)
        names = ('claims', 'tiles_scanned', 'postings_copied', 'block_tiles', 'blocks_kept', 'postings_read',
                 'queries_streamed')
        return dict(zip(names, out))

    def search_device(self, qoffsets_ptr, words_ptr, q, k, scores_ptr, ids_ptr, stream_ptr=None):
        """Device-resident Search on raw device pointers (e.g. torch ``data_ptr()``); asynchronous."""
        status = self._lib.bm25_search_device(self._handle, c_void_p(qoffsets_ptr), c_void_p(words_ptr), q, k,
                                              c_void_p(scores_ptr), c_void_p(ids_ptr), c_void_p(stream_ptr))
        _raise(self._lib, status, self._handle)

    def prepare_batch_graphs(self, max_batch, learned=False):
        """Instantiates the graphs search_batch replays for batches of up to max_batch queries
        (bm25_prepare_batch_graphs); a server does this when it is created."""
        _raise(self._lib, self._lib.bm25_prepare_batch_graphs(self._handle, int(max_batch), int(bool(learned))),
               self._handle)

    def tuning(self):
        """The session's runtime tuning (bm25_get_tuning) as a dict."""
        t = n.Tuning()
        _raise(self._lib, self._lib.bm25_get_tuning(self._handle, ctypes.byref(t)), self._handle)
        return {name: getattr(t, name) for name, _ in n.Tuning._fields_ if name != 'reserved'}

    def set_tuning(self, **changes):
        """Changes some runtime tuning fields (bm25_set_tuning): speed only, never results; the
        session's instantiated graphs are dropped."""
        t = self.tuning()
        unknown = set(changes) - set(t)
        if unknown:
            raise InvalidParam(n.BM25_ERR_INVALID_PARAM, f'unknown tuning fields {sorted(unknown)}')
        t.update(changes)
        _raise(self._lib, self._lib.bm25_set_tuning(self._handle, ctypes.byref(n.Tuning(**t))), self._handle)

    def inject(self, what):
        """Test hook (bm25_test_inject): the next ``search`` fails as a device error, either on the host
        (BM25_INJECT_HOST_FAILURE) or by a stalled ring producer whose consumers' bounded waits run out
        (BM25_INJECT_STALL)."""
        _raise(self._lib, self._lib.bm25_test_inject(self._handle, int(what)), self._handle)

    def kernel_timing(self, enable=True):
        """Record CUDA events around the main search kernel of each ``search_device`` call."""
        _raise(self._lib, self._lib.bm25_kernel_timing(self._handle, int(bool(enable))), self._handle)

    def kernel_times(self, capacity=4096):
        """Durations (ms) of the main search kernel for the timed Searches since the last read."""
        ms = np.zeros(capacity, dtype=np.float32)
        count = c_int64(0)
        _raise(self._lib, self._lib.bm25_kernel_times(self._handle, n.ptr(ms, c_float), capacity,
                                                      ctypes.byref(count)), self._handle)
        return ms[:count.value].copy()

    def device_status(self):
        s = ctypes.c_uint32(0)
        _raise(self._lib, self._lib.bm25_device_status(self._handle, ctypes.byref(s)), self._handle)
        return s.value

    def info(self):
        i = n.Info()
        _raise(self._lib, self._lib.bm25_get_info(self._handle, ctypes.byref(i)), self._handle)
        return {name: getattr(i, name) for name, _ in n.Info._fields_}

    def last_error(self):
        return _last_error(self._lib, self._handle)

    def close(self):
        if self._handle:
            _raise(self._lib, self._lib.bm25_close(self._handle), self._handle)
            self._lib.bm25_destroy(self._handle)
            self._handle = None
            self._handle_int = 0  # a later call reaches the ABI with no handle: ILLEGAL_OPERATION

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            if self._handle:
                self._lib.bm25_destroy(self._handle)
                self._handle = None
        except Exception:
            pass


# --- SDK-shaped facade -------------------------------------------------------

APP_ERR_OK = 0
# IndexSDK's numeric APP_ERR values (common/ErrorCode.h) are not part of the
# reference tree; these local values are unpinned.
APP_ERR_INVALID_PARAM = 2001
APP_ERR_ILLEGAL_OPERATION = 2002
APP_ERR_INNER_ERROR = 2003
_APP = {n.BM25_ERR_INVALID_PARAM: APP_ERR_INVALID_PARAM, n.BM25_ERR_ILLEGAL_OPERATION: APP_ERR_ILLEGAL_OPERATION,
        n.BM25_ERR_INNER_ERROR: APP_ERR_INNER_ERROR}


class Bm25Config:
    """AscendIndexBm25.h:17-25 with the ACL context/resources replaced by an optional CUDA stream."""

    def __init__(self, deviceId=0, queryCount=8, maxQueryWords=24, topK=10, k1=1.2, stream=None):
        self.deviceId = deviceId
        self.queryCount = queryCount
        self.maxQueryWords = maxQueryWords
        self.topK = topK
        self.k1 = k1
        self.stream = stream


class Bm25SearchResult:
    def __init__(self):
        self.scores = []
        self.labels = []


class AscendIndexBm25:
    """Init/Search/Close/GetLastError returning APP_ERR codes (AscendIndexBm25.cpp:33-84)."""

    def __init__(self):
        self._session = None
        self._config = None
        self._error = ('', 0)

    def _invoke(self, fn):
        self._error = ('', 0)
        try:
            fn()
            return APP_ERR_OK
        except Bm25Error as e:
            self._error = (str(e), e.code)
            return _APP.get(e.status, APP_ERR_INNER_ERROR)
        except (ValueError, TypeError) as e:
            self._error = (str(e), 0)
            return APP_ERR_INVALID_PARAM

    def Init(self, index, config):
        """index: object with offsets, docs, tf, norm, idf (the reference's lazy Index)."""

        def run():
            if self._session is not None:
                raise IllegalOperation(n.BM25_ERR_ILLEGAL_OPERATION, 'BM25 is already initialized; Close before Init')
            self._session = Bm25Session.from_lazy(
                index.offsets, index.docs, index.tf, index.norm, index.idf, k1=config.k1,
                query_capacity=config.queryCount, word_capacity=config.maxQueryWords, max_k=config.topK,
                device_id=config.deviceId, stream=config.stream)
            self._config = config

        return self._invoke(run)

    def Search(self, queries, result):
        """Output is replaced only on success; the batch must hold queryCount queries."""

        def run():
            if self._session is None:
                raise IllegalOperation(n.BM25_ERR_ILLEGAL_OPERATION, 'BM25 is not initialized')
            if len(queries) != self._config.queryCount:
                raise InvalidParam(n.BM25_ERR_INVALID_PARAM, 'Fixed session requires its declared query count')
            scores, ids = self._session.search(queries, self._config.topK)
            result.scores = scores.reshape(-1).tolist()
            result.labels = [int(x) for x in ids.reshape(-1)]

        return self._invoke(run)

    def Close(self):
        def run():
            if self._session is not None:
                self._session.close()
                self._session = None

        return self._invoke(run)

    def GetLastError(self):
        return self._error
