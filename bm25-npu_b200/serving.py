"""Continuous-batching server (csrc/serve.cpp) from Python.

Server wraps bm25_server_*: submit single queries from any thread, wait on
tickets.  serve_poisson runs the library's open-loop Poisson load generator and
returns every query's latency.
"""

import ctypes
from ctypes import c_double, c_float, c_int32, c_int64, c_uint64

import numpy as np

from . import _native as n
from .search import _ERRORS, Bm25Error


def _server_error(status):
    buf = ctypes.create_string_buffer(512)
    n.engine_library().bm25_server_last_error(buf, len(buf))
    return _ERRORS.get(status, Bm25Error)(status, buf.value.decode())


def server_options(max_batch=256, learned=False, max_wait_us=0, candidate_budget=0):
    o = n.ServerOptions()
    n.engine_library().bm25_default_server_options(ctypes.byref(o))
    o.max_batch = max_batch
    o.learned = int(bool(learned))
    o.max_wait_us = max_wait_us
    o.candidate_budget = candidate_budget
    return o


class Server:
    """A serving loop over one session (which must outlive it)."""

    def __init__(self, session, **options):
        self._lib = n.engine_library()
        self._o = server_options(**options)
        self._h = ctypes.c_void_p()
        status = self._lib.bm25_server_create(session._handle, ctypes.byref(self._o), ctypes.byref(self._h))
        if status != n.BM25_OK:
            raise _server_error(status)

    def submit(self, words, k):
        w = np.ascontiguousarray(words, dtype=np.int32)
        ticket = c_uint64(0)
        status = self._lib.bm25_server_submit(self._h, n.ptr(w, c_int32) if w.size else None, w.size, k,
                                              ctypes.byref(ticket))
        if status != n.BM25_OK:
            raise _server_error(status)
        return ticket.value, k

    def wait(self, ticket):
        t, k = ticket
        scores = np.empty(k, dtype=np.float32)
        ids = np.empty(k, dtype=np.int32)
        exact = c_int32(1)
        lat = c_double(0)
        status = self._lib.bm25_server_wait(self._h, c_uint64(t), n.ptr(scores, c_float), n.ptr(ids, c_int32),
                                            ctypes.byref(exact), ctypes.byref(lat))
        if status != n.BM25_OK:
            raise _server_error(status)
        return scores, ids, exact.value, lat.value

    def stats(self):
        b, s = c_int64(0), c_int64(0)
        self._lib.bm25_server_stats(self._h, ctypes.byref(b), ctypes.byref(s))
        return {'batches': b.value, 'served': s.value}

    def close(self):
        if self._h:
            self._lib.bm25_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def serve_poisson(session, qoffsets, words, ks, rate_qps, total, seed=1, **options):
    """Open-loop Poisson arrivals at rate_qps over a query pool; returns (latency_us [total], stats)."""
    lib = n.engine_library()
    o = server_options(**options)
    qoffsets = np.ascontiguousarray(qoffsets, dtype=np.int64)
    words = np.ascontiguousarray(words if len(words) else np.zeros(1), dtype=np.int32)
    ks = np.ascontiguousarray(ks, dtype=np.int32)
    lat = np.zeros(total, dtype=np.float64)
    elapsed = c_double(0)
    batches = c_int64(0)
    status = lib.bm25_serve_poisson(session._handle, ctypes.byref(o), n.ptr(qoffsets, c_int64), n.ptr(words, c_int32),
                                    n.ptr(ks, c_int32), ks.size, c_double(rate_qps), total, c_uint64(seed),
                                    lat.ctypes.data_as(ctypes.POINTER(c_double)), ctypes.byref(elapsed),
                                    ctypes.byref(batches))
    if status != n.BM25_OK:
        raise _server_error(status)
    return lat, {'elapsed_s': elapsed.value, 'batches': batches.value, 'achieved_qps': total / elapsed.value,
                 'p50_us': float(np.percentile(lat, 50)), 'p95_us': float(np.percentile(lat, 95)),
                 'p99_us': float(np.percentile(lat, 99)), 'mean_batch': total / max(1, batches.value)}
