"""Autotuner for the tile-group engine: picks tile size, ring stage size and ring depth
(and, for K > 32, the candidate capacity) by timing device-resident Searches of a sample
batch on the caller's index and GPU.

Every configuration is a separate session over the same index (the index is uploaded
once per configuration); each is timed with CUDA events on its launching stream over
`reps` Searches after `warmup`, with the L2 flushed between Searches, and its results are
checked bit for bit against the first configuration's -- a configuration changes speed,
never results.
"""

import itertools

import numpy as np

from .search import Bm25Session, InvalidParam

DEFAULT_SPACE = {
    'tile_docs': (1024, 2048),
    'ring_chunk': (1024, 1536, 2048),
    'ring_stages': (2, 3, 4),
}


def candidates(space=None, max_k=10):
    """Every combination of the search space (dicts of session options)."""
    space = dict(DEFAULT_SPACE if space is None else space)
    if max_k > 32 and 'candidate_capacity' not in space:
        space['candidate_capacity'] = (0, 64 * max_k)
    keys = sorted(space)
    return [dict(zip(keys, values)) for values in itertools.product(*(space[k] for k in keys))]


def _time(session, queries, k, reps, warmup, flush):
    import torch
    offsets, words = queries
    q = offsets.size - 1
    dev = torch.device('cuda', torch.cuda.current_device())
    d_off = torch.from_numpy(np.ascontiguousarray(offsets, dtype=np.int64)).to(dev)
    d_w = torch.from_numpy(np.ascontiguousarray(words if len(words) else np.zeros(1), dtype=np.int32)).to(dev)
    d_s = torch.empty((q, k), dtype=torch.float32, device=dev)
    d_i = torch.empty((q, k), dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(dev)
    ms = []
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            session.search_device(d_off.data_ptr(), d_w.data_ptr(), q, k, d_s.data_ptr(), d_i.data_ptr(),
                                  stream.cuda_stream)
        for _ in range(reps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            session.search_device(d_off.data_ptr(), d_w.data_ptr(), q, k, d_s.data_ptr(), d_i.data_ptr(),
                                  stream.cuda_stream)
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
    if session.device_status():
        raise RuntimeError('device status set while tuning')
    return float(np.median(ms)), d_s.cpu().numpy(), d_i.cpu().numpy()


def autotune(indptr, indices, data, num_docs, queries, k, *, space=None, reps=20, warmup=3, device_id=0,
             **session_kwargs):
    """Times every configuration of `space` on the sample batch `queries` (offsets, words) with K `k`.

    Returns (best options dict, table of (options, median ms per Search)).  Extra keyword
    arguments (query_capacity, word_capacity, max_k, ...) are passed to every session."""
    import torch
    torch.cuda.set_device(device_id)
    offsets, words = queries
    q = np.asarray(offsets).size - 1
    session_kwargs.setdefault('query_capacity', q)
    session_kwargs.setdefault('word_capacity', max(1, int(np.asarray(offsets)[-1])))
    session_kwargs.setdefault('max_k', k)
    flush = torch.empty(64 << 20, dtype=torch.float32, device=f'cuda:{device_id}')  # 256 MiB > L2
    table, ref = [], None
    for opts in candidates(space, session_kwargs['max_k']):
        try:
            with Bm25Session.from_csc(indptr, indices, data, num_docs, device_id=device_id, kernel=4,
                                      **session_kwargs, **opts) as s:
                ms, scores, ids = _time(s, (offsets, words), k, reps, warmup, flush)
        except InvalidParam:
            continue  # a combination the engine refuses (e.g. a ring too deep for one SM)
        if ref is None:
            ref = (scores, ids)
        elif not (np.array_equal(ids, ref[1]) and np.array_equal(scores.view(np.uint32), ref[0].view(np.uint32))):
            raise RuntimeError(f'configuration {opts} changed the results')
        table.append((opts, ms))
    if not table:
        raise InvalidParam(0, 'no configuration of the search space could be created')
    best = min(table, key=lambda row: row[1])[0]
    return best, table
