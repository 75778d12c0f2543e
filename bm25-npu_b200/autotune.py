"""Autotuners: pick the engine's speed knobs by timing device-resident Searches of a
sample batch on the caller's index and GPU.  A configuration changes speed, never
results: every one is checked bit for bit against the first.

tune() works on a live session (bm25_set_tuning: warp-tile claim sizes, tile-group ring
shape, candidate capacity, learned routing cut) without re-uploading the index; this is
what a server or the benchmark runs before it serves.  autotune() also chooses what is
fixed when a session is created (tile size): every configuration is a separate session
over the same index.

Each configuration is timed with CUDA events on its launching stream over `reps`
Searches after `warmup`, with the L2 flushed between Searches (a write of 256 MiB).
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


def _time(session, queries, k, reps, warmup, flush, learned=False, ks=None):
    """Median ms of a device Search of `queries` with K k, or (ks given: a K per query, k their
    largest) of a batch Search; returns (ms, scores, ids)."""
    import torch
    offsets, words = queries
    q = offsets.size - 1
    dev = flush.device
    d_off = torch.from_numpy(np.ascontiguousarray(offsets, dtype=np.int64)).to(dev)
    d_w = torch.from_numpy(np.ascontiguousarray(words if len(words) else np.zeros(1), dtype=np.int32)).to(dev)
    rows = q * k if ks is None else int(np.sum(ks))
    d_s = torch.empty(rows, dtype=torch.float32, device=dev)
    d_i = torch.empty(rows, dtype=torch.int32, device=dev)
    d_x = torch.empty(q, dtype=torch.int32, device=dev)
    if ks is not None:
        d_ks = torch.from_numpy(np.ascontiguousarray(ks, dtype=np.int32)).to(dev)
        kout = np.zeros(q, dtype=np.int64)
        np.cumsum(ks[:-1], out=kout[1:])
        d_kout = torch.from_numpy(kout).to(dev)
    stream = torch.cuda.Stream(dev)

    def one():
        if ks is not None:
            session.search_batch_device(d_off.data_ptr(), d_w.data_ptr(), d_ks.data_ptr(), d_kout.data_ptr(), q, k,
                                        d_s.data_ptr(), d_i.data_ptr(), d_x.data_ptr() if learned else None,
                                        learned=learned, stream_ptr=stream.cuda_stream)
        elif learned:
            session.search_learned_device(d_off.data_ptr(), d_w.data_ptr(), q, k, d_s.data_ptr(), d_i.data_ptr(),
                                          d_x.data_ptr(), stream.cuda_stream)
        else:
            session.search_device(d_off.data_ptr(), d_w.data_ptr(), q, k, d_s.data_ptr(), d_i.data_ptr(),
                                  stream.cuda_stream)

    ms = []
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            one()
        for _ in range(reps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            one()
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


def tuning_space(session, k, learned=False):
    """The runtime knobs that matter for this session's kernel and K (dict of value tuples)."""
    info = session.info()
    space = {}
    if info['kernel'] == 5:  # warp tile
        space['claim_tiles'] = (2, 4, 8)
        space['tail_claims'] = (1, 2, 4)
    if info['kernel'] in (4, 5):  # tile group (also the warp-tile sessions' K > 32 batches)
        space['ring_stages'] = (2, 3, 4)
        space['ring_chunk'] = (1024, 2048)
    if info['max_k'] > 32:
        space['candidate_cap'] = (0, max(2048, 8 * info['max_k'], 64 * k))
    if learned:
        space['prune_route'] = (0.3, 0.6, 1.0)
    return space


def tune(session, queries, k, *, space=None, learned=False, ks=None, reps=10, warmup=3, keep=True):
    """Times every combination of `space` (default tuning_space) on a live session with the sample
    batch `queries` (offsets, words) and K `k`, through search_device (search_learned_device when
    `learned`; search_batch_device when `ks` gives a K per query, k their largest); checks that every
    combination returns the first one's results bit for bit; sets the fastest on the session when
    `keep` (else restores the tuning it had).

    Returns (best tuning dict, table of (changes, median ms per Search))."""
    import torch
    if space is None:
        space = tuning_space(session, k, learned)
    keys = sorted(space)
    combos = [dict(zip(keys, values)) for values in itertools.product(*(space[key] for key in keys))] or [{}]
    start = session.tuning()
    flush = torch.empty(64 << 20, dtype=torch.float32, device=f'cuda:{torch.cuda.current_device()}')
    offsets, words = (np.asarray(queries[0], np.int64), np.asarray(queries[1], np.int32))
    table, ref = [], None
    done = False
    try:
        for changes in combos:
            try:
                session.set_tuning(**{**start, **changes})
            except InvalidParam:
                continue  # e.g. a ring too deep for one SM's shared memory
            ms, scores, ids = _time(session, (offsets, words), k, reps, warmup, flush, learned, ks)
            if ref is None:
                ref = (scores, ids)
            elif not (np.array_equal(ids, ref[1]) and np.array_equal(scores.view(np.uint32),
                                                                     ref[0].view(np.uint32))):
                raise RuntimeError(f'tuning {changes} changed the results')
            table.append((changes, ms))
        best = {**start, **min(table, key=lambda row: row[1])[0]} if table else start
        session.set_tuning(**(best if keep else start))
        done = True
    finally:
        if not done:  # a failed run leaves the session as it found it (when it is still usable)
            try:
                session.set_tuning(**start)
            except Exception:
                pass
    return best, table
