"""bm25s native retrieve, restated with numba -- TEST INFRASTRUCTURE / TIMED CPU BASELINE ONLY.

Only bench.py's CPU-baseline leg and tests/ use this module: it times the second CPU
baseline the reference reports beside its own C++ search, the bm25s library's native
numba retrieve (vendored in the reference at reference_only/bm25s_original, pinned
commit 03eac5a8).  The algorithm restated here is bm25s's query step:

  * per query (queries in parallel, numba prange, n_threads workers):
    scores = zeros(N) in FP32; for each query term in order, scores[indices[j]] +=
    data[j] over the term's CSC postings (bm25s/scoring.py:345-368,
    _compute_relevance_from_scores_jit_ready);
  * top-K by a size-K min-heap over all N scores, a score replacing the root when
    strictly larger, then the K kept sorted by score descending
    (bm25s/numba/selection.py:87-124, _numba_sorted_top_k; retrieve_utils.py:13-64).

Ties are not ranked by document id (bm25s's own contract; the reference runs a strict
adapter around it for parity, run_bm25s_reference.py:93-132): this module is a timed
baseline, and its scores equal the oracle's as a sorted list, not its ids under ties.
"""

import numpy as np

try:
    import numba
    from numba import njit, prange
except ImportError:  # the baseline is reported as unavailable without numba
    numba = None


def available():
    return numba is not None


if numba is not None:

    @njit(nogil=True, cache=False)
    def _sift_down(values, ids, length):
        # restore the min-heap from the root
        i = 0
        while True:
            l_ = 2 * i + 1
            r_ = l_ + 1
            m = i
            if l_ < length and values[l_] < values[m]:
                m = l_
            if r_ < length and values[r_] < values[m]:
                m = r_
            if m == i:
                return
            values[i], values[m] = values[m], values[i]
            ids[i], ids[m] = ids[m], ids[i]
            i = m

    @njit(nogil=True, cache=False)
    def _push(values, ids, length, v, d):
        # insert at the end and move up while smaller than the parent
        i = length
        values[i] = v
        ids[i] = d
        while i > 0:
            p = (i - 1) // 2
            if values[i] < values[p]:
                values[i], values[p] = values[p], values[i]
                ids[i], ids[p] = ids[p], ids[i]
                i = p
            else:
                return

    @njit(parallel=True, cache=False)
    def _retrieve(indptr, indices, data, num_docs, qoffsets, words, k, out_scores, out_ids):
        nq = qoffsets.size - 1
        for q in prange(nq):
            scores = np.zeros(num_docs, dtype=np.float32)
            for w in range(qoffsets[q], qoffsets[q + 1]):
                t = words[w]
                if t < 0 or t >= indptr.size - 1:
                    continue
                for j in range(indptr[t], indptr[t + 1]):
                    scores[indices[j]] += data[j]
            values = np.zeros(k, dtype=np.float32)
            ids = np.zeros(k, dtype=np.int32)
            length = 0
            for d in range(num_docs):
                v = scores[d]
                if length < k:
                    _push(values, ids, length, v, d)
                    length += 1
                elif v > values[0]:
                    values[0] = v
                    ids[0] = d
                    _sift_down(values, ids, length)
            order = np.argsort(values)[::-1]
            for r in range(k):
                out_scores[q, r] = values[order[r]]
                out_ids[q, r] = ids[order[r]]


def retrieve(indptr, indices, data, num_docs, qoffsets, words, k, n_threads):
    """Top-K (scores, ids) [Q][K] of every query, bm25s's way, on n_threads numba threads."""
    if numba is None:
        raise RuntimeError('numba is not installed')
    numba.set_num_threads(int(n_threads))
    q = np.asarray(qoffsets).size - 1
    out_s = np.zeros((q, k), np.float32)
    out_i = np.zeros((q, k), np.int32)
    _retrieve(np.asarray(indptr, np.int64), np.asarray(indices, np.int32), np.asarray(data, np.float32),
              int(num_docs), np.asarray(qoffsets, np.int64), np.asarray(words, np.int32), int(k), out_s, out_i)
    return out_s, out_i


def max_threads():
    return numba.config.NUMBA_NUM_THREADS if numba is not None else 0
