"""Document-sharded Search: one process per GPU, each holding a document range.

Rank r of W holds documents [N*r/W, N*(r+1)/W) as its own CSC with local ids
(the same terms, each list cut to the range).  A Search runs in two steps:

  1. local search: this rank's top-K lists over its own documents (the engine on
     this rank's GPU, or any search handed in with the same contract);
  2. gather and merge: the W local lists are all-gathered (torch.distributed:
     NCCL for CUDA tensors, gloo for CPU tensors; Q*K*8 bytes per rank, the
     only data-path exchange) and merged exactly on every rank -- by the
     bm25_merge_topk kernel on the GPU (csrc/merge_kernel.cuh), or by
     merge_topk_host, the same rank merge on the host.

Exactness follows from disjoint ranges: a document in the global top-K is in its
shard's top-K, and zero-score fills come from each shard's smallest ids, so the
merged fill takes the smallest global ids (the reference's
topk_document_shards.h:4 argument).  Remote lists reach this rank through the
collective's own buffers; no kernel reads another GPU's memory.
"""

import ctypes
from ctypes import c_void_p

import numpy as np

from . import _native as n
from .search import Bm25Session, InnerError, pack_queries


def shard_range(num_docs, rank, world):
    """Document range [lo, hi) of rank `rank` among `world` shards."""
    return num_docs * rank // world, num_docs * (rank + 1) // world


def shard_csc(indptr, indices, data, lo, hi):
    """CSC of the documents [lo, hi) with local ids (doc - lo); every term keeps its row."""
    indptr = np.asarray(indptr, dtype=np.int64)
    indices = np.asarray(indices, dtype=np.int32)
    keep = (indices >= lo) & (indices < hi)
    csum = np.zeros(indices.size + 1, dtype=np.int64)
    np.cumsum(keep, out=csum[1:])
    new_indptr = csum[indptr]
    return new_indptr, (indices[keep] - lo).astype(np.int32), np.asarray(data, dtype=np.float32)[keep], hi - lo


def merge_topk_device(scores, ids, bases, q, shards, k, num_docs, out_scores, out_ids, shard_major=False,
                      stream=None):
    """bm25_merge_topk on torch CUDA tensors (data_ptr()s); asynchronous on `stream`."""
    lib = n.engine_library()
    status = lib.bm25_merge_topk(c_void_p(scores), c_void_p(ids), c_void_p(bases), q, shards, k, num_docs,
                                 int(bool(shard_major)), c_void_p(out_scores), c_void_p(out_ids), c_void_p(stream))
    if status != n.BM25_OK:
        buf = ctypes.create_string_buffer(512)
        lib.bm25_last_error(None, buf, len(buf), None)
        raise InnerError(status, buf.value.decode())


def merge_topk_host(scores, ids, bases, num_docs):
    """The rank merge of bm25_merge_topk on host arrays: scores/ids [S][Q][K] (an all-gather's layout,
    local ids), bases [S] (or None: global ids) -> global [Q][K].  An entry's output rank is its
    position in its own list plus, in every other list, the number of entries ranked before it (score
    desc, id asc); a query with a list that is not a valid strict ranking (negative or non-finite score,
    id outside [0, num_docs), order broken) gets a row of -1, as the kernel and the reference's merge
    operator (bm25_top_k_merge.cpp:10-86) give."""
    scores = np.asarray(scores, dtype=np.float32)
    ids = np.asarray(ids, dtype=np.int64)
    s_, q_, k = scores.shape
    gid = ids + (np.asarray(bases, dtype=np.int64)[:, None, None] if bases is not None else 0)
    out_s = np.full((q_, k), -1.0, np.float32)
    out_i = np.full((q_, k), -1, np.int32)
    for q in range(q_):
        sc, gi, li = scores[:, q, :], gid[:, q, :], ids[:, q, :]
        ok = np.all(np.isfinite(sc) & (sc >= 0) & (li >= 0) & (gi >= 0) & (gi < num_docs))
        if ok and k > 1:
            prev_s, prev_i, cur_s, cur_i = sc[:, :-1], gi[:, :-1], sc[:, 1:], gi[:, 1:]
            ok = bool(np.all((prev_s > cur_s) | ((prev_s == cur_s) & (prev_i < cur_i))))
        if not ok:
            continue
        for s in range(s_):
            for r in range(k):
                rank = r
                for o in range(s_):
                    if o == s or rank >= k:
                        continue
                    # entries of list o ranked before (sc, id): a binary search of a sorted list
                    lo, hi = 0, k
                    while lo < hi:
                        mid = (lo + hi) // 2
                        if sc[o, mid] > sc[s, r] or (sc[o, mid] == sc[s, r] and gi[o, mid] < gi[s, r]):
                            lo = mid + 1
                        else:
                            hi = mid
                    rank += lo
                if rank < k:
                    out_s[q, rank] = sc[s, r]
                    out_i[q, rank] = gi[s, r]
    return out_s, out_i


class ShardedSession:
    """This rank's shard of a document-sharded index; search() returns the global top-K on every rank.

    local_search: None runs the engine on this rank's GPU (a Bm25Session over the shard, made with
    session_kwargs).  Otherwise a callable (indptr, indices, data, num_docs, offsets, words, k) ->
    (scores [Q][K], ids [Q][K]) over this rank's shard with local ids, under the engine's contract
    (score desc, id asc, zero fill by id): e.g. the CPU oracle in tests.  device: where the gather and
    the merge run -- a CUDA device (NCCL and the merge kernel) or 'cpu' (gloo and merge_topk_host)."""

    def __init__(self, indptr, indices, data, num_docs, *, group=None, device=None, local_search=None,
                 **session_kwargs):
        import torch
        import torch.distributed as dist
        self._dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.num_docs = int(num_docs)
        self.lo, self.hi = shard_range(self.num_docs, self.rank, self.world)
        if device is None:
            device = torch.device('cuda', torch.cuda.current_device()) if local_search is None else 'cpu'
        self.device = torch.device(device)
        self._shard = shard_csc(indptr, indices, data, self.lo, self.hi)
        self._local_search = local_search
        self.session = None
        if local_search is None:
            self.session = Bm25Session.from_csc(*self._shard, device_id=self.device.index or 0, **session_kwargs)
        self._bases_host = np.array([shard_range(self.num_docs, r, self.world)[0] for r in range(self.world)],
                                    dtype=np.int32)
        self.bases = torch.from_numpy(self._bases_host).to(self.device)
        self._bufs = {}  # gather and output buffers per (q, k), reused across Searches
        # device Searches run on a stream of their own, fenced against the caller's current stream on
        # both sides (the caller's may be the legacy default stream, whose handle the engine would read
        # as "the session's own stream")
        self._stream = torch.cuda.Stream(self.device) if self.device.type == 'cuda' else None

    def local(self, queries, k):
        """This rank's top-K over its own documents (local ids), host arrays."""
        offsets, words = queries if isinstance(queries, tuple) else pack_queries(queries)
        if self._local_search is not None:
            return self._local_search(*self._shard, np.asarray(offsets, np.int64), np.asarray(words, np.int32), k)
        return self.session.search((offsets, words), k)

    def _buffers(self, q, k):
        import torch
        key = (q, k)
        if key not in self._bufs:
            dev = self.device
            self._bufs[key] = (torch.empty((self.world, q, k), dtype=torch.float32, device=dev),
                               torch.empty((self.world, q, k), dtype=torch.int32, device=dev),
                               torch.empty((q, k), dtype=torch.float32, device=dev),
                               torch.empty((q, k), dtype=torch.int32, device=dev))
        return self._bufs[key]

    def gather_merge(self, local_scores, local_ids):
        """All-gathers every rank's local lists ([Q][K] tensors on self.device, local ids) and merges them:
        the global (scores, ids) [Q][K] tensors, the same on every rank."""
        import torch
        q, k = local_scores.shape
        gs, gi, out_s, out_i = self._buffers(q, k)
        if self.device.type == 'cuda':
            self._dist.all_gather_into_tensor(gs, local_scores.contiguous(), group=self.group)
            self._dist.all_gather_into_tensor(gi, local_ids.contiguous(), group=self.group)
            stream = torch.cuda.current_stream(self.device).cuda_stream
            merge_topk_device(gs.data_ptr(), gi.data_ptr(), self.bases.data_ptr(), q, self.world, k, self.num_docs,
                              out_s.data_ptr(), out_i.data_ptr(), shard_major=True, stream=stream)
            return out_s, out_i
        self._dist.all_gather(list(gs.unbind(0)), local_scores.contiguous(), group=self.group)
        self._dist.all_gather(list(gi.unbind(0)), local_ids.contiguous(), group=self.group)
        ms, mi = merge_topk_host(gs.numpy(), gi.numpy(), self._bases_host, self.num_docs)
        out_s.copy_(torch.from_numpy(ms))
        out_i.copy_(torch.from_numpy(mi))
        return out_s, out_i

    def search(self, queries, k):
        """Host queries -> the global top-K (numpy scores, ids [Q][K]) on every rank."""
        import torch
        ls, li = self.local(queries, k)
        out_s, out_i = self.gather_merge(torch.from_numpy(np.ascontiguousarray(ls)).to(self.device),
                                         torch.from_numpy(np.ascontiguousarray(li)).to(self.device))
        return out_s.cpu().numpy(), out_i.cpu().numpy()

    def search_device(self, d_offsets, d_words, q, k, learned=False):
        """Device query batch (torch int64 offsets, int32 words) -> global (scores, ids) [q, k] tensors (this
        session's buffers, valid until its next Search of the same shape), ordered after the caller's
        current stream's prior work and before its later work; no allocation per call."""
        import torch
        if self.session is None:
            raise InnerError(n.BM25_ERR_ILLEGAL_OPERATION, 'search_device needs the engine as local search')
        dev = self.device
        key = ('local', q, k)
        if key not in self._bufs:
            self._bufs[key] = (torch.empty((q, k), dtype=torch.float32, device=dev),
                               torch.empty((q, k), dtype=torch.int32, device=dev),
                               torch.empty(q, dtype=torch.int32, device=dev))
        ls, li, ex = self._bufs[key]
        caller = torch.cuda.current_stream(dev)
        self._stream.wait_stream(caller)  # the query batch is ready
        with torch.cuda.stream(self._stream):
            stream = self._stream.cuda_stream
            if learned:
                self.session.search_learned_device(d_offsets.data_ptr(), d_words.data_ptr(), q, k, ls.data_ptr(),
                                                   li.data_ptr(), ex.data_ptr(), stream)
            else:
                self.session.search_device(d_offsets.data_ptr(), d_words.data_ptr(), q, k, ls.data_ptr(),
                                           li.data_ptr(), stream)
            out = self.gather_merge(ls, li)
        caller.wait_stream(self._stream)  # the caller sees the merged lists
        return out

    def close(self):
        if self.session is not None:
            self.session.close()
