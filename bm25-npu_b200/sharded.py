"""Document-sharded Search: one process per GPU, each holding a document range.

Rank r of W holds documents [N*r/W, N*(r+1)/W) as its own CSC with local ids
(the same terms, each list cut to the range).  A Search runs the plain (or
learned) engine on every rank, all-gathers the W local top-K lists
(torch.distributed: NCCL on GPUs, gloo on CPU for the host-side tests) and merges
them exactly on every rank with bm25_merge_topk (csrc/merge_kernel.cuh).
Exactness follows from disjoint ranges: a document in the global top-K is in its
shard's top-K, and zero-score fills come from each shard's smallest ids, so the
merged fill takes the smallest global ids (the reference's
topk_document_shards.h:4 argument).
"""

import ctypes
from ctypes import c_void_p

import numpy as np

from . import _native as n
from .search import Bm25Session, InnerError, _raise


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


class ShardedSession:
    """This rank's shard of a document-sharded index; search() returns the global top-K on every rank."""

    def __init__(self, indptr, indices, data, num_docs, *, group=None, device=None, **session_kwargs):
        import torch
        import torch.distributed as dist
        self._dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.num_docs = int(num_docs)
        self.lo, self.hi = shard_range(self.num_docs, self.rank, self.world)
        self.device = device if device is not None else torch.device('cuda', torch.cuda.current_device())
        sub = shard_csc(indptr, indices, data, self.lo, self.hi)
        self.session = Bm25Session.from_csc(*sub, device_id=self.device.index or 0, **session_kwargs)
        self.bases = torch.tensor([shard_range(self.num_docs, r, self.world)[0] for r in range(self.world)],
                                  dtype=torch.int32, device=self.device)

    def search_device(self, d_offsets, d_words, q, k, learned=False):
        """Device query batch (torch int64 offsets, int32 words) -> global (scores, ids) [q, k] tensors."""
        import torch
        dev = self.device
        ls = torch.empty((q, k), dtype=torch.float32, device=dev)
        li = torch.empty((q, k), dtype=torch.int32, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        if learned:
            ex = torch.empty(q, dtype=torch.int32, device=dev)
            self.session.search_learned_device(d_offsets.data_ptr(), d_words.data_ptr(), q, k, ls.data_ptr(),
                                               li.data_ptr(), ex.data_ptr(), stream)
        else:
            self.session.search_device(d_offsets.data_ptr(), d_words.data_ptr(), q, k, ls.data_ptr(),
                                       li.data_ptr(), stream)
        gs = torch.empty((self.world, q, k), dtype=torch.float32, device=dev)
        gi = torch.empty((self.world, q, k), dtype=torch.int32, device=dev)
        self._dist.all_gather_into_tensor(gs, ls, group=self.group)
        self._dist.all_gather_into_tensor(gi, li, group=self.group)
        out_s = torch.empty((q, k), dtype=torch.float32, device=dev)
        out_i = torch.empty((q, k), dtype=torch.int32, device=dev)
        merge_topk_device(gs.data_ptr(), gi.data_ptr(), self.bases.data_ptr(), q, self.world, k, self.num_docs,
                          out_s.data_ptr(), out_i.data_ptr(), shard_major=True, stream=stream)
        return out_s, out_i

    def close(self):
        self.session.close()
