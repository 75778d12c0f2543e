"""Document-sharded Search: shard slicing, the gather step and the exact merge.

CPU: shard_csc slices every list exactly; two gloo ranks each search their shard
with the oracle and all-gather their local lists, and the restated rank merge of
the gathered lists equals the unsharded oracle (the exchange and merge logic of
ShardedSession without a GPU).  GPU: bm25_merge_topk over shards searched by
the engine equals the unsharded oracle, in both input layouts, and an invalid
list makes its query's row -1 (the reference's merge contract).
"""

import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from helpers import assert_same_topk, mixed_queries, pack


def merge_restated(scores, ids, bases, k):
    """numpy restatement of the rank merge: [S][Q][K] local lists -> [Q][K] global."""
    s_, q_, _ = scores.shape
    out_s = np.empty((q_, k), np.float32)
    out_i = np.empty((q_, k), np.int32)
    for q in range(q_):
        cand = [(float(scores[s, q, r]), int(ids[s, q, r]) + int(bases[s])) for s in range(s_) for r in range(k)]
        cand.sort(key=lambda c: (-c[0], c[1]))
        out_s[q] = [c[0] for c in cand[:k]]
        out_i[q] = [c[1] for c in cand[:k]]
    return out_s, out_i


@pytest.fixture(scope='module')
def corpus(pkg, oracle_mod):
    spec = pkg.CorpusSpec(docs=30_000, vocab=3_000, seed=9, k1=1.2)
    index = pkg.synthetic_index(spec)
    return index, oracle_mod.contributions(index, spec.k1)


def test_shard_csc_slices_every_list(pkg, corpus):
    sh = pkg.sharded
    index, data = corpus
    parts = [sh.shard_csc(index.offsets, index.docs, data, *sh.shard_range(index.num_docs, r, 3)) for r in range(3)]
    assert sum(p[3] for p in parts) == index.num_docs
    for t in (0, 7, 100, index.vocab - 1):
        whole = index.docs[index.offsets[t]:index.offsets[t + 1]]
        got = np.concatenate([p[1][p[0][t]:p[0][t + 1]] + sh.shard_range(index.num_docs, r, 3)[0]
                              for r, p in enumerate(parts)])
        assert np.array_equal(got, whole)
    assert all(p[0][-1] == p[1].size == p[2].size for p in parts)


def _gloo_rank(rank, world, port, index, data, offsets, words, k, out):
    import torch
    import torch.distributed as dist
    from importlib import import_module
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    from oracle import oracle
    sh = import_module('bm25-npu_b200.sharded')
    lo, hi = sh.shard_range(index.num_docs, rank, world)
    ip, ix, dt, nd = sh.shard_csc(index.offsets, index.docs, data, lo, hi)
    ls, li = oracle.search(ip, ix, dt, nd, offsets, words, k)
    gs = [torch.empty(ls.shape, dtype=torch.float32) for _ in range(world)]
    gi = [torch.empty(li.shape, dtype=torch.int32) for _ in range(world)]
    dist.all_gather(gs, torch.from_numpy(ls))
    dist.all_gather(gi, torch.from_numpy(li))
    bases = [sh.shard_range(index.num_docs, r, world)[0] for r in range(world)]
    ms, mi = merge_restated(np.stack([g.numpy() for g in gs]), np.stack([g.numpy() for g in gi]), bases, k)
    out[rank] = (ms, mi)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_gather_and_merge_exactly(pkg, oracle_mod, corpus):
    index, data = corpus
    offsets, words = pack(mixed_queries(index.vocab, np.random.default_rng(2), 12, 0, 6, oov=True))
    k = 10
    want = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words, k)
    ctx = mp.get_context('spawn')
    with ctx.Manager() as m:
        out = m.dict()
        port = 29500 + os.getpid() % 1000
        procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, index, data, offsets, words, k, out))
                 for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        for r in range(2):
            assert_same_topk(*out[r], *want, f'rank {r}')


@pytest.mark.gpu
@pytest.mark.parametrize('shards', [2, 3])
def test_device_merge_equals_unsharded(pkg, oracle_mod, corpus, cuda_ok, shards):
    import torch
    sh = pkg.sharded
    index, data = corpus
    offsets, words = pack(mixed_queries(index.vocab, np.random.default_rng(shards), 20, 0, 8, oov=True) + [[]])
    q = offsets.size - 1
    dev = torch.device('cuda:0')
    for k in (10, 100):
        want = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words, k)
        loc_s, loc_i, bases = [], [], []
        for r in range(shards):
            lo, hi = sh.shard_range(index.num_docs, r, shards)
            with pkg.Bm25Session.from_csc(*sh.shard_csc(index.offsets, index.docs, data, lo, hi), query_capacity=32,
                                          word_capacity=256, max_k=100) as s:
                ls, li = s.search((offsets, words), k)
            loc_s.append(ls)
            loc_i.append(li)
            bases.append(lo)
        d_b = torch.tensor(bases, dtype=torch.int32, device=dev)
        for major in (True, False):
            ss = np.stack(loc_s) if major else np.stack(loc_s, axis=1)
            ii = np.stack(loc_i) if major else np.stack(loc_i, axis=1)
            d_s = torch.from_numpy(np.ascontiguousarray(ss)).to(dev)
            d_i = torch.from_numpy(np.ascontiguousarray(ii)).to(dev)
            o_s = torch.empty((q, k), dtype=torch.float32, device=dev)
            o_i = torch.empty((q, k), dtype=torch.int32, device=dev)
            sh.merge_topk_device(d_s.data_ptr(), d_i.data_ptr(), d_b.data_ptr(), q, shards, k, index.num_docs,
                                 o_s.data_ptr(), o_i.data_ptr(), shard_major=major)
            torch.cuda.synchronize()
            assert_same_topk(o_s.cpu().numpy(), o_i.cpu().numpy(), *want, f'k={k} shards={shards} major={major}')
        # an out-of-order list: that query's row becomes -1, the others stay exact
        bad = np.stack(loc_s).copy()
        bad[0, 1, [0, 1]] = bad[0, 1, [1, 0]] if bad[0, 1, 0] != bad[0, 1, 1] else [-1.0, bad[0, 1, 1]]
        d_s = torch.from_numpy(bad).to(dev)
        d_i = torch.from_numpy(np.stack(loc_i)).to(dev)
        sh.merge_topk_device(d_s.data_ptr(), d_i.data_ptr(), d_b.data_ptr(), q, shards, k, index.num_docs,
                             o_s.data_ptr(), o_i.data_ptr(), shard_major=True)
        torch.cuda.synchronize()
        got_s, got_i = o_s.cpu().numpy(), o_i.cpu().numpy()
        assert np.all(got_s[1] == -1.0) and np.all(got_i[1] == -1)
        assert_same_topk(got_s[[0, 2]], got_i[[0, 2]], want[0][[0, 2]], want[1][[0, 2]], 'untouched rows')
