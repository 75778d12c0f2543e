"""Document-sharded Search: shard slicing, the gather step and the exact merge.

CPU: shard_csc slices every list exactly; ShardedSession itself runs on two
gloo ranks (each rank's local search is the oracle over its shard), all-gathers
the local lists and merges them with the host rank merge, and equals the
unsharded oracle; the host merge rejects a broken list as the kernel does.  GPU: bm25_merge_topk over shards searched by
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


def _oracle_local(indptr, indices, data, num_docs, offsets, words, k):
    """The local search handed to ShardedSession on CPU ranks: the oracle over the rank's shard."""
    from oracle import oracle
    return oracle.search(indptr, indices, data, num_docs, offsets, words, k)


def _gloo_rank(rank, world, port, index, data, queries, ks, out):
    import torch.distributed as dist
    from importlib import import_module
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    from datetime import timedelta
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=timedelta(seconds=60))
    sh = import_module('bm25-npu_b200.sharded')
    session = sh.ShardedSession(index.offsets, index.docs, data, index.num_docs, local_search=_oracle_local,
                                device='cpu')
    assert (session.lo, session.hi) == sh.shard_range(index.num_docs, rank, world)
    out[rank] = [session.search(queries, k) for k in ks]
    session.close()
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_session_on_gloo_ranks_equals_unsharded(pkg, oracle_mod, corpus):
    """ShardedSession itself on 2 gloo ranks (the CPU oracle as each rank's local search): shard slicing,
    the all-gather and the host rank merge give the unsharded oracle's top-K on both ranks, K in {10, 100},
    including queries with fewer than K positive documents (zero fill from the smallest global ids across
    shards), empty queries and unknown words."""
    index, data = corpus
    df = np.diff(index.offsets)
    rare = [int(t) for t in np.nonzero((df > 0) & (df < 4))[0][:3]]
    rows = mixed_queries(index.vocab, np.random.default_rng(2), 12, 0, 6, oov=True) + [rare[:1], rare, []]
    offsets, words = pack(rows)
    ks = (10, 100)
    ctx = mp.get_context('spawn')
    with ctx.Manager() as m:
        out = m.dict()
        port = 29500 + os.getpid() % 1000
        procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, index, data, (offsets, words), ks, out))
                 for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
        assert all(p.exitcode == 0 for p in procs)
        for j, k in enumerate(ks):
            want = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words, k)
            for r in range(2):
                assert_same_topk(*out[r][j], *want, f'rank {r} k={k}')


def test_host_merge_matches_restatement_and_rejects_bad_lists(pkg, oracle_mod, corpus):
    """merge_topk_host (the host rank merge) equals a sort of all lists, and an out-of-order list turns its
    query's row to -1 while the other queries stay exact (the merge operator's contract)."""
    sh = pkg.sharded
    index, data = corpus
    offsets, words = pack(mixed_queries(index.vocab, np.random.default_rng(5), 8, 0, 6, oov=True) + [[]])
    k, shards = 10, 3
    loc_s, loc_i, bases = [], [], []
    for r in range(shards):
        lo, hi = sh.shard_range(index.num_docs, r, shards)
        ls, li = oracle_mod.search(*sh.shard_csc(index.offsets, index.docs, data, lo, hi), offsets, words, k)
        loc_s.append(ls)
        loc_i.append(li)
        bases.append(lo)
    ss, ii = np.stack(loc_s), np.stack(loc_i)
    got = sh.merge_topk_host(ss, ii, bases, index.num_docs)
    assert_same_topk(*got, *merge_restated(ss, ii, bases, k), 'host merge vs restatement')
    assert_same_topk(*got, *oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words, k),
                     'host merge vs unsharded')
    bad = ss.copy()
    bad[1, 2, 0], bad[1, 2, 1] = bad[1, 2, 1], bad[1, 2, 0] + 1.0  # order broken in shard 1, query 2
    bs, bi = sh.merge_topk_host(bad, ii, bases, index.num_docs)
    assert np.all(bs[2] == -1.0) and np.all(bi[2] == -1)
    keep = [q for q in range(ss.shape[1]) if q != 2]
    assert_same_topk(bs[keep], bi[keep], got[0][keep], got[1][keep], 'untouched rows')


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
        # the host rank merge gives the kernel's result
        assert_same_topk(*sh.merge_topk_host(np.stack(loc_s), np.stack(loc_i), bases, index.num_docs), *want,
                         f'host merge k={k}')
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


def _nccl_single_rank(port, index, data, offsets, words, k, out):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from importlib import import_module
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group('nccl', rank=0, world_size=1, timeout=timedelta(seconds=60),
                            device_id=torch.device('cuda', 0))
    sh = import_module('bm25-npu_b200.sharded')
    session = sh.ShardedSession(index.offsets, index.docs, data, index.num_docs, query_capacity=32,
                                word_capacity=256, max_k=100)
    host = session.search((offsets, words), k)
    d_o = torch.from_numpy(offsets).cuda()
    d_w = torch.from_numpy(words).cuda()
    # an empty batch between the real ones: each result must be its own batch's, on the legacy
    # default stream (the caller's current stream here), with no synchronisation in between
    e_o = torch.zeros(offsets.size, dtype=torch.int64, device='cuda')
    e_w = torch.zeros(1, dtype=torch.int32, device='cuda')
    results = []
    for _ in range(3):
        gs, gi = session.search_device(d_o, d_w, offsets.size - 1, k)
        results.append((gs.clone(), gi.clone()))
        session.search_device(e_o, e_w, offsets.size - 1, k)
    torch.cuda.synchronize()
    out['host'] = host
    out['device'] = [(a.cpu().numpy(), b.cpu().numpy()) for a, b in results]
    session.close()
    dist.destroy_process_group()


@pytest.mark.gpu
def test_sharded_session_on_the_gpu(pkg, oracle_mod, corpus, cuda_ok):
    """ShardedSession with the engine as local search, NCCL and the merge kernel (one rank on the one GPU
    here): search and search_device equal the unsharded oracle."""
    index, data = corpus
    offsets, words = pack(mixed_queries(index.vocab, np.random.default_rng(4), 10, 0, 6, oov=True) + [[]])
    k = 10
    want = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words, k)
    ctx = mp.get_context('spawn')
    with ctx.Manager() as m:
        out = m.dict()
        p = ctx.Process(target=_nccl_single_rank, args=(29700 + os.getpid() % 200, index, data, offsets, words, k,
                                                        out))
        p.start()
        p.join(300)
        assert p.exitcode == 0
        assert_same_topk(*out['host'], *want, 'search')
        for r, got in enumerate(out['device']):
            assert_same_topk(*got, *want, f'search_device {r}')
