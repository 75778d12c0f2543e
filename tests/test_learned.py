"""Learned starting bounds: features, safe bounds, GPU training and what the trained network gains.

CPU: the margin search and the model file.  GPU: the device term statistics and
query features against a numpy restatement; Searches with the safe bounds alone
never fall back; a network trained on the GPU (the engine's own MLP kernels)
keeps fewer 128-document blocks and reads fewer postings than the safe bounds
alone on held-out queries, while every result stays bit-exact with the oracle.
"""

import numpy as np
import pytest

from helpers import assert_same_topk


@pytest.fixture(scope='module')
def learned(pkg):
    return pkg.learned


def test_margin_meets_target(learned):
    rng = np.random.default_rng(0)
    kth = rng.uniform(1, 20, 5000).astype(np.float32)
    pred = (np.log(kth) + rng.normal(0, 0.3, kth.size)).astype(np.float32)
    safe = (kth * rng.uniform(0.2, 0.9, kth.size)).astype(np.float32)
    for target in (0.01, 0.05, 0.2):
        m = learned.choose_margin(pred, safe, kth, target)
        assert learned.fallback_rate(pred, safe, kth, m) <= target
        assert learned.fallback_rate(pred, safe, kth, m - 0.01) > target - 1e-3
    tau = learned.bounds(pred, safe, 100.0)
    assert np.array_equal(tau, safe)  # a huge margin leaves the safe bounds
    assert np.all(learned.bounds(pred, -np.ones_like(safe), 0.0) == 0)  # fewer than K postings: no pruning


def test_model_file_round_trip(learned, tmp_path):
    m = learned.ThresholdModel(learned.init_params(3, 1.5), 0.75)
    m.save(tmp_path / 'model.npz')
    back = learned.ThresholdModel.load(tmp_path / 'model.npz')
    assert np.array_equal(back.params, m.params) and back.margin == np.float32(0.75)
    assert m.params.size == learned.param_count() == 6337
    assert m.params[-1] == np.float32(1.5)


def term_top(indptr, data, term, top=32):
    s, e = indptr[term], indptr[term + 1]
    v = np.sort(np.maximum(data[s:e], 0))[::-1][:top]
    return np.pad(v, (0, top - v.size)).astype(np.float32)


def features_restated(indptr, data, vocab, words, k):
    """numpy restatement of QueryFeatures (csrc/learned_kernels.cuh): features [32] and the safe bound."""
    lg = lambda x: np.log1p(np.float32(max(x, 0)))  # noqa: E731
    f = np.zeros(32, np.float64)
    terms = [w for w in words if 0 <= w < vocab]
    oov = len(words) - len(terms)
    stats = []
    kk = min(k, 32)
    postings = 0
    for w in terms:
        t = term_top(indptr, data, w)
        df = int(indptr[w + 1] - indptr[w])
        postings += df
        mean = float(np.mean(data[indptr[w]:indptr[w + 1]])) if df else 0.0
        stats.append((t[0], t[kk - 1], t[(kk - 1) // 2], mean, np.log1p(df)))
    order = sorted(range(len(terms)), key=lambda i: (-stats[i][0], i))[:4]
    for j, i in enumerate(order):
        mx, kth, _, mean, ldf = stats[i]
        f[4 * j:4 * j + 4] = [lg(mx), lg(kth), lg(mean), ldf / 16]
    if stats:
        s = np.array(stats, dtype=np.float64)
        f[16:28] = [len(terms) / 8, lg(s[:, 0].sum()), lg(s[:, 1].sum()), lg(s[:, 1].max()), lg(s[:, 3].sum()),
                    np.log(k) / 4, s[:, 4].sum() / 64, s[:, 4].min() / 16, lg(s[:, 2].max()), lg(s[:, 2].sum()),
                    oov / 8, 1]
        safe = float(s[:, 1].max()) if k <= 32 else 0.0
    else:
        f[16:28] = [0, 0, 0, 0, 0, np.log(k) / 4, 0, 0, 0, 0, oov / 8, 1]
        safe = 0.0
    return f, (-1.0 if postings < k else safe)


@pytest.fixture(scope='module')
def corpus(pkg, oracle_mod):
    spec = pkg.CorpusSpec(docs=1_000_000, vocab=100_000, seed=41, k1=1.2, len_mean=80.0)
    index = pkg.synthetic_index(spec)
    data = oracle_mod.contributions(index, spec.k1)
    return index, data


def _session(pkg, index, data, q, words):
    return pkg.Bm25Session.from_csc(index.offsets, index.docs, data, index.num_docs, query_capacity=q,
                                    word_capacity=words, max_k=32, prune=True)


@pytest.mark.gpu
def test_device_features_match_restatement(pkg, corpus, cuda_ok):
    import torch
    index, data = corpus
    qo, w = pkg.synthetic_queries(index.offsets, 64, 1, 12, 5)
    w = w.copy()
    w[::17] = index.vocab + 3  # out-of-vocabulary words are counted, not used
    dev = torch.device('cuda:0')
    with _session(pkg, index, data, 64, int(qo[-1])) as s:
        for k in (10, 32):
            d_f = torch.empty((64, 32), dtype=torch.float32, device=dev)
            d_safe = torch.empty(64, dtype=torch.float32, device=dev)
            d_qo, d_w = torch.from_numpy(qo).to(dev), torch.from_numpy(w).to(dev)
            s.query_features_device(d_qo.data_ptr(), d_w.data_ptr(), 64, k, d_f.data_ptr(), d_safe.data_ptr(),
                                    torch.cuda.current_stream(dev).cuda_stream)
            torch.cuda.synchronize()
            got_f, got_safe = d_f.cpu().numpy(), d_safe.cpu().numpy()
            for i in range(64):
                f, safe = features_restated(index.offsets, data, index.vocab, w[qo[i]:qo[i + 1]], k)
                np.testing.assert_allclose(got_f[i], f, rtol=2e-5, atol=2e-6, err_msg=f'query {i} k={k}')
                assert got_safe[i] == np.float32(safe)  # an exact posting score


@pytest.mark.gpu
def test_trained_network_prunes_more_than_safe_bounds(pkg, oracle_mod, corpus, cuda_ok, learned):
    index, data = corpus
    batch = 256
    with _session(pkg, index, data, 2048, 2048 * 10) as s:
        model = learned.fit(s, index.offsets, queries=40_000, ks=(10, 32), lo=2, hi=4, steps=2000, batch=2048,
                            target_fallback=0.03, gen_batch=2048)
        r = model.report
        assert r['last_loss'] < 0.25 * r['first_loss'], r
        assert r['val_fallback'] <= 0.03, r
        assert r['val_tau_share_of_kth'] > r['val_safe_share_of_kth'], r
        stats = {}
        for k in (10, 32):
            qo, w = pkg.synthetic_queries(index.offsets, batch, 2, 4, 1000 + k)
            want = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, qo, w, k)
            plain = s.search((qo, w), k)
            assert_same_topk(*plain, *want, f'plain k={k}')
            s.search_stats(reset=True)
            for label, m in (('safe', None), ('model', model)):
                s.set_threshold_model(m)
                s.search_stats(reset=True)
                got_s, got_i, exact = s.search_learned((qo, w), k)
                st = s.search_stats(reset=True)
                assert_same_topk(got_s, got_i, *want, f'{label} k={k}')
                if label == 'safe':
                    assert exact.all(), 'the safe bounds never fall back'
                stats[label, k] = (st, float(np.mean(exact == 0)))
            # the plain path reads every posting of every query word
            s.search((qo, w), k)
            stats['plain', k] = (s.search_stats(reset=True), 0.0)
        def postings(st):  # read block by block, or streamed (queries routed to the tile-group kernel)
            return st['postings_read'] + st['postings_copied']

        for k in (10, 32):
            plain, safe, net = stats['plain', k][0], stats['safe', k][0], stats['model', k][0]
            assert postings(safe) < 0.5 * plain['postings_copied'], (k, plain, safe)
            # the network's gain over the method without it: fewer blocks kept, and fewer postings
            # in all, the retry pass of the queries it sent back included (the warp-tile session reads
            # each word's run from its first to its last kept block, so postings shrink less than blocks)
            assert net['blocks_kept'] < 0.8 * safe['blocks_kept'], (k, plain, safe, net)
            assert postings(net) < 0.9 * postings(safe), (k, safe, net)
            assert stats['model', k][1] <= 0.1, (k, stats['model', k][1])
