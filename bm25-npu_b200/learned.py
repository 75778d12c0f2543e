"""Learned starting bounds of the pruned Search (no counterpart in the reference).

The plain engine generates the training data -- each training query's true K-th
score -- and the session's device feature kernel gives each query 32 features
from per-term statistics (its words' largest posting scores, means and document
frequencies; the layout is in csrc/learned_kernels.cuh).  The threshold MLP
(32 -> 64 -> 64 -> 1, FP32) is trained on the GPU with the engine's own forward,
backward and Adam kernels (bm25_mlp_*) to predict log(K-th score) under a loss
that weighs over-estimates more (an over-estimate sends the query back to the
plain path).  A margin, chosen on held-out queries for a target fallback rate,
turns a prediction y into the starting bound tau = max(exp(y - margin), safe
bound).  Pruning never changes a result: a query whose bound proves too high is
searched again on the plain path.
"""

import ctypes
from ctypes import c_float, c_int32, c_void_p
from dataclasses import dataclass, field

import numpy as np

from . import _native as n

FEATURES = 32
HIDDEN = 64


def param_count():
    return int(n.engine_library().bm25_mlp_param_count())


def _check(status, what):
    if status != n.BM25_OK:
        buf = ctypes.create_string_buffer(512)
        n.engine_library().bm25_mlp_last_error(buf, len(buf))
        raise RuntimeError(f'{what}: {buf.value.decode()} (status {status})')


def init_params(seed, bias=0.0):
    """He-initialised flat parameters (W1 | b1 | W2 | b2 | w3 | b3), b3 = bias."""
    rng = np.random.default_rng(seed)
    w1 = rng.normal(0.0, np.sqrt(2.0 / FEATURES), (HIDDEN, FEATURES))
    w2 = rng.normal(0.0, np.sqrt(2.0 / HIDDEN), (HIDDEN, HIDDEN))
    w3 = rng.normal(0.0, np.sqrt(1.0 / HIDDEN), HIDDEN)
    p = np.concatenate([w1.ravel(), np.zeros(HIDDEN), w2.ravel(), np.zeros(HIDDEN), w3, [bias]])
    assert p.size == param_count()
    return p.astype(np.float32)


@dataclass
class ThresholdModel:
    """Trained MLP parameters plus the margin subtracted from its log-score prediction."""

    params: np.ndarray
    margin: float
    report: dict = field(default_factory=dict)

    def save(self, path):
        np.savez(path, params=self.params, margin=np.float32(self.margin))

    @classmethod
    def load(cls, path):
        z = np.load(path)
        return cls(np.ascontiguousarray(z['params'], dtype=np.float32), float(z['margin']))


def training_set(session, qoffsets, words, k, batch=2048, device='cuda:0'):
    """Features [N, 32], safe bounds [N] and the plain engine's K-th scores [N] for one K.

    The session must be a prune session with query_capacity >= batch and enough word capacity."""
    import torch
    dev = torch.device(device)
    qoffsets = np.ascontiguousarray(qoffsets, dtype=np.int64)
    words = np.ascontiguousarray(words, dtype=np.int32)
    q = qoffsets.size - 1
    feats = np.empty((q, FEATURES), dtype=np.float32)
    safe = np.empty(q, dtype=np.float32)
    kth = np.empty(q, dtype=np.float32)
    stream = torch.cuda.current_stream(dev)
    for b in range(0, q, batch):
        e = min(q, b + batch)
        off = qoffsets[b:e + 1] - qoffsets[b]
        w = words[qoffsets[b]:qoffsets[e]]
        d_off = torch.from_numpy(off).to(dev)
        d_w = torch.from_numpy(w if w.size else np.zeros(1, np.int32)).to(dev)
        d_s = torch.empty((e - b, k), dtype=torch.float32, device=dev)
        d_i = torch.empty((e - b, k), dtype=torch.int32, device=dev)
        d_f = torch.empty((e - b, FEATURES), dtype=torch.float32, device=dev)
        d_safe = torch.empty(e - b, dtype=torch.float32, device=dev)
        session.search_device(d_off.data_ptr(), d_w.data_ptr(), e - b, k, d_s.data_ptr(), d_i.data_ptr(),
                              stream.cuda_stream)
        session.query_features_device(d_off.data_ptr(), d_w.data_ptr(), e - b, k, d_f.data_ptr(),
                                      d_safe.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize(dev)
        if session.device_status():
            raise RuntimeError('plain Search reported a device error while generating targets')
        kth[b:e] = d_s[:, k - 1].cpu().numpy()
        feats[b:e] = d_f.cpu().numpy()
        safe[b:e] = d_safe.cpu().numpy()
    return feats, safe, kth


def train(features, targets, *, steps=3000, batch=4096, lr=2e-3, over_weight=4.0, seed=0, device='cuda:0'):
    """Adam on the GPU with the engine's MLP kernels; returns (params, per-step loss)."""
    import torch
    lib = n.engine_library()
    dev = torch.device(device)
    x = torch.from_numpy(np.ascontiguousarray(features, dtype=np.float32)).to(dev)
    t = torch.from_numpy(np.ascontiguousarray(targets, dtype=np.float32)).to(dev)
    count = x.shape[0]
    batch = min(batch, count)
    p = torch.from_numpy(init_params(seed, float(np.mean(targets)))).to(dev)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    g = torch.zeros_like(p)
    loss = torch.zeros(steps, dtype=torch.float32, device=dev)
    scratch = torch.empty(int(lib.bm25_mlp_scratch_floats(batch)), dtype=torch.float32, device=dev)
    xb = torch.empty((batch, FEATURES), dtype=torch.float32, device=dev)
    tb = torch.empty(batch, dtype=torch.float32, device=dev)
    rng = np.random.default_rng(seed + 1)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for step in range(steps):
        idx = torch.from_numpy(rng.integers(0, count, batch)).to(dev)
        torch.index_select(x, 0, idx, out=xb)
        torch.index_select(t, 0, idx, out=tb)
        _check(lib.bm25_mlp_gradient(c_void_p(p.data_ptr()), c_void_p(xb.data_ptr()), c_void_p(tb.data_ptr()), batch,
                                     c_float(over_weight), c_void_p(scratch.data_ptr()), c_void_p(g.data_ptr()),
                                     c_void_p(loss[step:].data_ptr()), c_void_p(stream)), 'MLP gradient')
        _check(lib.bm25_mlp_adam(c_void_p(p.data_ptr()), c_void_p(m.data_ptr()), c_void_p(v.data_ptr()),
                                 c_void_p(g.data_ptr()), c_float(lr), c_int32(step + 1), c_void_p(stream)),
               'MLP Adam')
    torch.cuda.synchronize(dev)
    return p.cpu().numpy(), loss.cpu().numpy()


def predict(params, features, device='cuda:0'):
    """MLP forward on the GPU: log K-th score predictions [N]."""
    import torch
    lib = n.engine_library()
    dev = torch.device(device)
    x = torch.from_numpy(np.ascontiguousarray(features, dtype=np.float32)).to(dev)
    p = torch.from_numpy(np.ascontiguousarray(params, dtype=np.float32)).to(dev)
    y = torch.empty(x.shape[0], dtype=torch.float32, device=dev)
    _check(lib.bm25_mlp_forward(c_void_p(p.data_ptr()), c_void_p(x.data_ptr()), x.shape[0], c_void_p(y.data_ptr()),
                                c_void_p(torch.cuda.current_stream(dev).cuda_stream)), 'MLP forward')
    torch.cuda.synchronize(dev)
    return y.cpu().numpy()


def bounds(pred, safe, margin):
    """The starting bounds the device computes: max(exp(y - margin), safe), 0 where safe is -1
    (the query's words hold fewer than K postings)."""
    pred = np.asarray(pred, dtype=np.float32)
    safe = np.asarray(safe, dtype=np.float32)
    tau = np.maximum(np.exp(pred - np.float32(margin)).astype(np.float32), safe)
    return np.where(safe < 0, np.float32(0), tau).astype(np.float32)


def fallback_rate(pred, safe, kth, margin):
    """Share of queries whose bound exceeds their K-th score (they re-run on the plain path)."""
    return float(np.mean(bounds(pred, safe, margin) > kth))


def choose_margin(pred, safe, kth, target=0.02, lo=-1.0, hi=8.0, iters=40):
    """Smallest margin whose fallback rate on these queries is at most `target`."""
    if fallback_rate(pred, safe, kth, hi) > target:
        return hi
    for _ in range(iters):
        mid = 0.5 * (lo + hi)
        if fallback_rate(pred, safe, kth, mid) > target:
            lo = mid
        else:
            hi = mid
    return hi


def fit(session, index_offsets, *, queries=200_000, ks=(10, 32), lo=2, hi=10, seed=7, val_share=0.1,
        target_fallback=0.02, steps=3000, batch=4096, lr=2e-3, over_weight=4.0, gen_batch=2048, device='cuda:0'):
    """Generates training queries (terms drawn by document frequency), their targets and features,
    trains the MLP and chooses the margin; returns a ThresholdModel whose report holds the losses
    and the held-out fallback rate."""
    from .corpus import synthetic_queries
    feats, safes, kths = [], [], []
    per_k = queries // len(ks)
    for i, k in enumerate(ks):
        qo, w = synthetic_queries(index_offsets, per_k, lo, hi, seed + i)
        f, s, t = training_set(session, qo, w, k, gen_batch, device)
        feats.append(f)
        safes.append(s)
        kths.append(t)
    f, s, t = np.concatenate(feats), np.concatenate(safes), np.concatenate(kths)
    order = np.random.default_rng(seed).permutation(t.size)
    nval = max(1, int(t.size * val_share))
    val, tr = order[:nval], order[nval:]
    tr = tr[t[tr] > 0]  # a query with fewer than K matching documents has no K-th score to learn
    params, loss = train(f[tr], np.log(t[tr]), steps=steps, batch=batch, lr=lr, over_weight=over_weight,
                         seed=seed, device=device)
    pred = predict(params, f[val], device)
    margin = choose_margin(pred, s[val], t[val], target_fallback)
    report = {
        'train_queries': int(tr.size), 'val_queries': int(val.size), 'first_loss': float(loss[0]),
        'last_loss': float(np.mean(loss[-50:])), 'margin': float(margin),
        'val_fallback': fallback_rate(pred, s[val], t[val], margin),
        'val_safe_share_of_kth': float(np.mean(np.maximum(s[val], 0)[t[val] > 0] / t[val][t[val] > 0])),
        'val_tau_share_of_kth': float(np.mean(bounds(pred, s[val], margin)[t[val] > 0] / t[val][t[val] > 0])),
    }
    return ThresholdModel(params, float(margin), report)
