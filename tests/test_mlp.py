"""Threshold MLP: the CUDA forward/backward/Adam kernels against the float64 CPU oracle."""

import ctypes

import numpy as np
import pytest

from oracle import mlp_oracle as mo


def test_oracle_gradient_matches_central_differences():
    rng = np.random.default_rng(1)
    p = mo.init(3).astype(np.float64)
    x = rng.normal(size=(40, mo.IN))
    t = rng.normal(size=40)
    g = mo.gradient(p, x, t, 4.0)
    for q in rng.choice(mo.PARAMS, size=60, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[q] += h
        pm[q] -= h
        num = (mo.loss(pp, x, t, 4.0) - mo.loss(pm, x, t, 4.0)) / (2 * h)
        assert abs(num - g[q]) <= 1e-6 + 1e-4 * abs(num), (q, num, g[q])


def test_param_count_matches_oracle(pkg):
    assert pkg._native.engine_library().bm25_mlp_param_count() == mo.PARAMS


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


@pytest.mark.gpu
def test_forward_and_gradient_match_oracle(pkg, cuda_ok):
    import torch
    lib = pkg._native.engine_library()
    rng = np.random.default_rng(7)
    p = mo.init(11)
    batch = 300  # not a multiple of the kernels' row blocks
    x = rng.normal(size=(batch, mo.IN)).astype(np.float32)
    t = rng.normal(size=batch).astype(np.float32)
    dp, dx, dt = _dev(torch, p), _dev(torch, x), _dev(torch, t)
    y = torch.empty(batch, dtype=torch.float32, device='cuda')
    assert lib.bm25_mlp_forward(dp.data_ptr(), dx.data_ptr(), batch, y.data_ptr(), None) == 0
    ref = mo.forward(p, x)
    assert np.allclose(y.cpu().numpy(), ref, rtol=1e-5, atol=1e-5)
    scratch = torch.empty(lib.bm25_mlp_scratch_floats(batch), dtype=torch.float32, device='cuda')
    g = torch.empty(mo.PARAMS, dtype=torch.float32, device='cuda')
    loss = torch.empty(1, dtype=torch.float32, device='cuda')
    assert lib.bm25_mlp_gradient(dp.data_ptr(), dx.data_ptr(), dt.data_ptr(), batch, ctypes.c_float(4.0),
                                 scratch.data_ptr(), g.data_ptr(), loss.data_ptr(), None) == 0
    gref = mo.gradient(p, x, t, 4.0)
    gg = g.cpu().numpy()
    scale = np.abs(gref).max()
    assert np.abs(gg - gref).max() <= 1e-4 * scale, np.abs(gg - gref).max() / scale
    assert abs(loss.item() - mo.loss(p, x, t, 4.0)) <= 1e-4 * mo.loss(p, x, t, 4.0)
    # deterministic: the same call gives the same bits
    g2 = torch.empty_like(g)
    lib.bm25_mlp_gradient(dp.data_ptr(), dx.data_ptr(), dt.data_ptr(), batch, ctypes.c_float(4.0),
                          scratch.data_ptr(), g2.data_ptr(), None, None)
    assert torch.equal(g, g2)


@pytest.mark.gpu
def test_adam_training_fits_a_smooth_target(pkg, cuda_ok):
    import torch
    lib = pkg._native.engine_library()
    rng = np.random.default_rng(3)
    batch = 2048
    x = rng.normal(size=(batch, mo.IN)).astype(np.float32)
    t = (np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2] - 0.3 * np.abs(x[:, 3])).astype(np.float32)
    dp = _dev(torch, mo.init(5))
    m = torch.zeros(mo.PARAMS, device='cuda')
    v = torch.zeros(mo.PARAMS, device='cuda')
    dx, dt = _dev(torch, x), _dev(torch, t)
    scratch = torch.empty(lib.bm25_mlp_scratch_floats(batch), dtype=torch.float32, device='cuda')
    g = torch.empty(mo.PARAMS, device='cuda')
    loss = torch.empty(1, device='cuda')
    first = None
    for step in range(1, 301):
        assert lib.bm25_mlp_gradient(dp.data_ptr(), dx.data_ptr(), dt.data_ptr(), batch, ctypes.c_float(1.0),
                                     scratch.data_ptr(), g.data_ptr(), loss.data_ptr(), None) == 0
        if first is None:
            first = loss.item()
        assert lib.bm25_mlp_adam(dp.data_ptr(), m.data_ptr(), v.data_ptr(), g.data_ptr(), ctypes.c_float(3e-3), step,
                                 None) == 0
    torch.cuda.synchronize()
    final = mo.loss(dp.cpu().numpy(), x, t, 1.0)
    assert final < 0.2 * first, (first, final)
