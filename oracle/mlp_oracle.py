"""CPU oracle of the threshold MLP (test infrastructure only; not on any product path).

Float64 restatement of bm25-npu_b200/csrc/mlp.cu: a 32 -> 64 -> 64 -> 1 ReLU network
whose parameters are one flat array (W1[64][32] | b1[64] | W2[64][64] | b2[64] | w3[64] | b3)
and its loss mean_i w_i * (f(x_i) - t_i)^2 with w_i = over_weight when f(x_i) > t_i, else 1.
The GPU kernels are checked against forward() and gradient() here; gradient() is itself
checked against central differences of loss().
"""

import numpy as np

IN, H = 32, 64
SHAPES = [('W1', (H, IN)), ('b1', (H,)), ('W2', (H, H)), ('b2', (H,)), ('w3', (H,)), ('b3', (1,))]
PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p):
    out, at = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[at:at + n], dtype=np.float64).reshape(shape)
        at += n
    return out


def init(seed=0):
    """He-style initialisation, float32 (the GPU's parameter type)."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in SHAPES:
        if name.startswith('W'):
            parts.append(rng.normal(0.0, np.sqrt(2.0 / shape[1]), size=shape).ravel())
        elif name == 'w3':
            parts.append(rng.normal(0.0, np.sqrt(1.0 / H), size=shape))
        else:
            parts.append(np.zeros(shape))
    return np.concatenate(parts).astype(np.float32)


def forward(p, x, keep=False):
    w = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    a1 = x @ w['W1'].T + w['b1']
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ w['W2'].T + w['b2']
    h2 = np.maximum(a2, 0.0)
    y = h2 @ w['w3'] + w['b3'][0]
    return (y, h1, h2) if keep else y


def loss(p, x, t, over_weight):
    y = forward(p, x)
    e = y - np.asarray(t, dtype=np.float64)
    w = np.where(e > 0, over_weight, 1.0)
    return float(np.mean(w * e * e))


def gradient(p, x, t, over_weight):
    w = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    y, h1, h2 = forward(p, x, keep=True)
    e = y - np.asarray(t, dtype=np.float64)
    wt = np.where(e > 0, over_weight, 1.0)
    dy = 2.0 * wt * e / x.shape[0]
    d2 = (dy[:, None] * w['w3'][None, :]) * (h2 > 0)
    d1 = (d2 @ w['W2']) * (h1 > 0)
    g = {'W1': d1.T @ x, 'b1': d1.sum(0), 'W2': d2.T @ h1, 'b2': d2.sum(0), 'w3': h2.T @ dy, 'b3': np.array([dy.sum()])}
    return np.concatenate([g[name].ravel() for name, _ in SHAPES])
