"""CPU oracle of the learned scheduler's cost model.  TEST INFRASTRUCTURE ONLY:
the tests use it to check the library's GPU training kernels (forward,
gradient); the product never imports it.

The model is the library's own (the reference has no learned scheduler; its
queues flush when full or older than the latency limit, front_end.cc:325-376,
563-598): y = W3 . relu(W2 relu(W1 x + b1) + b2) + b3, x in R^8, hidden 64,
loss = mean squared error.  Parameters are one flat float vector laid out as
W1 [64][8], b1 [64], W2 [64][64] (W2[j][i]: output j, input i), b2 [64],
W3 [64], b3.  Everything here is float64 numpy; the gradient is the
analytic back-propagation, pinned by finite differences in the CPU tests.
"""
import numpy as np

IN, H = 8, 64
W1, B1 = 0, H * IN
W2 = B1 + H
B2 = W2 + H * H
W3 = B2 + H
B3 = W3 + H
N_PARAMS = B3 + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[W1:B1].reshape(H, IN), p[B1:W2], p[W2:B2].reshape(H, H), p[B2:W3], p[W3:B3], p[B3])


def forward(p, x):
    w1, b1, w2, b2, w3, b3 = unpack(p)
    x = np.asarray(x, dtype=np.float64).reshape(-1, IN)
    a1 = x @ w1.T + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ w2.T + b2
    h2 = np.maximum(a2, 0.0)
    return h2 @ w3 + b3, (x, a1, h1, a2, h2)


def loss(p, x, t):
    y, _ = forward(p, x)
    return float(np.mean((y - np.asarray(t, dtype=np.float64)) ** 2))


def loss_grad(p, x, t):
    """(outputs, gradient of the mean squared error, loss)."""
    w1, b1, w2, b2, w3, b3 = unpack(p)
    y, (x, a1, h1, a2, h2) = forward(p, x)
    t = np.asarray(t, dtype=np.float64)
    n = max(y.size, 1)
    e = y - t
    dy = 2.0 * e / n
    g = np.zeros(N_PARAMS)
    g[W3:B3] = h2.T @ dy
    g[B3] = dy.sum()
    d2 = np.outer(dy, w3) * (a2 > 0)
    g[W2:B2] = (d2.T @ h1).reshape(-1)
    g[B2:W3] = d2.sum(axis=0)
    d1 = (d2 @ w2) * (a1 > 0)
    g[W1:B1] = (d1.T @ x).reshape(-1)
    g[B1:W2] = d1.sum(axis=0)
    return y, g, float(np.mean(e ** 2))


def init(seed):
    """He-initialised parameters (the distribution the library uses)."""
    r = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS)
    p[W1:B1] = r.standard_normal(H * IN) * np.sqrt(2.0 / IN)
    p[W2:B2] = r.standard_normal(H * H) * np.sqrt(2.0 / H)
    p[W3:B3] = r.standard_normal(H) * np.sqrt(1.0 / H)
    p[B1:W2] = r.standard_normal(H) * 0.1
    p[B2:W3] = r.standard_normal(H) * 0.1
    p[B3] = 0.3
    return p
