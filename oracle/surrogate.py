"""Oracle: FP64 forward/backward of the surrogate network (test infrastructure).

Restates, in numpy FP64, the network the surrogate trains on the GPU:
  h1 = GELU(x W1^T + b1), h2 = GELU(h1 W2^T + b2), h3 = GELU(h2 W3^T + b3)
  Y  = [h3, x] W4^T + b4                  (W4: 3k x (w + kin), skip from x)
with GELU(z) = z Phi(z) (erf form) and the per-row relative squared error
of the heads L = (1/B) sum_b |Y_b - t_b|^2 / (|t_b|^2 + delta).  There is no learned
component in the reference; this oracle checks the project's own gradient
kernels.
"""
import numpy as np
from math import erf, sqrt, pi

_verf = np.vectorize(erf)


def gelu(z):
    return 0.5 * z * (1.0 + _verf(z / sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _verf(z / sqrt(2.0))) + z * np.exp(-0.5 * z * z) / sqrt(2.0 * pi)


def forward(x, W, b):
    acts, zs = [x], []
    h = x
    for l in range(3):
        z = h @ W[l].T + b[l]
        zs.append(z)
        h = gelu(z)
        acts.append(h)
    xc = np.concatenate([h, x], axis=1)
    return xc @ W[3].T + b[3], acts, zs, xc


def combine(Y, s):
    """y = Y0 + s Y1 + s^2 Y2 (heads of equal width)."""
    k = Y.shape[1] // 3
    s1 = s[:, None]
    return Y[:, :k] + s1 * Y[:, k:2 * k] + s1 * s1 * Y[:, 2 * k:]


def loss_and_grads(x, t, W, b, delta=1e-12):
    Y, acts, zs, xc = forward(x, W, b)
    B = x.shape[0]
    w = W[0].shape[0]
    den = (t * t).sum(1, keepdims=True) + delta
    L = float((((Y - t)**2).sum(1, keepdims=True) / den).mean())
    g = 2.0 * (Y - t) / (den * B)
    gW, gb = [None] * 4, [None] * 4
    for l in (3, 2, 1, 0):
        gW[l] = g.T @ (xc if l == 3 else acts[l])
        gb[l] = g.sum(0)
        if l > 0:
            g = (g @ W[l][:, :w]) * gelu_grad(zs[l - 1])
    return L, gW, gb
