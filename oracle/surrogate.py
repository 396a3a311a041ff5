"""Oracle: FP64 forward/backward of the surrogate MLP (test infrastructure).

Restates, in numpy FP64, the network the surrogate trains on the GPU:
x -> GELU(x W1^T + b1) -> GELU(. W2^T + b2) -> GELU(. W3^T + b3) -> . W4^T + b4
with GELU(z) = z Phi(z) (erf form) and the per-row relative squared error
L = (1/B) sum_b |y_b - t_b|^2 / (|t_b|^2 + delta).  There is no learned
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
    return h @ W[3].T + b[3], acts, zs


def loss_and_grads(x, t, W, b, delta=1e-12):
    y, acts, zs = forward(x, W, b)
    B = x.shape[0]
    den = (t * t).sum(1, keepdims=True) + delta
    L = float((((y - t)**2).sum(1, keepdims=True) / den).mean())
    g = 2.0 * (y - t) / (den * B)
    gW, gb = [None] * 4, [None] * 4
    for l in (3, 2, 1, 0):
        gW[l] = g.T @ acts[l]
        gb[l] = g.sum(0)
        if l > 0:
            g = (g @ W[l]) * gelu_grad(zs[l - 1])
    return L, gW, gb
