"""Gauss-Jacobi and Gauss-Legendre-Lobatto rules (host, FP64).

Same rules as frfs/quadratures.py:7-54 (``zwgj``/``zwglj``): nodes and
weights of the Jacobi weight (1-x)^a (1+x)^b on [-1, 1], here computed by
the Golub-Welsch eigenvalue method from the three-term recurrence of the
monic Jacobi polynomials.
"""
from math import gamma, lgamma, exp

import numpy as np


def _jacobi_recurrence(n, a, b):
    """alpha_k, beta_k (k < n) of the monic Jacobi recurrence."""
    alpha = np.zeros(n)
    beta = np.zeros(n)
    for k in range(n):
        s = 2 * k + a + b
        if k == 0:
            alpha[0] = (b - a) / (a + b + 2)
            beta[0] = 2.0**(a + b + 1) * exp(lgamma(a + 1) + lgamma(b + 1)
                                             - lgamma(a + b + 2))
        else:
            alpha[k] = (b * b - a * a) / (s * (s + 2))
            if k == 1:
                beta[1] = 4 * (a + 1) * (b + 1) / ((a + b + 2)**2 * (a + b + 3))
            else:
                beta[k] = (4 * k * (k + a) * (k + b) * (k + a + b)
                           / (s * s * (s + 1) * (s - 1)))
    return alpha, beta


def _golub_welsch(alpha, beta):
    J = np.diag(alpha) + np.diag(np.sqrt(beta[1:]), 1) + np.diag(np.sqrt(beta[1:]), -1)
    z, V = np.linalg.eigh(J)
    idx = np.argsort(z)
    return z[idx], beta[0] * V[0, idx]**2


def gauss_jacobi(n, a=0.0, b=0.0):
    """n-point Gauss-Jacobi rule on [-1, 1]."""
    return _golub_welsch(*_jacobi_recurrence(n, a, b))


def gauss_lobatto_jacobi(n, a=0.0, b=0.0):
    """n-point Gauss-Lobatto-Jacobi rule on [-1, 1] (endpoints included)."""
    alpha, beta = _jacobi_recurrence(n, a, b)
    # Lobatto modification: choose alpha[n-1], beta[n-1] so that the n-point
    # rule has nodes at -1 and +1 (Golub 1973).
    N = n - 2
    apb1 = a + b + 1.0
    alpha[n - 1] = (a - b) / (2.0 * N + apb1 + 1.0)
    beta[n - 1] = (4.0 * (N + a + 1) * (N + b + 1) * (N + apb1)
                   / ((2.0 * N + apb1) * (2.0 * N + apb1 + 1)**2))
    return _golub_welsch(alpha, beta)


def gll_points(n):
    """Gauss-Legendre-Lobatto points (n >= 2) in increasing order."""
    z, _ = gauss_lobatto_jacobi(n)
    z[0], z[-1] = -1.0, 1.0
    # enforce exact symmetry
    return 0.5 * (z - z[::-1])


def gll_weights(n):
    """GLL weights 2 / (n (n-1) P_{n-1}(x)^2)."""
    x = gll_points(n)
    P = np.polynomial.legendre.legval(x, [0] * (n - 1) + [1])
    return 2.0 / (n * (n - 1) * P * P)
