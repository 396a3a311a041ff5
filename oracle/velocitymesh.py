"""Oracle: velocity mesh, radial quadrature and half-sphere directions.

Restates ``DGFSVelocityMesh`` (frfs/solvers/dgfs/velocitymesh.py:25-135)
and the Gauss-Jacobi rule of frfs/quadratures.py:7-54 in FP64 numpy.
Test infrastructure only (see oracle/__init__.py).
"""
from math import gamma

import numpy as np

R0 = 8.3144598            # velocitymesh.py:8
NA = 6.0221409e+23        # velocitymesh.py:9


def gauss_jacobi(n, a=0.0, b=0.0):
    """Gauss-Jacobi nodes/weights on [-1, 1] by Golub-Welsch.

    Follows frfs/quadratures.py:7-49 (``rjacobi`` recurrence + ``gauss``).
    """
    ra, rb = np.zeros(n), np.zeros(n)
    apbp2 = 2.0 + a + b
    ra[0] = (b - a) / apbp2
    rb[0] = 2.0**(a + b + 1) * gamma(a + 1) * gamma(b + 1) / gamma(apbp2)
    if n > 1:
        rb[1] = 4.0 * (a + 1) * (b + 1) / ((apbp2 + 1) * apbp2 * apbp2)
    apbp2 += 2
    for i in range(1, n - 1):
        ra[i] = (b * b - a * a) / ((apbp2 - 2) * apbp2)
        rb[i + 1] = (4.0 * (i + 1) * (i + 1 + a) * (i + 1 + b) * (i + 1 + a + b)
                     / ((apbp2 * apbp2 - 1) * apbp2 * apbp2))
        apbp2 += 2
    ra[n - 1] = (b * b - a * a) / ((apbp2 - 2) * apbp2)
    scal = rb[0]
    off = np.sqrt(rb[1:])
    z, V = np.linalg.eigh(np.diag(ra) + np.diag(off, -1))
    idx = np.argsort(z)
    z = z[idx]
    V = V[:, idx]
    w = scal * V[0, :]**2
    return z, w


class VelocityMesh:
    """FP64 velocity mesh (velocitymesh.py:25-84, 112-135).

    ``sz`` is the half-sphere direction set (first M points of a 2M-point
    antipodal design), supplied by the caller.
    """

    def __init__(self, Nv, Nrho, sz, *, H0, T0, rho0, molarMass0,
                 cmax, Tmax, dev, quad_alpha=0.0, quad_beta=0.0):
        self.Nv, self.Nrho = int(Nv), int(Nrho)
        self.vsize = self.Nv**3
        self.H0, self.T0, self.rho0, self.molarMass0 = H0, T0, rho0, molarMass0
        self.n0 = rho0 / molarMass0 * NA                       # :32
        self.u0 = np.sqrt(2 * R0 / molarMass0 * T0)            # :33
        cmax_nd = cmax / self.u0                               # :55
        Tmax_nd = Tmax / T0                                    # :58
        self.L = cmax_nd + dev * np.sqrt(Tmax_nd)              # :61
        self.S = self.L * 2.0 / (3.0 + np.sqrt(2.0))           # :62
        self.R = 2 * self.S                                    # :63
        self.cw = (2.0 * self.L / self.Nv)**3                  # :72
        N, L = self.Nv, self.L
        self.c0 = np.linspace(-L + L / N, L - L / N, N)        # :73-74
        I, J, K = np.meshgrid(np.arange(N), np.arange(N), np.arange(N),
                              indexing='ij')
        # idv = I*N^2 + J*N + K, x slowest (:77-84)
        self.cv = np.stack([self.c0[I].ravel(), self.c0[J].ravel(),
                            self.c0[K].ravel()])
        qz, qw = gauss_jacobi(self.Nrho, quad_alpha, quad_beta)
        self.qz = (self.R / 2.0) * (1.0 + qz)                  # :124
        self.qw = (self.R / 2.0) * qw                          # :125
        self.sz = np.asarray(sz, dtype=np.float64)
        self.M = self.sz.shape[0]
        self.sw = 2 * np.pi / self.M                           # :135
