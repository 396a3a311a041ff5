"""Oracle: fast-spectral VHS collision operator Q(f, f), FP64.

Restates ``DGFSVHSGLLScatteringModel`` (frfs/solvers/dgfs/scattering.py:44-286)
and its kernels (frfs/solvers/dgfs/kernels/scattering/vhs-gll.mako:45-301)
step by step, with the reference's FFT count and operation order:
3 + 3*M*Nrho complex 3-D FFTs per distribution.  Test infrastructure only.
"""
from math import gamma as _gamma

import numpy as np

try:                                    # pocketfft with threads, if present
    import scipy.fft as _fft

    def _fftn(a, workers=1):
        return _fft.fftn(a, axes=(-3, -2, -1), workers=workers)

    def _ifftn_unnorm(a, workers=1):
        return _fft.ifftn(a, axes=(-3, -2, -1), norm='forward',
                          workers=workers)
except ImportError:                     # pragma: no cover
    def _fftn(a, workers=1):
        return np.fft.fftn(a, axes=(-3, -2, -1))

    def _ifftn_unnorm(a, workers=1):
        return np.fft.ifftn(a, axes=(-3, -2, -1), norm='forward')


def vhs_prefactor(vm, omega, dRef, Tref, alpha=1.0):
    """scattering.py:50-65: gamma = 2(1-omega), prefactor from invKn."""
    gam = 2.0 * (1 - omega)
    invKn = vm.H0 * np.sqrt(2.0) * np.pi * vm.n0 * dRef * dRef * \
        (Tref / vm.T0)**(omega - 0.5)
    pref = invKn * alpha / (2.0**(2 - omega + alpha) * _gamma(2.5 - omega)
                            * np.pi)
    return gam, pref, 1.0 / invKn


def lgrid(N):
    """scattering.py:79-89: l0 = [0..N/2-1, -N/2..-1], l[:, idv], x slowest."""
    l0 = np.concatenate((np.arange(0, N // 2), np.arange(-N // 2, 0)))
    I, J, K = np.meshgrid(np.arange(N), np.arange(N), np.arange(N),
                          indexing='ij')
    return np.stack([l0[I].ravel(), l0[J].ravel(), l0[K].ravel()]).astype(
        np.float64)


def _sinc(s):
    # vhs-gll.mako:11-14 (FP64 branch): sin(s+1e-15)/(s+1e-15)
    return np.sin(s + 1e-15) / (s + 1e-15)


def precompute(vm, gam):
    """precompute_aa / precompute_bb (vhs-gll.mako:45-101).

    Returns aa[(p*M+q), r], bb1[p, r], bb2[r] in FP64.
    """
    l = lgrid(vm.Nv)
    L, qz, qw, sz = vm.L, vm.qz, vm.qw, vm.sz
    Nrho, M = vm.Nrho, vm.M
    aa = np.empty((Nrho * M, vm.vsize))
    for p in range(Nrho):
        fac = np.pi / L * qz[p] / 2.0
        for q in range(M):
            aa[p * M + q] = fac * (sz[q, 0] * l[0] + sz[q, 1] * l[1]
                                   + sz[q, 2] * l[2])
    cs = np.sqrt(l[0] * l[0] + l[1] * l[1] + l[2] * l[2])
    bb1 = np.empty((Nrho, vm.vsize))
    bb2 = np.zeros(vm.vsize)
    for p in range(Nrho):
        bb1[p] = qz[p]**(gam + 2.0) * 4 * np.pi * _sinc(np.pi / L * qz[p] / 2.0 * cs)
        bb2 += qw[p] * qz[p]**(gam + 2.0) * 16 * np.pi * np.pi * \
            _sinc(np.pi / L * qz[p] * cs)
    return aa, bb1, bb2


class VHSOracle:
    """Q(f) exactly as ``fs`` computes it (scattering.py:227-286)."""

    def __init__(self, vm, omega, dRef, Tref, workers=1):
        self.vm = vm
        self.gamma, self.prefac, self.Kn = vhs_prefactor(vm, omega, dRef, Tref)
        self.aa, self.bb1, self.bb2 = precompute(vm, self.gamma)
        self.workers = workers

    def Q(self, f):
        """One distribution f[vsize] (FP64) -> Q[vsize]."""
        vm = self.vm
        N, n, P = vm.Nv, vm.vsize, vm.Nrho * vm.M
        shp = (N, N, N)
        w = self.workers
        fC = np.asarray(f, dtype=np.float64).astype(np.complex128)   # r2z
        FTf = _fftn(fC.reshape(shp), w).ravel()                        # FWD
        FTf = FTf / n                                                  # cosSinMul scale
        cosa, sina = np.cos(self.aa), np.sin(self.aa)
        t1 = cosa * FTf[None, :]
        t2 = sina * FTf[None, :]
        t3 = _ifftn_unnorm(t1.reshape((P,) + shp), w).reshape(P, n)    # INV
        t4 = _ifftn_unnorm(t2.reshape((P,) + shp), w).reshape(P, n)    # INV
        t2 = t3 * t3 + t4 * t4                                         # magSqr
        t1 = _fftn(t2.reshape((P,) + shp), w).reshape(P, n)            # FWD
        # computeQG (vhs-gll.mako:172-207)
        intw = (2.0 * vm.qw * vm.sw / n)[:, None] * self.bb1           # [Nrho, n]
        QGhat = np.einsum('pr,pqr->r', intw, t1.reshape(vm.Nrho, vm.M, n))
        QG = _ifftn_unnorm(QGhat.reshape(shp), w).ravel()              # INV
        FTf = FTf * self.bb2                                           # ax
        fCl = _ifftn_unnorm(FTf.reshape(shp), w).ravel()               # INV
        # output (vhs-gll.mako:246-266)
        return self.prefac * (QG.real - np.asarray(f) * fCl.real)

    def Q_batch(self, F):
        return np.stack([self.Q(f) for f in F])

    def gain_loss(self, f):
        """Split of Q into prefac*QG and prefac*f*fC (same steps as ``Q``)."""
        q = self.Q(f)
        vm = self.vm
        n = vm.vsize
        FTf = _fftn(np.asarray(f, np.complex128).reshape((vm.Nv,) * 3)).ravel() / n
        fCl = _ifftn_unnorm((FTf * self.bb2).reshape((vm.Nv,) * 3)).ravel().real
        loss = self.prefac * np.asarray(f) * fCl
        return q + loss, loss
