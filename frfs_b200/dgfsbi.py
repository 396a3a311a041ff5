"""Gas mixtures: the velocity mesh and the fast-spectral VSS collision
operator of the reference's 'dgfsbi' solver.

``DGFSBiVelocityMesh`` (frfs/solvers/dgfsbi/velocitymesh.py:11-180): the
box [-L, L]^3 shared by all species, molar masses from
``[velocity-mesh] molarMass1, molarMass2, ...`` (over molarMass0), the
mass-ratio-dependent radius R = 2 S, Gauss-Jacobi radii on [0, R] and M
full-sphere directions (sw = 4 pi / M).

``DGFSBiVSSGLLScatteringModel`` ('vss-gll',
frfs/solvers/dgfsbi/scattering.py:45-330): per ordered species pair the
keys alpha{p}{q}, omega{p}{q}, dRef{p}{q}, Tref{p}{q} of
``[scattering-model]``, and Mpre / ssrulepre for the pre-computation
sphere.  The tables of precompute_a / precompute_bc_pq
(kernels/scattering/vss-gll.mako:31-95) are built here on the host in FP64;
``collide`` evaluates Q_p = sum_q Q_pq for every species and distribution
in one ``bdgfs_vss_collide`` launch, and ``fs`` is the reference's
per-point call.
"""
import ctypes as C
from itertools import product
from math import gamma as _gamma

import numpy as np
import torch

from . import _lib
from .quadratures import gauss_jacobi, gauss_lobatto_jacobi
from .sphericaldesign import full_sphere_design


class DGFSBiVelocityMesh:
    R0 = 8.3144598
    NA = 6.0221409e+23

    def __init__(self, backend, cfg, nspcs):
        self.backend, self.cfg, self._nspcs = backend, cfg, nspcs
        self._construct_velocity_mesh()
        self._load_quadrature()
        self._construct_spherical_mesh()

    def _construct_velocity_mesh(self):
        cfg = self.cfg
        self._H0 = cfg.getfloat('non-dim', 'H0')
        self._T0 = cfg.getfloat('non-dim', 'T0')
        self._rho0 = cfg.getfloat('non-dim', 'rho0')
        self._molarMass0 = cfg.getfloat('non-dim', 'molarMass0')
        self._n0 = self._rho0 / self._molarMass0 * self.NA
        self._u0 = np.sqrt(2 * self.R0 / self._molarMass0 * self._T0)
        self._Nv = cfg.getint('constants', 'Nv')
        self._vsize = self._Nv**3
        self._Nrho = cfg.getint('constants', 'Nrho', self._Nv // 2)
        cmax = cfg.getfloat('velocity-mesh', 'cmax') / self._u0
        Tmax = cfg.getfloat('velocity-mesh', 'Tmax') / self._T0
        dev = cfg.getfloat('velocity-mesh', 'dev')
        self._masses = [cfg.getfloat('velocity-mesh', f'molarMass{p + 1}') / self._molarMass0
                        for p in range(self._nspcs)]
        mr = max(self._masses)
        self._L = cmax + dev * np.sqrt(Tmax)
        self._S = min(self._L * 2.0 / (max(4. * mr / (1. + mr), 2.) + np.sqrt(1. + mr) + 1.),
                      self._L * 2.0 / (max(4. / (1. + mr), 2.) + np.sqrt(1. + 1. / mr) + 1.))
        self._R = 2 * self._S
        N, L = self._Nv, self._L
        self._cw = (2.0 * L / N)**3
        self._c0 = np.linspace(-L + L / N, L - L / N, N)
        idx = np.arange(self._vsize)
        self._cv = np.stack([self._c0[idx // (N * N)], self._c0[(idx // N) % N], self._c0[idx % N]])

    def _load_quadrature(self):
        rule = self.cfg.get('velocity-mesh', 'quad-rule', 'jacobi')
        a = self.cfg.getfloat('velocity-mesh', 'quad-rule-alpha', 0.0)
        b = self.cfg.getfloat('velocity-mesh', 'quad-rule-beta', 0.0)
        rules = {'jacobi': gauss_jacobi, 'lobatto': gauss_lobatto_jacobi}
        if rule not in rules:
            raise ValueError('Valid quads: ' + str(list(rules)))
        z, w = rules[rule](self._Nrho, a, b)
        self._qz = (self._R / 2.0) * (1.0 + z)
        self._qw = (self._R / 2.0) * w

    def _construct_spherical_mesh(self):
        self._ssrule = self.cfg.get('spherical-design-rule', 'ssrule', 'womersley')
        self._M = self.cfg.getint('spherical-design-rule', 'M')
        self._sz = full_sphere_design(self._M, self._ssrule)
        self._sw = 4 * np.pi / self._M

    def Nv(self): return self._Nv
    def Nrho(self): return self._Nrho
    def M(self): return self._M
    def L(self): return self._L
    def vsize(self): return self._vsize
    def qz(self): return self._qz
    def qw(self): return self._qw
    def cv(self): return self._cv
    def c0(self): return self._c0
    def cw(self): return self._cw
    def sz(self): return self._sz
    def sw(self): return self._sw
    def H0(self): return self._H0
    def T0(self): return self._T0
    def rho0(self): return self._rho0
    def n0(self): return self._n0
    def u0(self): return self._u0
    def molarMass0(self): return self._molarMass0
    def masses(self): return self._masses
    def nspcs(self): return self._nspcs


def _lgrid(N):
    l0 = np.concatenate((np.arange(0, N // 2), np.arange(-N // 2, 0))).astype(np.float64)
    idx = np.arange(N**3)
    return np.stack([l0[idx // (N * N)], l0[(idx // N) % N], l0[idx % N]])


class DGFSBiScatteringModel:
    scattering_model = None

    def __init__(self, backend, cfg, velocitymesh):
        self.backend, self.cfg, self.vm = backend, cfg, velocitymesh
        self._nspcs = velocitymesh.nspcs()
        self.load_parameters()
        self.perform_precomputation()


class DGFSBiVSSGLLScatteringModel(DGFSBiScatteringModel):
    scattering_model = 'vss-gll'

    def load_parameters(self):
        cfg, vm = self.cfg, self.vm
        self._Mpre = cfg.getint('scattering-model', 'Mpre')
        self._szpre = full_sphere_design(self._Mpre, cfg.get('scattering-model', 'ssrulepre',
                                                             'womersley'))
        self._swpre = 4 * np.pi / self._Mpre
        self._cases = list(product(range(self._nspcs), repeat=2))
        self._gamma, self._eta, self._prefactor = {}, {}, {}
        m = vm.masses()
        for p, q in self._cases:
            pq = f'{p}{q}'
            alpha = cfg.getfloat('scattering-model', 'alpha' + pq)
            omega = cfg.getfloat('scattering-model', 'omega' + pq)
            dRef = cfg.getfloat('scattering-model', 'dRef' + pq)
            Tref = cfg.getfloat('scattering-model', 'Tref' + pq)
            self._eta[pq] = alpha - 1.
            self._gamma[pq] = 2.0 * (1. - omega)
            invKn = (np.sqrt(1. + m[p] / m[q]) * np.pi * vm.n0() * dRef * dRef
                     * (Tref / vm.T0())**(omega - 0.5) * vm.H0())
            mu = m[p] * m[q] / (m[p] + m[q])
            self._prefactor[pq] = invKn * alpha / (np.sqrt(1. + m[p] / m[q]) * mu**(omega - 0.5)
                                                   * 2.**(1 + alpha) * _gamma(2.5 - omega) * np.pi)

    def kernel_tables(self, p, q):
        """b_pq[r*M+s][l], c_pq[l] (precompute_bc_pq, vss-gll.mako:53-95), FP64."""
        vm = self.vm
        pq = f'{p}{q}'
        m = vm.masses()
        mq = m[q] / (m[p] + m[q])
        sz, szpre = vm.sz(), self._szpre
        Bst = (1.0 + sz @ szpre.T)**self._eta[pq]               # [M, Mpre]
        tl = szpre @ _lgrid(vm.Nv())                            # [Mpre, n]
        b = np.empty((vm.Nrho() * vm.M(), vm.vsize()), complex)
        c = np.zeros(vm.vsize(), complex)
        for r in range(vm.Nrho()):
            fac = np.pi / vm.L() * vm.qz()[r]
            fac_b = self._swpre * vm.qz()[r]**(self._gamma[pq] + 2)
            fac_c = vm.qw()[r] * vm.sw() * fac_b
            b[r * vm.M():(r + 1) * vm.M()] = fac_b * (Bst @ np.exp(-1j * mq * fac * tl))
            c += fac_c * Bst.sum(axis=0) @ np.exp(-1j * fac * tl)
        return b, c

    def perform_precomputation(self):
        vm, be = self.vm, self.backend
        dev = be.device
        S, n = self._nspcs, vm.vsize()
        self.fp64 = int(be.fpdtype == torch.float64)
        ct = torch.complex128 if self.fp64 else torch.complex64
        m = vm.masses()
        b = torch.empty((S * S, vm.Nrho() * vm.M(), n), dtype=ct, device=dev)
        c = torch.empty((S * S, n), dtype=ct, device=dev)
        for p, q in self._cases:
            bb, cc = self.kernel_tables(p, q)
            b[p * S + q].copy_(torch.from_numpy(bb))
            c[p * S + q].copy_(torch.from_numpy(cc))
        self.d_b, self.d_c = b, c
        f64 = lambda a: torch.as_tensor(np.asarray(a, np.float64), device=dev).contiguous()
        self.d_mfrac = f64([m[q] / (m[p] + m[q]) for p, q in self._cases])
        self.d_prefac = f64([self._prefactor[f'{p}{q}'] for p, q in self._cases])
        self.d_rfac = f64(np.pi / vm.L() * vm.qz())
        self.d_rw = f64(vm.qw() * vm.sw() / n)
        self.d_sz = f64(vm.sz())
        nsm = torch.cuda.get_device_properties(dev).multi_processor_count if dev.type == 'cuda' else 1
        self._nctas = nsm
        self._scratch = None

    def _scratch_for(self, items):
        L = _lib.lib()
        nctas = max(1, min(self._nctas, items))
        nb = L.bdgfs_vss_scratch_bytes(self.vm.Nv(), self.fp64, nctas)
        if self._scratch is None or self._scratch.numel() < nb:
            self._scratch = torch.empty(nb, dtype=torch.uint8, device=self.backend.device)
        return self._scratch, nb

    def collide(self, fs, Qs):
        """Qs[p][dof] <- sum_q Q_pq(fs[p][dof], fs[q][dof]) for every
        distribution of the species banks fs (each [..., Nv^3])."""
        S, n = self._nspcs, self.vm.vsize()
        if len(fs) != S or len(Qs) != S:
            raise ValueError(f'need {S} species banks')
        ndof = fs[0].numel() // n
        a = _lib.VssArgs(Nv=self.vm.Nv(), nspcs=S, Nrho=self.vm.Nrho(), M=self.vm.M(),
                         ndof=ndof, fp64=self.fp64, mfrac=self.d_mfrac.data_ptr(),
                         prefac=self.d_prefac.data_ptr(), rfac=self.d_rfac.data_ptr(),
                         rw=self.d_rw.data_ptr(), sz=self.d_sz.data_ptr(), b=self.d_b.data_ptr(),
                         c=self.d_c.data_ptr())
        for p in range(S):
            if fs[p].numel() != ndof * n or Qs[p].numel() != ndof * n:
                raise ValueError('species banks must hold the same distributions')
            a.f[p], a.Q[p] = fs[p].data_ptr(), Qs[p].data_ptr()
        scratch, nb = self._scratch_for(ndof * S)
        _lib.check(_lib.lib().bdgfs_vss_collide(C.byref(a), scratch.data_ptr(), nb,
                                                _lib.stream_ptr()), 'bdgfs_vss_collide')

    def fs(self, elem, upt, *args):
        """The reference's per-point call: args = f_0..f_{S-1}, Q_0..Q_{S-1}
        banks [neles][nupts][Nv^3]; Q_p(elem, upt) = sum_q Q_pq."""
        S = self._nspcs
        if len(args) != 2 * S:
            raise ValueError('Need to be equal')
        self.collide([a[elem, upt] for a in args[:S]], [a[elem, upt] for a in args[S:]])
