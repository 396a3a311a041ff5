"""Velocity mesh of the DGFS system (host precompute, FP64).

Interface and numbers of ``DGFSVelocityMesh``
(frfs/solvers/dgfs/velocitymesh.py:11-162): reads ``[non-dim]``,
``[constants]``, ``[velocity-mesh]`` and ``[spherical-design-rule]``.

* L = cmax/u0 + dev*sqrt(Tmax/T0); S = 2L/(3+sqrt(2)); R = 2S
  (velocitymesh.py:61-63); cw = (2L/Nv)^3; cell centres
  c0 = linspace(-L+L/Nv, L-L/Nv, Nv); velocity index (I*Nv + J)*Nv + K with
  I the x index (slowest) (velocitymesh.py:72-84).
* radial Gauss-Jacobi rule mapped to [0, R] (velocitymesh.py:112-126).
* half-sphere directions and sw = 2*pi/M (velocitymesh.py:128-135).

For a species of molar mass ``molarMass`` != molarMass0 (multi-species
self-collisions) the mesh is the same construction; the mass enters only
the collision prefactor.
"""
import numpy as np

from .quadratures import gauss_jacobi, gauss_lobatto_jacobi
from .sphericaldesign import half_sphere_design


class DGFSVelocityMesh:
    R0 = 8.3144598
    NA = 6.0221409e+23

    def __init__(self, backend, cfg, sect_suffix=''):
        self.backend = backend
        self.cfg = cfg
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
        # NvBatchSize is read for interface compatibility; the FR kernels
        # process all Nv^3 velocities in one pass (no batching).
        self._NvBatchSize = cfg.getint('constants', 'NvBatchSize', self._vsize)
        if self._vsize % self._NvBatchSize:
            raise ValueError('NvBatchSize must divide Nv^3')
        self._NvBatches = self._vsize // self._NvBatchSize
        self._Nrho = cfg.getint('constants', 'Nrho', self._Nv // 2)
        cmax = cfg.getfloat('velocity-mesh', 'cmax') / self._u0
        Tmax = cfg.getfloat('velocity-mesh', 'Tmax') / self._T0
        dev = cfg.getfloat('velocity-mesh', 'dev')
        self._L = cmax + dev * np.sqrt(Tmax)
        self._S = self._L * 2.0 / (3.0 + np.sqrt(2.0))
        self._R = 2 * self._S
        N, L = self._Nv, self._L
        self._cw = (2.0 * L / N)**3
        self._c0 = np.linspace(-L + L / N, L - L / N, N)
        idx = np.arange(self._vsize)
        I, J, K = idx // (N * N), (idx // N) % N, idx % N
        self._cv = np.stack([self._c0[I], self._c0[J], self._c0[K]])

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
        self._sz = half_sphere_design(self._M, self._ssrule)
        self._sw = 2 * np.pi / self._M

    def Nv(self): return self._Nv
    def Nrho(self): return self._Nrho
    def NvBatches(self): return self._NvBatches
    def NvBatchSize(self): return self._NvBatchSize
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
