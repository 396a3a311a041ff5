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
from fractions import Fraction
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


def mixture_gram_inverse(c0, masses):
    """Inverse Gram matrix of the mixture's constraint functions over the
    grid, the species' values concatenated: 1 on species p (one per
    species), then m_p c_x, m_p c_y, m_p c_z and m_p |c|^2 on every species."""
    S = len(masses)
    cx, cy, cz = np.meshgrid(c0, c0, c0, indexing='ij')
    phi = np.stack([np.ones_like(cx), cx, cy, cz, cx * cx + cy * cy + cz * cz]).reshape(5, -1)
    G1 = phi @ phi.T                                   # per-species sums of phi_i phi_j
    K = S + 4
    G = np.zeros((K, K))
    for p, m in enumerate(masses):
        G[p, p] = G1[0, 0]
        G[p, S:] = G[S:, p] = m * G1[0, 1:]
        G[S:, S:] += m * m * G1[1:, 1:]
    return np.linalg.inv(G)


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

    @staticmethod
    def one_plus_cos(sz, szpre):
        """1 + s . t for every direction s of sz [M, 3] and t of szpre
        [Mpre, 3], rounded as the reference's precompute_bc_pq evaluates it
        on the GPU (vss-gll.mako:80-82: 1 + s_x t_x + s_y t_y + s_z t_z,
        contracted into three fused multiply-adds, each rounded once).  Where
        t = -s the exact value is 0 and the rounded one is noise of order
        1e-16 that (.)^(alpha - 1) lifts to order 1e-5; rounding it the same
        way keeps B, and Q, equal to the reference's.  A negative rounded value
        (the reference's pow then gives NaN) is taken as the exact 0."""
        def fma(a, b, c):
            return float(Fraction(a) * Fraction(b) + Fraction(c))
        sz, szpre = np.asarray(sz, dtype=np.float64), np.asarray(szpre, dtype=np.float64)
        out = np.empty((sz.shape[0], szpre.shape[0]))
        for y, s in enumerate(sz.tolist()):
            for t, u in enumerate(szpre.tolist()):
                out[y, t] = fma(s[2], u[2], fma(s[1], u[1], fma(s[0], u[0], 1.0)))
        return np.maximum(out, 0.0)

    def kernel_tables(self, p, q):
        """b_pq[r*M+s][l], c_pq[l] (precompute_bc_pq, vss-gll.mako:53-95), FP64."""
        vm = self.vm
        pq = f'{p}{q}'
        m = vm.masses()
        mq = m[q] / (m[p] + m[q])
        sz, szpre = vm.sz(), self._szpre
        Bst = self.one_plus_cos(sz, szpre)**self._eta[pq]        # [M, Mpre]
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
        # FP64 conservation projection (species masses, total momentum and
        # energy); the reference's operator has none, so parity runs disable it
        self._project = self.cfg.getbool('scattering-model', 'conservation-projection', True)
        self.d_c0 = f64(vm.c0())
        self.d_mass = f64(m)
        self.d_ginv = f64(mixture_gram_inverse(vm.c0(), m).ravel())

    def _scratch_for(self, items):
        L = _lib.lib()
        nctas = max(1, min(self._nctas, items))
        nb = L.bdgfs_vss_scratch_bytes(self.vm.Nv(), self.fp64, nctas)
        if self._scratch is None or self._scratch.numel() < nb:
            self._scratch = torch.empty(nb, dtype=torch.uint8, device=self.backend.device)
        return self._scratch, nb

    def collide(self, fs, Qs, project=None):
        """Qs[p][dof] <- sum_q Q_pq(fs[p][dof], fs[q][dof]) for every
        distribution of the species banks fs (each [..., Nv^3]), then the
        FP64 conservation projection unless disabled (``project`` or
        ``[scattering-model] conservation-projection``)."""
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
        if self._project if project is None else project:
            pa = _lib.VssProjArgs(Nv=self.vm.Nv(), nspcs=S, ndof=ndof, fp64=self.fp64,
                                  c0=self.d_c0.data_ptr(), mass=self.d_mass.data_ptr(),
                                  ginv=self.d_ginv.data_ptr())
            for p in range(S):
                pa.Q[p] = Qs[p].data_ptr()
            _lib.check(_lib.lib().bdgfs_vss_project(C.byref(pa), _lib.stream_ptr()),
                       'bdgfs_vss_project')

    def fs(self, elem, upt, *args):
        """The reference's per-point call: args = f_0..f_{S-1}, Q_0..Q_{S-1}
        banks [neles][nupts][Nv^3]; Q_p(elem, upt) = sum_q Q_pq."""
        S = self._nspcs
        if len(args) != 2 * S:
            raise ValueError('Need to be equal')
        self.collide([a[elem, upt] for a in args[:S]], [a[elem, upt] for a in args[S:]])


# ---------------------------------------------------------------------------
# The 'dgfsbi' system: one FR advection per species on the shared mesh and
# velocity grid, the mixture collision operator across species.
# ---------------------------------------------------------------------------
from .mesh import ElementGeometry                                      # noqa: E402
from .system import (DGFSBCInters, DGFSBoundaries, DGFSElements,       # noqa: E402
                     DGFSSystem, DGFSWallSpecularBCInters)
from .util import npeval, subclass_where                               # noqa: E402


class SpeciesMesh:
    """One species' view of the mixture velocity mesh: the shared grid,
    with that species' molar mass for its Maxwellians."""

    def __init__(self, vm, p):
        self._vm, self.species = vm, p

    def __getattr__(self, k):
        return getattr(self._vm, k)

    def mass(self):
        return self._vm.masses()[self.species]


def species_maxwellian(vm, m, nden, T, u):
    """nden (m/(pi T))^1.5 exp(-m |c - u|^2 / T) on the grid (non-dimensional;
    frfs/solvers/dgfsbi/initcond.py:68-76)."""
    return nden * (m / (np.pi * T))**1.5 * np.exp(-m * np.sum((vm.cv() - u)**2, axis=0) / T)


class DGFSBiMaxwellianInitCondition:
    """'maxwellian' of the 'dgfsbi' system (frfs/solvers/dgfsbi/initcond.py:
    47-117): per species the number density nden{p+1} (over n0), the shared
    T and (ux, uy, uz); walls use nden = 1.  Raises ``ValueError`` when the
    grid does not hold a species' number density, velocity and temperature
    to 1e-5 (the reference's support test)."""
    model = 'maxwellian'

    def __init__(self, backend, cfg, vm, name, wall=False):
        self.vm, S = vm, vm.nspcs()
        u0 = vm.u0()
        self._nden = [1.0] * S if wall else [cfg.getfloat(name, f'nden{p + 1}') / vm.n0()
                                             for p in range(S)]
        self._T = cfg.getfloat(name, 'T') / vm.T0()
        self._u = np.array([cfg.getfloat(name, k) / u0 for k in ('ux', 'uy', 'uz')]).reshape(3, 1)
        m, cv, cw = vm.masses(), vm.cv(), vm.cw()
        self._init_vals = []
        for p in range(S):
            f = species_maxwellian(vm, m[p], self._nden[p], self._T, self._u)
            mcw = m[p] * cw
            rho = np.sum(f) * mcw
            u = cv @ f * mcw / rho
            T = np.sum(f * np.sum((cv - u[:, None])**2, axis=0)) * (2.0 / 3.0 * mcw * m[p]) / rho
            ok = (np.isclose(self._nden[p], rho / m[p], rtol=1e-5, atol=1e-5)
                  and np.allclose(self._u[:, 0] * u0, u * u0, rtol=1e-5, atol=1e-5)
                  and np.isclose(self._T * vm.T0(), T * vm.T0(), rtol=1e-5, atol=1e-5))
            if not ok:
                raise ValueError(f'Bulk properties not conserved for species {p}! Check Nv, dev')
            self._init_vals.append(f)

    def get_init_vals(self):
        return self._init_vals

    def unondim(self):
        return self._u


class DGFSBiMaxwellianExprInitCondition:
    """'maxwellianExpr' of the 'dgfsbi' system (frfs/solvers/dgfsbi/
    initcond.py:138-212): per species p a Maxwellian of mass m_p whose
    number density nden{p+1} and the shared ux, uy, uz, T are expressions of
    x, y, z and the [constants], evaluated at every solution point; built on
    the device (the species Maxwellian is the unit-mass one at T / m_p).
    Raises ``ValueError`` when a point's number density is not represented
    to 1e-5."""
    model = 'maxwellianExpr'

    def __init__(self, backend, cfg, vm, name):
        self.cfg, self.vm, self.name = cfg, vm, name
        self._vars = cfg.items_as('constants', float)
        if any(d in self._vars for d in 'xyz'):
            raise ValueError('Invalid constants (x, y, or z) in config file')

    def fields(self, p, ploc):
        """Non-dimensional (nden, ux, uy, uz, T) of species p at ploc[..., ndims]."""
        vm = self.vm
        v = dict(self._vars)
        v.update(zip('xyz', np.moveaxis(np.asarray(ploc, dtype=np.float64), -1, 0)))
        shp = np.asarray(ploc).shape[:-1]
        keys = (f'nden{p + 1}', 'ux', 'uy', 'uz', 'T')
        scale = (vm.n0(), vm.u0(), vm.u0(), vm.u0(), vm.T0())
        return [np.broadcast_to(np.asarray(npeval(self.cfg.getexpr(self.name, k), v),
                                           dtype=np.float64), shp) / sc
                for k, sc in zip(keys, scale)]

    def apply_init_vals(self, p, bank, ploc):
        vm = self.vm
        n, ux, uy, uz, T = (a.reshape(-1) for a in self.fields(p, ploc))
        Tm = T / vm.masses()[p]
        u2 = ux * ux + uy * uy + uz * uz
        U = np.stack([n, n * ux, n * uy, n * uz, 1.5 * n * Tm + n * u2], axis=-1)
        dev = bank.device
        Ud = torch.as_tensor(U, dtype=torch.float64, device=dev).contiguous()
        c0 = torch.as_tensor(vm.c0(), dtype=torch.float64, device=dev).contiguous()
        nv = vm.vsize()
        _lib.check(_lib.lib().bdgfs_bgk_maxwellian(Ud.data_ptr(), bank.numel() // nv, vm.Nv(),
                                                   int(bank.dtype == torch.float64), c0.data_ptr(),
                                                   bank.data_ptr(), _lib.stream_ptr()),
                   'bdgfs_bgk_maxwellian')
        bulk = bank.reshape(-1, nv).double().sum(-1).cpu().numpy() * vm.cw()
        if not np.allclose(n, bulk, atol=1e-5):
            raise ValueError(f'Bulk properties not conserved for species {p}! Check Nv, dev')


class _BiMaxwellianRows:
    """Wall / inflow rows of one species (frfs/solvers/dgfsbi/inters.py)."""
    wall = True

    def _maxwellian(self):
        vm = self.vm
        bc = DGFSBiMaxwellianInitCondition(self.be, self.cfg, vm._vm, self.sect, wall=self.wall)
        return bc.unondim()[:, 0], bc.get_init_vals()[vm.species]


class DGFSBiWallDiffuseBCInters(_BiMaxwellianRows, DGFSBCInters):
    """'dgfsbi-wall-diffuse' (inters.py:176-283): the diffuse wall with each
    species' wall Maxwellian (nden = 1, that species' mass)."""
    type = 'dgfsbi-wall-diffuse'
    oracle_type = 'dgfs-wall-diffuse'

    def load(self):
        self.rows = [self._maxwellian()]


class DGFSBiWallDiffuseCylBCInters(DGFSBCInters):
    """'dgfsbi-wall-diffuse-cyl' (inters.py:679-759): U_w, T_w expressions of
    the face-point location; f_w = exp(-m |c - U_w|^2/T_w) per face point."""
    type = 'dgfsbi-wall-diffuse-cyl'
    oracle_type = 'dgfs-wall-diffuse'

    def load(self):
        cfg, vm, geo = self.cfg, self.vm, self.geo
        x = np.zeros((3, len(self.pts)))
        for i, w in enumerate(self.pts):
            e, f = geo.wall_fpts[w]
            x[:geo.ndims, i] = geo.plocfpts[e, f]
        env = cfg.items_as('constants', float)
        env.update(x=x[0], y=x[1], z=x[2])

        def ev(k):
            v = npeval(cfg.getexpr(self.sect, k), env)
            return np.broadcast_to(np.asarray(v, dtype=np.float64), (len(self.pts),))
        U = np.stack([ev('ux'), ev('uy'), ev('uz')]) / vm.u0()
        T = ev('T') / vm.T0()
        m, cv = vm.mass(), vm.cv()
        self.rows = [(U[:, i].copy(), np.exp(-m * np.sum((cv - U[:, i:i + 1])**2, axis=0) / T[i]))
                     for i in range(len(self.pts))]

    def point_rows(self):
        return np.arange(len(self.pts), dtype=np.int64)


class DGFSBiWallSpecularBCInters(DGFSWallSpecularBCInters):
    """'dgfsbi-wall-specular' (inters.py:286-421)."""
    type = 'dgfsbi-wall-specular'


class DGFSBiInletBCInters(_BiMaxwellianRows, DGFSBCInters):
    """'dgfsbi-inlet' (inters.py:424-495): u_R = f_in,p where (c - U_in).n < 0,
    f_in,p with the section's nden{p+1}."""
    type = 'dgfsbi-inlet'
    kind = _lib.BC_INLET
    wall = False

    def load(self):
        self.rows = [self._maxwellian()]


class DGFSBiInletNormalShockBCInters(_BiMaxwellianRows, DGFSBCInters):
    """'dgfsbi-inlet-normalshock' (inters.py:498-560): u_R = f_in,p where c.n < 0."""
    type = 'dgfsbi-inlet-normalshock'
    kind = _lib.BC_INLET
    wall = False

    def load(self):
        self.rows = [(np.zeros(3), self._maxwellian()[1])]


class DGFSBiOutletBCInters(DGFSBCInters):
    """'dgfsbi-outlet' (inters.py:563-617): u_R = u_L."""
    type = 'dgfsbi-outlet'
    kind = _lib.BC_OUTLET


class DGFSBiVanishBCInters(DGFSBCInters):
    """'dgfsbi-vanish' (inters.py:620-676): u_R = 0 where c.n < 0."""
    type = 'dgfsbi-vanish'
    kind = _lib.BC_INLET


class DGFSBiSpecies(DGFSSystem):
    """The FR advection of one species: the 'dgfs' system's kernels and fused
    stage on the shared geometry and operators, with this species' boundary
    rows and register banks; no collision model of its own."""

    def __init__(self, bi, p, nreg):
        be = bi.backend
        self.backend, self.cfg, self.mesh = be, bi.cfg, bi.mesh
        self.vm = SpeciesMesh(bi.vm, p)
        self.geo, self.ele, self.ndims = bi.geo, bi.ele, bi.geo.ndims
        self.domain, self.transport = bi.domain, bi.transport
        self.walls = DGFSBoundaries(be, self.geo, self.vm, self.cfg, self.geo.wall_names)
        self.unitCFLdt = bi.unitCFLdt
        E, U, nv = self.ele.neles, self.ele.nupts, self.vm.vsize()
        self.eles_scal_upts_inb_full = [be.empty(E, U, nv) for _ in range(nreg)]
        # face values, then the ghost rows of a partitioned mesh
        nghost = self.domain.nghost if self.domain is not None else 0
        self._uf_rows = be.empty(E * self.ele.nfpts + nghost, nv)
        self._uf = self._uf_rows[:E * self.ele.nfpts].view(E, self.ele.nfpts, nv)
        self._send_rows = {}
        if self.domain is not None:
            for r, rows in self.domain.send.items():
                self._send_rows[r] = torch.as_tensor(rows, dtype=torch.int64, device=be.device)
        self._gen_kernels()

    def collide(self, t, uinbank, foutbank):
        raise NotImplementedError('a species collides through DGFSBiSystem.collide')


class DGFSBiSystem:
    """Drop-in for ``DGFSBiSystem`` (frfs/solvers/dgfsbi/system.py:17-264,
    name 'dgfsbi').  ``species[p]`` advects species p (banks
    ``species[p].eles_scal_upts_inb_full[reg]``, each [neles][nupts][Nv^3]);
    ``rhs`` / ``updatebc`` take the reference's species index ``idx`` ('0',
    '1', ...), ``collide(t, regids)`` takes the reference's register list
    (the S input registers, then the S output registers; or use
    ``collide_banks``).  The species count is that of the
    ``[velocity-mesh] molarMass{p}`` keys (the reference fixes it at 2)."""
    name = 'dgfsbi'

    def __init__(self, backend, mesh, cfg, nreg=3, initsoln=None, partition=None,
                 transport=None):
        """partition = (parts, rank): this system owns the elements
        parts[rank] of the mesh (frfs_b200.partition); transport exchanges
        every species' face values with the neighbouring parts after disu
        (species by species, in the same order on every rank)."""
        self.backend, self.cfg, self.mesh = backend, cfg, mesh
        self.transport = transport
        S = 0
        while cfg.hasopt('velocity-mesh', f'molarMass{S + 1}'):
            S += 1
        if S < 1:
            raise ValueError('[velocity-mesh] needs molarMass1, molarMass2, ...')
        self._nspcs = S
        self.vm = DGFSBiVelocityMesh(backend, cfg, S)
        self.geo = ElementGeometry(mesh, cfg.getint('solver', 'order'))
        self.domain = None
        if partition is not None:
            from .partition import LocalDomain
            self.domain = self.geo = LocalDomain(self.geo, *partition)
        self.ele = DGFSElements(backend, self.geo, self.vm)
        self.ndims = self.geo.ndims
        # time-step estimate (system.py:58-75)
        self.unitCFLdt = np.sqrt(np.min(self.geo.djac)) / self.vm.L() / self.ndims
        smn = cfg.get('scattering-model', 'type')
        self.sm = subclass_where(DGFSBiScatteringModel, scattering_model=smn)(backend, cfg, self.vm)
        self.species = [DGFSBiSpecies(self, p, nreg) for p in range(S)]
        if initsoln is not None:
            for p in range(S):
                self.species[p].eles_scal_upts_inb_full[0].copy_(
                    torch.as_tensor(initsoln[p]).to(self.species[p].eles_scal_upts_inb_full[0]))
        else:
            icn = cfg.get('soln-ics', 'type')
            if icn == 'maxwellian':
                ic = DGFSBiMaxwellianInitCondition(backend, cfg, self.vm, 'soln-ics')
                for p, f in enumerate(ic.get_init_vals()):
                    u = self.species[p].eles_scal_upts_inb_full[0]
                    u.copy_(backend.const(f).expand_as(u))
            elif icn == 'maxwellianExpr':
                ic = DGFSBiMaxwellianExprInitCondition(backend, cfg, self.vm, 'soln-ics')
                for p in range(S):
                    ic.apply_init_vals(p, self.species[p].eles_scal_upts_inb_full[0],
                                       self.geo.plocupts)
            else:
                raise ValueError(f'unsupported initial condition {icn} for dgfsbi')

    def nspcs(self):
        return self._nspcs

    def bank(self, p, reg):
        return self.species[p].eles_scal_upts_inb_full[reg]

    # -- reference system methods ----------------------------------------
    def rhs(self, t, idx, uinbank, foutbank, batch=None, varidx=None):
        """foutbank <- -div F(uinbank) of species int(idx) (system.py:179-218)."""
        self.species[int(idx)].rhs(t, uinbank, foutbank, batch, varidx)

    def updatebc(self, t, idx, uinbank, foutbank, batch=None, varidx=None):
        """disu + update_bc of species int(idx) (system.py:221-238)."""
        self.species[int(idx)].updatebc(t, uinbank, foutbank, batch, varidx)

    def collide(self, t, regids):
        """The reference's call (system.py:241-252): regids = the S input
        registers then the S output registers."""
        S = self._nspcs
        if len(regids) != 2 * S:
            raise ValueError(f'need {2 * S} registers')
        self.sm.collide([self.bank(p, regids[p]) for p in range(S)],
                        [self.bank(p, regids[S + p]) for p in range(S)])

    def collide_banks(self, t, uinbank, foutbank):
        """Q_p(uinbank) -> foutbank of every species p, one launch."""
        S = self._nspcs
        self.collide(t, [uinbank] * S + [foutbank] * S)

    def invmass(self, uinbank, foutbank):
        """foutbank <- M12 uinbank of every species (dgfsbi/system.py:253-263)."""
        for sp in self.species:
            sp.invmass(uinbank, foutbank)

    def macroscopic(self, bank):
        """The per-species fields of the reference's mixture moment writer
        (plugins/dgfsmomwriterbi.py:258-385), non-dimensional and FP64 on the
        GPU, per DOF: mass density rho_p = m_p n_p, velocity U_p, temperature
        T_p, heat flux q_p = m_p^2 sum f |c-U|^2 (c-U) cw and pressure tensor
        P_p = 2 m_p^2 sum f (c-U)(c-U) cw (xx xy xz yy yz zz), both about the
        mixture velocity U = sum rho_p U_p / sum rho_p; plus 'nden' = n_p.
        Returns ([per-species dict], {'rho': mixture rho, 'U': U})."""
        from .system import raw_moments
        ij = ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))
        raws, out = [], []
        for p in range(self._nspcs):
            m = raw_moments(self.bank(p, bank), self.species[p].vm)
            mp = self.vm.masses()[p]
            n = m[:, 0]
            U = m[:, 1:4] / n[:, None]
            trS = m[:, 4] + m[:, 7] + m[:, 9]
            c2 = trS - 2.0 * (U * m[:, 1:4]).sum(1) + (U * U).sum(1) * n
            out.append({'nden': n, 'rho': mp * n, 'U': U, 'T': (2.0 / 3.0) * mp * c2 / n})
            raws.append(m)
        rho = sum(o['rho'] for o in out)
        W = sum(o['rho'][:, None] * o['U'] for o in out) / rho[:, None]
        W2 = (W * W).sum(1)
        for p, (m, o) in enumerate(zip(raws, out)):
            mp2 = self.vm.masses()[p]**2
            m0, m1 = m[:, 0], m[:, 1:4]
            S = torch.zeros(m.shape[0], 3, 3, dtype=torch.float64, device=m.device)
            for k, (a, b) in enumerate(ij):
                S[:, a, b] = S[:, b, a] = m[:, 4 + k]
            trS = S[:, 0, 0] + S[:, 1, 1] + S[:, 2, 2]
            # sum f (c-W)_a (c-W)_b and sum f |c-W|^2 (c-W)_a from the raw moments
            C = (S - W[:, :, None] * m1[:, None, :] - m1[:, :, None] * W[:, None, :]
                 + m0[:, None, None] * W[:, :, None] * W[:, None, :])
            q = (m[:, 10:13] - trS[:, None] * W - 2.0 * torch.einsum('nab,nb->na', S, W)
                 + 2.0 * W * (W * m1).sum(1, keepdim=True) + W2[:, None] * m1
                 - (m0 * W2)[:, None] * W)
            o['q'] = mp2 * q
            o['P'] = torch.stack([2.0 * mp2 * C[:, a, b] for a, b in ij], 1)
        return out, {'rho': rho, 'U': W}

    def moments(self, bank):
        """Per species and DOF (FP64 on the GPU, non-dimensional): number
        density n = sum f cw, velocity U and temperature T = (2/3) m
        sum |c - U|^2 f cw / n, the definitions of the reference's support
        test (initcond.py:80-117)."""
        from .system import macroscopic
        out = []
        for p in range(self._nspcs):
            n, U, T, _, _ = macroscopic(self.bank(p, bank), self.species[p].vm)
            out.append((n, U, T * self.vm.masses()[p]))
        return out
