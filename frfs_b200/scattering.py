"""Scattering-model plugins: the fast-spectral VHS collision operator.

Drop-in for ``DGFSScatteringModel`` / ``DGFSVHSGLLScatteringModel``
(frfs/solvers/dgfs/scattering.py:16-286): registered by
``scattering_model = 'vhs-gll'``, constructed as ``(backend, cfg, vm)``,
with ``fs(d_arr_in, d_arr_out, elem, upt)`` for one DOF.  The batched
``collide(fin, fout)`` evaluates every DOF in one persistent launch of
``bdgfs_vhs_collide`` (hand-written sm_100a kernel, libbdgfs.so).

Host precompute (FP64, then cast to the state precision):
  prefactor  scattering.py:50-65
  phase      exp(i (pi/L)(qz_p/2) s_{q,a} l0[k]) per axis: the separable
             factors of exp(i a_pq) with a_pq = (pi/L)(qz_p/2)(l . s_q)
             (vhs-gll.mako:45-69)
  gw, bb2    (2 qw_p sw / n) bb1_p and bb2 (vhs-gll.mako:71-101, 172-207);
             sinc(s) = sin(s + 1e-15)/(s + 1e-15) as in vhs-gll.mako:11-14
"""
from math import gamma

import numpy as np
import torch

from . import _lib
from .util import subclass_where  # noqa: F401  (registry helper re-export)


class DGFSScatteringModel:
    scattering_model = None

    def __init__(self, backend, cfg, velocitymesh):
        self.backend = backend
        self.cfg = cfg
        self.vm = velocitymesh
        self.load_parameters()
        self.perform_precomputation()

    def load_parameters(self):
        raise NotImplementedError

    def perform_precomputation(self):
        raise NotImplementedError

    def fs(self, d_arr_in, d_arr_out, elem, upt):
        raise NotImplementedError


def _sinc_ref(s):
    return np.sin(s + 1e-15) / (s + 1e-15)


def vhs_prefactor(vm, omega, dRef, Tref, alpha=1.0, mass=1.0):
    """scattering.py:50-65.  For a species of (normalised) mass ``mass`` the
    self-collision form of frfs/solvers/dgfsbi/scattering.py:81-91 with
    p = q, which reduces to the single-species formula at mass 1."""
    gam = 2.0 * (1 - omega)
    invKn = (vm.H0() * np.sqrt(2.0) * np.pi * vm.n0() * dRef * dRef
             * (Tref / vm.T0())**(omega - 0.5))
    mu = mass / 2.0
    pref = invKn * alpha / (np.sqrt(2.0) * mu**(omega - 0.5)
                            * 2.0**(1 + alpha) * gamma(2.5 - omega) * np.pi)
    return gam, pref, 1.0 / invKn


def vhs_tables(Nv, L, qz, qw, sz, sw, gam):
    """Kernel tables in FP64 numpy (layouts of include/bdgfs.h)."""
    N = Nv
    NH = N // 2 + 1
    n = N**3
    l0 = np.concatenate((np.arange(0, N // 2), np.arange(-N // 2, 0))).astype(np.float64)
    Nrho, M = len(qz), sz.shape[0]
    beta = np.pi / L * qz / 2.0                                    # [Nrho]
    arg = beta[:, None, None, None] * sz[None, :, :, None] * l0[None, None, None, :]
    phase = np.exp(1j * arg)                                       # [Nrho][M][3][N]
    # |l| on the [kz][kx][ky] index order
    kz, kx, ky = np.meshgrid(l0, l0, l0, indexing='ij')
    lmag = np.sqrt(kx * kx + ky * ky + kz * kz)                    # [kz][kx][ky]
    gw = np.empty((Nrho, N, NH, N))
    bb2 = np.zeros((N, N, N))
    for p in range(Nrho):
        bb1 = qz[p]**(gam + 2.0) * 4 * np.pi * _sinc_ref(np.pi / L * qz[p] / 2.0 * lmag)
        gw[p] = (2.0 * qw[p] * sw / n) * bb1[:, :NH, :]
        bb2 += qw[p] * qz[p]**(gam + 2.0) * 16 * np.pi * np.pi * \
            _sinc_ref(np.pi / L * qz[p] * lmag)
    return phase, gw, bb2


def gram_inverse(c0, ndims_vel=3):
    """Inverse Gram matrix of phi = {1, cx, cy, cz, |c|^2} over the grid."""
    N = len(c0)
    cx, cy, cz = np.meshgrid(c0, c0, c0, indexing='ij')
    phi = np.stack([np.ones_like(cx), cx, cy, cz, cx * cx + cy * cy + cz * cz]).reshape(5, -1)
    G = phi @ phi.T
    return np.linalg.inv(G)


class VHSGrid:
    """Device-resident tables of one velocity grid (owned by the caller of
    the C ABI; the kernel never allocates)."""

    def __init__(self, Nv, L, qz, qw, sz, sw, gam, prefac, cw, c0, dtype, device):
        self.Nv, self.Nrho, self.M = Nv, len(qz), sz.shape[0]
        self.dtype = dtype
        phase, gw, bb2 = vhs_tables(Nv, L, qz, qw, sz, sw, gam)
        cdt = torch.complex64 if dtype == torch.float32 else torch.complex128
        self.phase = torch.from_numpy(phase).to(cdt).to(device).contiguous()
        self.gw = torch.from_numpy(gw).to(dtype).to(device).contiguous()
        self.bb2 = torch.from_numpy(bb2).to(dtype).to(device).contiguous()
        self.c0 = torch.from_numpy(np.asarray(c0, np.float64)).to(device)
        self.ginv = torch.from_numpy(gram_inverse(c0)).to(device).contiguous()
        self.prefac, self.cw = float(prefac), float(cw)
        self.struct = _lib.VhsGrid(
            Nv=Nv, Nrho=self.Nrho, M=self.M, fp64=int(dtype == torch.float64), tile=0,
            prefac=self.prefac, cw=self.cw, phase=self.phase.data_ptr(),
            gw=self.gw.data_ptr(), bb2=self.bb2.data_ptr(), c0=self.c0.data_ptr(),
            ginv=self.ginv.data_ptr())


class VHSCollider:
    """Owns scratch and the work counter for one set of grids and runs
    ``bdgfs_vhs_collide`` (one persistent launch over all batches)."""

    def __init__(self, grids, device):
        self.grids = list(grids)
        self.device = device
        if any(g.phase.device.type != 'cuda' for g in self.grids):
            raise _lib.BdgfsError('collision tables must be on a CUDA device')
        arr = (_lib.VhsGrid * len(self.grids))(*[g.struct for g in self.grids])
        self._garr = arr
        L = _lib.lib()
        nbytes = L.bdgfs_vhs_scratch_bytes(arr, len(self.grids), 0)
        if nbytes == 0:
            raise _lib.BdgfsError('unsupported velocity grid set for bdgfs_vhs_collide')
        self.scratch = torch.empty(nbytes, dtype=torch.uint8, device=device)
        self.counter = torch.zeros(1, dtype=torch.int64, device=device)

    def __call__(self, batches, project=True, exact=False, stream=None, index=None, count=None):
        """batches: list of (grid_index, f[ndof, n], Q[ndof, n], moments|None).
        index (int32, device) / count (int64 device scalar) restrict the first
        batch to f[index[i]], i < count (read by the kernel)."""
        L = _lib.lib()
        bs = (_lib.VhsBatch * len(batches))()
        for i, (gi, f, Q, mom) in enumerate(batches):
            g = self.grids[gi]
            n3 = g.Nv**3
            if f.dtype != g.dtype or Q.dtype != g.dtype:
                raise TypeError('state dtype does not match the grid tables')
            if not (f.is_contiguous() and Q.is_contiguous()):
                raise ValueError('f and Q must be contiguous [ndof][Nv^3]')
            if f.numel() % n3 or Q.numel() != f.numel():
                raise ValueError('f/Q sizes must be a multiple of Nv^3 and equal')
            if mom is not None and (mom.dtype != torch.float64
                                    or mom.numel() < 10 * (f.numel() // n3)):
                raise ValueError('moments must be float64 [ndof][10]')
            if f.device.type != 'cuda' or Q.device.type != 'cuda':
                raise _lib.BdgfsError('f and Q must be CUDA tensors')
            bs[i] = _lib.VhsBatch(grid=gi, ndof=f.numel() // n3, f=f.data_ptr(),
                                  Q=Q.data_ptr(),
                                  moments=mom.data_ptr() if mom is not None else 0)
            if i == 0 and index is not None:
                if index.dtype != torch.int32 or not index.is_cuda:
                    raise TypeError('index must be an int32 CUDA tensor')
                bs[i].index = index.data_ptr()
            if i == 0 and count is not None:
                if count.dtype != torch.int64 or not count.is_cuda:
                    raise TypeError('count must be an int64 CUDA tensor')
                bs[i].count = count.data_ptr()
        rc = L.bdgfs_vhs_collide(self._garr, len(self.grids), bs, len(batches),
                                 (1 if project else 0) | (2 if exact else 0),
                                 _lib.ptr(self.scratch),
                                 self.scratch.numel(), _lib.ptr(self.counter),
                                 _lib.stream_ptr(stream))
        _lib.check(rc, 'bdgfs_vhs_collide')


class DGFSVHSGLLScatteringModel(DGFSScatteringModel):
    """'vhs-gll' (scattering.py:44-286) on the B200 kernel."""
    scattering_model = 'vhs-gll'

    def load_parameters(self):
        cfg = self.cfg
        self._omega = cfg.getfloat('scattering-model', 'omega')
        self._dRef = cfg.getfloat('scattering-model', 'dRef')
        self._Tref = cfg.getfloat('scattering-model', 'Tref')
        self._mass = cfg.getfloat('scattering-model', 'mass', 1.0)
        self._gamma, self._prefactor, self._Kn = vhs_prefactor(
            self.vm, self._omega, self._dRef, self._Tref, mass=self._mass)
        self._project = cfg.getbool('scattering-model', 'conservation-projection', True)
        # exact Nyquist-plane treatment (second transform per (p, q)): default
        # on for FP64 state and for coarse grids (Nv <= 16), where the
        # second-order Nyquist term reaches 1e-3 of Q; at Nv >= 24 it is ~1e-6
        self._exact = cfg.getbool('scattering-model', 'exact-nyquist',
                                  self.backend.fpdtype == torch.float64
                                  or self.vm.Nv() <= 16)

    def perform_precomputation(self):
        vm, be = self.vm, self.backend
        self.grid = VHSGrid(vm.Nv(), vm.L(), vm.qz(), vm.qw(), vm.sz(), vm.sw(),
                            self._gamma, self._prefactor, vm.cw(), vm.c0(),
                            be.fpdtype, be.device)
        # kernel variant: [scattering-model] tile = auto (autotuned, cached) | <int>
        tile = self.cfg.get('scattering-model', 'tile', 'auto')
        if tile == 'auto':
            from .autotune import tune_vhs
            self.grid.struct.tile = tune_vhs([self.grid], be.device)
        else:
            self.grid.struct.tile = int(tile)
        self.collider = VHSCollider([self.grid], be.device)

    def prefactor(self):
        return self._prefactor

    def collide(self, fin, fout, moments=None, project=None, exact=None):
        """Q for every DOF: fin/fout [ndof][Nv^3] (any leading shape)."""
        n3 = self.vm.vsize()
        self.collider([(0, fin.reshape(-1, n3), fout.reshape(-1, n3), moments)],
                      project=self._project if project is None else project,
                      exact=self._exact if exact is None else exact)

    def fs(self, d_arr_in, d_arr_out, elem, upt):
        """One DOF (elem, upt) of a [neles][nupts][Nv^3] bank (per-DOF shim
        of scattering.py:227)."""
        self.collide(d_arr_in[elem, upt], d_arr_out[elem, upt])


class DGFSVHSGLLHybridScatteringModel(DGFSVHSGLLScatteringModel):
    """'vhs-gll-hybrid': the spectral operator of 'vhs-gll' plus the learned
    surrogate on near-equilibrium cells (``frfs_b200.surrogate``).

    [scattering-model] keys (besides those of 'vhs-gll'):
      surrogate-threshold  Maxwellian deviation below which the surrogate
                           is used (default 0.05)
      surrogate-recheck    fraction of surrogate cells re-checked by the
                           spectral operator (default 0.02)
      surrogate-recheck-every
                           re-check on one collide call out of this many
                           (default 1, every call; 2 with dgfs-tvd-rk2
                           re-checks once per time step)
      surrogate-file       trained model to load (torch.save of state_dict);
                           trained and saved there when absent
      surrogate-family     training distributions: 'couette' (default) or
                           'cavity' (see frfs_b200.surrogate)
      surrogate-center     true: the network works on rows re-centred at
                           zero velocity (QSurrogate center=True: 3x lower
                           Q error on the Couette family); default false,
                           because at 24^3 the spectral operator is not
                           shift-equivariant to better than 0.3-1 % of Q,
                           and on near-equilibrium cells -- whose Q is
                           mostly that operator's own error on a drifting
                           Maxwellian -- the raw-row model follows the
                           spectral solve more closely
      surrogate-nsamples / -epochs / -modes / -width / -lr / -seed
                           training settings (200000 / 20 / 512 / 1024 /
                           3e-4 / 0)
    """
    scattering_model = 'vhs-gll-hybrid'

    def perform_precomputation(self):
        import os
        from .surrogate import CAVITY, COUETTE, HybridCollider, QSurrogate
        super().perform_precomputation()
        cfg, sect = self.cfg, 'scattering-model'
        fams = {'couette': COUETTE, 'cavity': CAVITY}
        fam = cfg.get(sect, 'surrogate-family', 'couette')
        if fam not in fams:
            raise ValueError(f'surrogate-family {fam!r}: expected one of {sorted(fams)}')
        self.surrogate = QSurrogate(self.grid,
                                    nmodes=cfg.getint(sect, 'surrogate-modes', 512),
                                    width=cfg.getint(sect, 'surrogate-width', 1024),
                                    family=fams[fam],
                                    center=cfg.getbool(sect, 'surrogate-center', False))
        path = cfg.get(sect, 'surrogate-file', '')
        if path and os.path.exists(path):
            self.surrogate.load_state_dict(torch.load(path, map_location='cpu'))
        else:
            self.surrogate.fit(nsamples=cfg.getint(sect, 'surrogate-nsamples', 200000),
                               epochs=cfg.getint(sect, 'surrogate-epochs', 20),
                               lr=cfg.getfloat(sect, 'surrogate-lr', 3e-4),
                               seed=cfg.getint(sect, 'surrogate-seed', 0))
            if path:
                torch.save(self.surrogate.state_dict(), path)
        self.hybrid = HybridCollider(self.surrogate,
                                     threshold=cfg.getfloat(sect, 'surrogate-threshold', 0.05),
                                     recheck=cfg.getfloat(sect, 'surrogate-recheck', 0.02),
                                     recheck_every=cfg.getint(sect, 'surrogate-recheck-every', 1),
                                     project=self._project)

    def collide(self, fin, fout, moments=None, project=None, exact=None):
        n3 = self.vm.vsize()
        self.hybrid(fin.reshape(-1, n3), fout.reshape(-1, n3))
