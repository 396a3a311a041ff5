"""The 'adgfs' system: FR advection with the BGK relaxation operator,
advanced by the ARS IMEX steppers.

Mirrors frfs/solvers/adgfs/system.py (ADGFSSystem, name 'adgfs') and
frfs/solvers/adgfs/scattering.py (ADGFSBGKDirectGLLScatteringModel,
``scattering_model = 'bgk-direct-gll'``), with the reference's method
names (``moment``, ``constructMaxwellian``, ``updateMomentARS``,
``updateDistARS``, ``get_nregs_moms``) on top of the fused stage entry
``bdgfs_ars_stage`` that the project's ARS steppers use.  Moment rows are
FP64 ``[ndof][nalph]``: (rho, rho u, E) for BGK (nalph = 5) and, for
ES-BGK (ADGFSESBGKDirectGLLScatteringModel, 'esbgk-direct-gll'), those
followed by the raw second moments (xx, yy, zz, xy, yz, zx) (nalph = 11),
and for Shakov (ADGFSShakovDirectGLLScatteringModel, 'shakov-direct-gll')
the raw third moments |c|^2 c after them (nalph = 14), as in the
reference.
"""
import ctypes as C

import torch

from . import _lib
from .system import DGFSSystem
from .util import subclass_where  # noqa: F401

ARS_MOM0, ARS_MOML, ARS_MOMU, ARS_DIST = 1, 2, 4, 8
BDF_MOMN, BDF_MOMU, BDF_DIST = 1, 2, 4
R0 = 8.3144598
NA = 6.0221409e+23


class ADGFSScatteringModel:
    """Registry base (scattering.py: ADGFSScatteringModel)."""
    scattering_model = None

    def __init__(self, backend, cfg, velocitymesh):
        self.backend, self.cfg, self.vm = backend, cfg, velocitymesh
        self.load_parameters()
        self.perform_precomputation()

    def collide(self, *args, **kwargs):
        raise RuntimeError('Not valid for asymptotic systems')


class ADGFSBGKDirectGLLScatteringModel(ADGFSScatteringModel):
    """BGK relaxation nu (M[f] - f), nu = prefac rho T^(1 - omega), Pr = 1."""
    scattering_model = 'bgk-direct-gll'
    nalph = 5

    def load_parameters(self):
        cfg, vm = self.cfg, self.vm
        omega = cfg.getfloat('scattering-model', 'omega')
        muRef = cfg.getfloat('scattering-model', 'muRef')
        Tref = cfg.getfloat('scattering-model', 'Tref')
        t0 = vm.H0() / vm.u0()                           # time scale
        visc = muRef * (vm.T0() / Tref)**omega           # viscosity at T0
        p0 = vm.n0() * R0 / NA * vm.T0()                 # pressure scale
        self._prefactor = t0 * p0 / visc
        self._omega = omega
        self._Pr = 1.0

    def nu(self, rho, T):
        return self._prefactor * rho * T**(1 - self._omega)

    def perform_precomputation(self):
        dev = self.backend.device
        self.c0 = torch.as_tensor(self.vm.c0(), dtype=torch.float64, device=dev).contiguous()
        self.cw = float(self.vm.cw())
        self.fp64 = int(self.backend.fpdtype == torch.float64)

    # reference kernels ---------------------------------------------------
    def moment(self, f, U):
        """U[dof] <- (rho, rho u, E) of f[dof] (FP64)."""
        n = self.vm.vsize()
        _lib.check(_lib.lib().bdgfs_bgk_moments(f.data_ptr(), f.numel() // n, self.vm.Nv(),
                                                self.fp64, self.c0.data_ptr(), self.cw,
                                                U.data_ptr(), _lib.stream_ptr()),
                   'bdgfs_bgk_moments')

    def constructMaxwellian(self, U, M):
        n = self.vm.vsize()
        _lib.check(_lib.lib().bdgfs_bgk_maxwellian(U.data_ptr(), M.numel() // n, self.vm.Nv(),
                                                   self.fp64, self.c0.data_ptr(), M.data_ptr(),
                                                   _lib.stream_ptr()), 'bdgfs_bgk_maxwellian')

    ars_model = 0          # BDGFS_ARS_BGK

    def ars_stage(self, ndof, dt, ar, flags, ae, ai, f, fout, L, U, LU):
        """One fused ARS stage (bdgfs_ars_stage) over ndof distributions;
        f, L, U, LU are lists of tensors (None where the flags do not need
        them)."""
        p = lambda t: t.data_ptr() if t is not None else None
        a = _lib.ArsArgs(ndof=int(ndof),
                         Nv=self.vm.Nv(), fp64=self.fp64, c0=self.c0.data_ptr(), cw=self.cw,
                         prefac=self._prefactor, omega=self._omega, dt=float(dt), stage=ar,
                         flags=flags, model=self.ars_model, Pr=self._Pr)
        for j, x in enumerate(ae):
            a.ae[j] = x
        for j, x in enumerate(ai):
            a.ai[j] = x
        for j, t in enumerate(f):
            a.f[j] = p(t)
        a.fout = p(fout)
        for j, t in enumerate(L):
            a.L[j] = p(t)
        for j, t in enumerate(U):
            a.U[j] = p(t)
        for j, t in enumerate(LU):
            a.LU[j] = p(t)
        _lib.check(_lib.lib().bdgfs_ars_stage(C.byref(a), _lib.stream_ptr()), 'bdgfs_ars_stage')


    def bdf_step(self, ndof, dt, q, flags, a, g, b, f, fout, L, U, LU, Unew):
        """One fused IMEX-BDF step (bdgfs_bdf_step) over ndof distributions;
        f, L, U, LU are lists of q tensors, oldest first (None where the
        flags do not need them)."""
        p = lambda t: t.data_ptr() if t is not None else None
        x = _lib.BdfArgs(ndof=int(ndof), Nv=self.vm.Nv(), fp64=self.fp64, c0=self.c0.data_ptr(),
                         cw=self.cw, prefac=self._prefactor, omega=self._omega, dt=float(dt),
                         q=int(q), model=self.ars_model, Pr=self._Pr, b=float(b), flags=flags,
                         Unew=p(Unew), fout=p(fout))
        for j, v in enumerate(a):
            x.a[j] = v
        for j, v in enumerate(g):
            x.g[j] = v
        for j in range(q):
            x.f[j], x.L[j], x.U[j], x.LU[j] = p(f[j]), p(L[j]), p(U[j]), p(LU[j])
        _lib.check(_lib.lib().bdgfs_bdf_step(C.byref(x), _lib.stream_ptr()), 'bdgfs_bdf_step')


class ADGFSESBGKDirectGLLScatteringModel(ADGFSBGKDirectGLLScatteringModel):
    """ES-BGK relaxation nu (G[f] - f) towards the anisotropic Gaussian of
    the ES tensor T_ij = T/Pr d_ij + 2 (1 - 1/Pr)(P_ij/rho - u_i u_j),
    nu = prefac rho T^(1 - omega), prefac = t0 Pr p0 / visc, Pr from the
    .ini (default 2/3) (scattering.py: ADGFSESBGKDirectGLLScatteringModel;
    kernels/scattering/esbgk-direct-gll.mako)."""
    scattering_model = 'esbgk-direct-gll'
    nalph = 11
    ars_model = 1          # BDGFS_ARS_ESBGK

    def load_parameters(self):
        super().load_parameters()
        Pr = self.cfg.getfloat('scattering-model', 'Pr', 2.0 / 3.0)
        if not Pr > 0:
            raise ValueError('scattering-model: Pr must be positive')
        self._prefactor *= Pr
        self._Pr = Pr

    def moment(self, f, U):
        """U[dof] <- the 11 moments of f[dof] (FP64)."""
        n = self.vm.vsize()
        _lib.check(_lib.lib().bdgfs_esbgk_moments(f.data_ptr(), f.numel() // n, self.vm.Nv(),
                                                  self.fp64, self.c0.data_ptr(), self.cw,
                                                  U.data_ptr(), _lib.stream_ptr()),
                   'bdgfs_esbgk_moments')

    def constructMaxwellian(self, U, M):
        """M[dof] <- the ES Gaussian of U[dof] (momentNorm + cmaxwellian)."""
        n = self.vm.vsize()
        _lib.check(_lib.lib().bdgfs_esbgk_gaussian(U.data_ptr(), M.numel() // n, self.vm.Nv(),
                                                   self.fp64, self.c0.data_ptr(), self._Pr,
                                                   M.data_ptr(), _lib.stream_ptr()),
                   'bdgfs_esbgk_gaussian')


class ADGFSShakovDirectGLLScatteringModel(ADGFSBGKDirectGLLScatteringModel):
    """Shakov relaxation nu (S[f] - f), S = M (1 + 2 (1 - Pr)/5 (q.d)/(rho T^2)
    (2 |d|^2/T - 5)), d = c - u, q the heat flux; nu = prefac rho T^(1 - omega)
    with the BGK prefactor t0 p0 / visc; Pr from the .ini (default 2/3)
    (scattering.py: ADGFSShakovDirectGLLScatteringModel;
    kernels/scattering/shakov-direct-gll.mako)."""
    scattering_model = 'shakov-direct-gll'
    nalph = 14
    ars_model = 2          # BDGFS_ARS_SHAKOV

    def load_parameters(self):
        super().load_parameters()
        Pr = self.cfg.getfloat('scattering-model', 'Pr', 2.0 / 3.0)
        if not Pr > 0:
            raise ValueError('scattering-model: Pr must be positive')
        self._Pr = Pr

    def moment(self, f, U):
        """U[dof] <- the 14 moments of f[dof] (FP64)."""
        n = self.vm.vsize()
        _lib.check(_lib.lib().bdgfs_shakov_moments(f.data_ptr(), f.numel() // n, self.vm.Nv(),
                                                   self.fp64, self.c0.data_ptr(), self.cw,
                                                   U.data_ptr(), _lib.stream_ptr()),
                   'bdgfs_shakov_moments')

    def constructMaxwellian(self, U, M):
        """M[dof] <- the Shakov distribution of U[dof] (momentNorm + cmaxwellian)."""
        n = self.vm.vsize()
        _lib.check(_lib.lib().bdgfs_shakov_target(U.data_ptr(), M.numel() // n, self.vm.Nv(),
                                                  self.fp64, self.c0.data_ptr(), self._Pr,
                                                  M.data_ptr(), _lib.stream_ptr()),
                   'bdgfs_shakov_target')


class ADGFSSystem(DGFSSystem):
    """'adgfs' (system.py:17-121): FR advection plus BGK relaxation."""
    name = 'adgfs'
    scatteringcls = ADGFSScatteringModel

    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self.nreg_moms = None

    @property
    def ndof(self):
        return self.ele.neles * self.ele.nupts

    def get_nregs_moms(self, nreg_moms):
        """Moment banks [ndof][nalph] FP64 (system.py:31-52)."""
        if self.nreg_moms is not None and self.nreg_moms != nreg_moms:
            raise RuntimeError('moment registers already allocated with another count')
        if self.nreg_moms is None:
            dev = self.backend.device
            self.eles_scal_upts_inb_moms = [
                torch.zeros(self.ndof, self.sm.nalph, dtype=torch.float64, device=dev)
                for _ in range(nreg_moms)]
            self.nreg_moms = nreg_moms
            self.nalph = self.sm.nalph
        return list(range(nreg_moms))

    def _mom(self, i):
        return self.eles_scal_upts_inb_moms[i] if isinstance(i, int) else i

    def _ref(self, i):
        return self._bank(i) if isinstance(i, int) else i

    def collide(self, *args, **kwargs):
        raise RuntimeError('Not valid for asymptotic systems')

    # reference methods (system.py:62-121) --------------------------------
    def moment(self, t, finbank, momoutbank, fscratchbank=None):
        self.sm.moment(self._bank(finbank), self._mom(momoutbank))

    def constructMaxwellian(self, t, mominbank, Mcoeffbank, momscratchbank=None):
        self.sm.constructMaxwellian(self._mom(mominbank), self._bank(Mcoeffbank))

    def updateMomentARS(self, dt, *args):
        """args = _A[ar][0:ar], A[ar][1:ar+1], LU_0..LU_{ar-1}, U_0..U_ar."""
        ar = (len(args) - 1) // 4
        if len(args) != 4 * ar + 1:
            raise ValueError('updateMomentARS: inconsistent number of arguments')
        ae, ai = args[:ar], args[ar:2 * ar]
        LU = [self._mom(x) for x in args[2 * ar:3 * ar]]
        U = [self._mom(x) for x in args[3 * ar:]]
        self.sm.ars_stage(self.ndof, dt, ar, ARS_MOMU, ae, ai, [None] * ar, None, [None] * ar, U,
                          LU)

    def updateDistARS(self, dt, *args):
        """args = _A[ar][0:ar], A[ar][1:ar+1], L_0..L_{ar-1}, U_0..U_ar,
        M_1..M_ar (unused: the Maxwellians are rebuilt from U on the fly),
        f_0..f_ar (f_ar is the output)."""
        q = (len(args) - 2) // 6
        if len(args) != 6 * q + 2:
            raise ValueError('updateDistARS: inconsistent number of arguments')
        ae, ai = args[:q], args[q:2 * q]
        L = [self._ref(x) for x in args[2 * q:3 * q]]
        U = [self._mom(x) for x in args[3 * q:4 * q + 1]]
        F = [self._ref(x) for x in args[5 * q + 1:]]
        self.sm.ars_stage(self.ndof, dt, q, ARS_DIST, ae, ai, F[:q], F[q], L, U, [None] * q)

    def updateMomentBDF(self, dt, *args):
        """args = a_0, U_0, g_0, LU_0, ..., a_{q-1}, U_{q-1}, g_{q-1},
        LU_{q-1}, a_q, U, b (system.py:108-111, updateMom{q}_BDF)."""
        q = (len(args) - 3) // 4
        if len(args) != 4 * q + 3:
            raise ValueError('updateMomentBDF: inconsistent number of arguments')
        a = [args[4 * i] for i in range(q)] + [args[4 * q]]
        g = [args[4 * i + 2] for i in range(q)]
        U = [self._mom(args[4 * i + 1]) for i in range(q)]
        LU = [self._mom(args[4 * i + 3]) for i in range(q)]
        self.sm.bdf_step(self.ndof, dt, q, BDF_MOMU, a, g, args[4 * q + 2], [None] * q, None,
                         [None] * q, U, LU, self._mom(args[4 * q + 1]))

    def updateDistBDF(self, dt, *args):
        """args = a_0, f_0, g_0, L_0, ..., b, M (unused: the target is rebuilt
        from U on the fly), a_q, U, f (system.py:113-121,
        updateDistribution{q}_BDF)."""
        q = (len(args) - 5) // 4
        if len(args) != 4 * q + 5:
            raise ValueError('updateDistBDF: inconsistent number of arguments')
        a = [args[4 * i] for i in range(q)] + [args[4 * q + 2]]
        g = [args[4 * i + 2] for i in range(q)]
        f = [self._ref(args[4 * i + 1]) for i in range(q)]
        L = [self._ref(args[4 * i + 3]) for i in range(q)]
        self.sm.bdf_step(self.ndof, dt, q, BDF_DIST, a, g, args[4 * q], f,
                         self._ref(args[4 * q + 4]), L, [None] * q, [None] * q,
                         self._mom(args[4 * q + 3]))

    def copy_dist(self, rdest, rsrc):
        self._ref(rdest).copy_(self._ref(rsrc))

    def copy_moms(self, rdest, rsrc):
        self._mom(rdest).copy_(self._mom(rsrc))

    def bdf_step(self, dt, q, flags, a, g, b, fbanks, foutbank, Lbanks, Umoms, LUmoms, Unew):
        self.sm.bdf_step(self.ndof, dt, q, flags, a, g, b, [self._bank(x) for x in fbanks],
                         self._bank(foutbank), [self._bank(x) for x in Lbanks],
                         [self._mom(m) for m in Umoms], [self._mom(m) for m in LUmoms],
                         self._mom(Unew))

    # fused stage used by the project's ARS steppers ------------------------
    def ars_stage(self, dt, ar, flags, ae, ai, fbanks, foutbank, Lbanks, Umoms, LUmoms):
        self.sm.ars_stage(self.ndof, dt, ar, flags, ae, ai, [self._bank(b) for b in fbanks],
                          self._bank(foutbank), [self._bank(b) for b in Lbanks],
                          [self._mom(m) for m in Umoms], [self._mom(m) for m in LUmoms])
