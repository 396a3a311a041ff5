"""The DGFS system: state banks, FR operators, boundary conditions and Q.

Drop-in for ``DGFSSystem`` (frfs/solvers/dgfs/system.py:17-231, name
'dgfs') on the path the steppers use: ``rhs``, ``updatebc``, ``collide``,
``invmass`` and the kernel registry ``_kernels`` keyed like
``BaseSystem._gen_kernels`` (frfs/solvers/base/system.py:167-176).

Differences of layout, not of meaning:
* the state bank of one element type is a device tensor
  ``[neles][nupts][Nv^3]`` (velocity contiguous) instead of the
  reference's AoSoA ``(nupts, Nv^3, neles)``;
* every velocity is advected in one pass, so ``batch``/``varidx`` are
  accepted and ignored (the reference's NvBatchSize loop and its
  copy_to/from_reg kernels disappear);
* ('eles','tdisf'), ('eles','tdivtpcorf'), ('iint','comm_flux'),
  ('bcint','comm_flux'), ('eles','tdivtconf') and ('eles','negdivconf')
  are fused into one launch of ``bdgfs_fr_rhs``; in the registry the first
  five resolve to no-ops and ``('eles','negdivconf')`` runs the fused
  kernel, so a caller that runs them in the reference's order gets the
  reference's result.
"""
import numpy as np
import torch

from . import _lib
from .initcond import DGFSInitCondition, DGFSMaxwellianInitCondition
from .mesh import ElementGeometry
from .scattering import DGFSScatteringModel
from .util import npeval, subclass_where
from .velocitymesh import DGFSVelocityMesh


class DGFSElements:
    """Device-resident operators and metrics of one element type."""

    def __init__(self, backend, geo, vm):
        self.be, self.geo, self.vm = backend, geo, vm
        shp = geo.shape
        dt = backend.fpdtype
        c = lambda a: backend.const(np.ascontiguousarray(a), dtype=dt)
        self.neles, self.nupts, self.nfpts, self.ndims = geo.neles, geo.nupts, geo.nfpts, geo.ndims
        m0 = np.asarray(shp.opmat('M0'))
        self.m0 = c(m0)
        # flux points on solution points (every row of M0 a unit vector, as
        # with GLL points): face values are rows of the state itself
        unit = np.all(np.count_nonzero(m0, axis=1) == 1) and np.all(m0.max(axis=1) == 1.0)
        self.fsel = (backend.const(np.argmax(m0, axis=1), dtype=torch.int32) if unit else None)
        self.tensor = self._tensor_form(shp, m0, c) if unit else None
        self.dcorr = c(shp.opmat('M1 - M3*M2'))
        self.m3 = c(shp.opmat('M3'))
        self.minv = c(shp.opmat('M12'))
        self.smats = c(geo.smats)
        self.rcpdjac = c(geo.rcpdjac)
        self.pnorm = c(geo.norm_pnorm)
        self.magn = c(geo.mag_pnorm)
        self.nbr = backend.const(geo.nbr, dtype=torch.int32)
        self.c0 = c(vm.c0())
        self.struct = _lib.FrEles(
            ndims=geo.ndims, nupts=geo.nupts, nfpts=geo.nfpts, neles=geo.neles,
            nv=vm.vsize(), Nv=vm.Nv(), fp64=int(dt == torch.float64),
            m0=self.m0.data_ptr(), dcorr=self.dcorr.data_ptr(), m3=self.m3.data_ptr(),
            smats=self.smats.data_ptr(), rcpdjac=self.rcpdjac.data_ptr(),
            pnorm=self.pnorm.data_ptr(), magn=self.magn.data_ptr(),
            nbr=self.nbr.data_ptr(), c0=self.c0.data_ptr())

    def _tensor_form(self, shp, m0, c):
        """bdgfs_fr_tensor of the shape when its solution points form a
        tensor product (p per line, first reference coordinate fastest), M1
        acts along the lines and M2 selects one column per flux point; else
        None."""
        nd, nu, nf = self.ndims, self.nupts, self.nfpts
        p = int(round(nu ** (1.0 / nd)))
        if p ** nd != nu or not 2 <= p <= 4:
            return None
        m1, m2 = np.asarray(shp.opmat('M1')), np.asarray(shp.opmat('M2'))
        fsel = np.argmax(m0, axis=1)
        line = np.zeros((nd, nu, 4))
        for d in range(nd):
            st = p ** d
            for j in range(nu):
                col = m1[:, d * nu + j].copy()
                base = j - ((j // st) % p) * st
                for t in range(p):
                    line[d, j, t] = col[base + t * st]
                    col[base + t * st] = 0.0
                if np.any(col != 0.0):
                    return None
        fdim = np.zeros(nf, dtype=np.int32)
        fsgn = np.zeros(nf)
        for f in range(nf):
            nz = np.flatnonzero(m2[f])
            if len(nz) != 1 or nz[0] % nu != fsel[f]:
                return None
            fdim[f], fsgn[f] = nz[0] // nu, m2[f, nz[0]]
        self.tp_fdim = self.be.const(fdim, dtype=torch.int32)
        self.tp_fsgn = c(fsgn)
        self.tp_m1line = c(line)
        self.tp_fsel = self.be.const(fsel, dtype=torch.int32)
        return _lib.FrTensor(fsel=self.tp_fsel.data_ptr(), fdim=self.tp_fdim.data_ptr(),
                             fsgn=self.tp_fsgn.data_ptr(), m1line=self.tp_m1line.data_ptr(), p=p)

    def ploc_at_np(self, name):
        return {'upts': self.geo.plocupts, 'fpts': self.geo.plocfpts}[name]


class DGFSBCInters:
    """One boundary condition of the 'dgfs' system, selected by its .ini
    ``type`` (frfs/solvers/dgfs/inters.py:115-480): its kernel kind and its
    rows (U[3], f_w[nv]) -- one row, or one per face point -- for the face
    points ``pts`` (indices into geo.wall_fpts) of the boundary."""
    type = None
    kind = _lib.BC_DIFFUSE
    oracle_type = None

    def __init__(self, backend, cfg, vm, sect, geo, pts):
        self.be, self.cfg, self.vm, self.sect, self.geo, self.pts = backend, cfg, vm, sect, geo, pts
        self.load()

    def load(self):
        self.rows = [(np.zeros(3), np.zeros(self.vm.vsize()))]

    def point_rows(self):
        return np.zeros(len(self.pts), dtype=np.int64)

    def kind_of(self):
        return self.kind

    def _maxwellian(self):
        bc = DGFSMaxwellianInitCondition(self.be, self.cfg, self.vm, self.sect)
        return bc.unondim()[:, 0], bc.get_init_vals()


class DGFSWallDiffuseBCInters(DGFSBCInters):
    """'dgfs-wall-diffuse' (inters.py:175-229): u_R = f_w (-bc0/bc1) where
    (c - U_w).n < 0, with the wall Maxwellian f_w of the section."""
    type = 'dgfs-wall-diffuse'

    def load(self):
        self.rows = [self._maxwellian()]


class DGFSWallDiffuseCylBCInters(DGFSBCInters):
    """'dgfs-wall-diffuse-cyl' (inters.py:446-500, bcs/dgfs-wall-diffuse-cyl
    .mako): the diffuse wall with U_w and T_w given as expressions of the
    face-point location (x, y, z and the [constants]); f_w = exp(-|c -
    U_w|^2/T_w) per face point (its normalisation cancels in bc0/bc1)."""
    type = 'dgfs-wall-diffuse-cyl'
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
        cv = vm.cv()
        self.rows = []
        for i in range(len(self.pts)):
            d2 = np.sum((cv - U[:, i:i + 1])**2, axis=0)
            self.rows.append((U[:, i].copy(), np.exp(-d2 / T[i])))

    def point_rows(self):
        return np.arange(len(self.pts), dtype=np.int64)


class DGFSWallSpecularBCInters(DGFSBCInters):
    """'dgfs-wall-specular' (inters.py:232-311): u_R(c) = u_L(c - 2 (c.n) n).
    The kernels mirror one velocity index, so the wall must be normal to a
    coordinate axis (every wall of a structured box mesh is)."""
    type = 'dgfs-wall-specular'

    def kind_of(self):
        geo = self.geo
        axes = set()
        for w in self.pts:
            e, f = geo.wall_fpts[w]
            n = np.asarray(geo.norm_pnorm[e, f], dtype=np.float64)
            a = int(np.argmax(np.abs(n)))
            if not np.allclose(np.delete(n, a), 0.0, atol=1e-12):
                raise ValueError(f'{self.sect}: specular walls must be normal to a coordinate axis')
            axes.add(a)
        if len(axes) > 1:
            raise ValueError(f'{self.sect}: a specular boundary must be one plane')
        c0 = np.asarray(self.vm.c0())
        if not np.allclose(c0[::-1], -c0, rtol=0, atol=1e-12 * np.abs(c0).max()):
            raise ValueError('specular walls need a velocity grid symmetric about 0')
        return _lib.BC_SPECULAR_X + (axes.pop() if axes else 0)


class DGFSInletBCInters(DGFSBCInters):
    """'dgfs-inlet' (inters.py:312-351): u_R = f_in where (c - U_in).n < 0."""
    type = 'dgfs-inlet'
    kind = _lib.BC_INLET

    def load(self):
        self.rows = [self._maxwellian()]


class DGFSInletNormalShockBCInters(DGFSBCInters):
    """'dgfs-inlet-normalshock' (inters.py:353-384): u_R = f_in where c.n < 0."""
    type = 'dgfs-inlet-normalshock'
    kind = _lib.BC_INLET

    def load(self):
        self.rows = [(np.zeros(3), self._maxwellian()[1])]


class DGFSOutletBCInters(DGFSBCInters):
    """'dgfs-outlet' (inters.py:386-414): u_R = u_L."""
    type = 'dgfs-outlet'
    kind = _lib.BC_OUTLET


class DGFSVanishBCInters(DGFSBCInters):
    """'dgfs-vanish' (inters.py:416-444): u_R = 0 where c.n < 0."""
    type = 'dgfs-vanish'
    kind = _lib.BC_INLET


class DGFSBoundaries:
    """Every boundary face point of the system in one bdgfs_fr_walls: the
    rows of all boundary conditions, each face point's row and each row's
    kind."""

    def __init__(self, backend, geo, vm, cfg, names):
        self.be = backend
        dt = backend.fpdtype
        nw = len(geo.wall_fpts)
        self.nwall = nw
        bcs = []
        for bid, name in enumerate(names):
            sect = f'soln-bcs-{name}'
            bctype = cfg.get(sect, 'type')
            try:
                cls = subclass_where(DGFSBCInters, type=bctype)
            except KeyError:
                raise ValueError(f'unsupported boundary condition {bctype} on {name}') from None
            pts = np.nonzero(np.asarray(geo.wall_bcid) == bid)[0]
            bcs.append(cls(backend, cfg, vm, sect, geo, pts))
        self.bcs = bcs
        rows, kinds, types = [], [], []
        bcid = np.zeros(nw, dtype=np.int64)
        for bc in bcs:
            base = len(rows)
            k = bc.kind_of()
            for r in bc.rows:
                rows.append(r)
                kinds.append(k)
                types.append(bc.oracle_type or bc.type)
            bcid[bc.pts] = base + bc.point_rows()
        if not rows:
            rows, kinds, types = [(np.zeros(3), np.zeros(vm.vsize()))], [0], ['dgfs-wall-diffuse']
        self.types = types
        self.row_of_point = bcid
        self.fw = backend.const(np.stack([r[1] for r in rows]), dtype=dt)
        self.uwall = backend.const(np.stack([r[0] for r in rows]), dtype=dt)
        self.fpt = backend.const(geo.wall_fpts.reshape(-1, 2) if nw else np.zeros((1, 2)),
                                 dtype=torch.int32)
        self.bcid = backend.const(bcid if nw else np.zeros(1), dtype=torch.int32)
        self.kind = backend.const(np.array(kinds), dtype=torch.int32)
        self.kinds_used = int(sum(1 << k for k in set(kinds)))
        self.bcv = backend.zeros(max(nw, 1), 2)
        self.struct = _lib.FrWall(nwall=nw, nbc=len(rows), fpt=self.fpt.data_ptr(),
                                  bcid=self.bcid.data_ptr(), uwall=self.uwall.data_ptr(),
                                  fw=self.fw.data_ptr(), bcv=self.bcv.data_ptr(),
                                  cw=float(vm.cw()), kind=self.kind.data_ptr(),
                                  kinds_used=self.kinds_used)

    @property
    def has_diffuse(self):
        return bool(self.kinds_used & (1 << _lib.BC_DIFFUSE)) and self.nwall > 0

    def oracle_walls(self):
        """(rows as (U, f_w, type), row of each face point) for oracle.fr."""
        rows = [(self.uwall[i].double().cpu().numpy(), self.fw[i].double().cpu().numpy(), t)
                for i, t in enumerate(self.types)]
        return rows, self.row_of_point


class DGFSSystem:
    name = 'dgfs'
    elementscls = DGFSElements
    velocitymeshcls = DGFSVelocityMesh
    scatteringcls = DGFSScatteringModel

    def __init__(self, backend, mesh, cfg, nreg=3, initsoln=None, partition=None,
                 transport=None):
        """partition = (parts, rank): this system owns the elements
        parts[rank] of the mesh (frfs_b200.partition); transport exchanges
        the face values of neighbouring parts after disu."""
        self.backend, self.cfg, self.mesh = backend, cfg, mesh
        self.vm = self.velocitymeshcls(backend, cfg)
        order = cfg.getint('solver', 'order')
        self.geo = ElementGeometry(mesh, order)
        self.domain = None
        if partition is not None:
            from .partition import LocalDomain
            self.domain = self.geo = LocalDomain(self.geo, *partition)
        self.transport = transport
        self.ele = self.elementscls(backend, self.geo, self.vm)
        self.ndims = self.geo.ndims
        # boundary conditions by the .ini type of every named boundary
        self.walls = DGFSBoundaries(backend, self.geo, self.vm, cfg, self.geo.wall_names)
        # time-step estimate (system.py:50-66)
        advmax = self.vm.L()
        self.unitCFLdt = np.sqrt(np.min(self.geo.djac)) / advmax / self.ndims
        # collision model by name (system.py:68-72)
        smn = cfg.get('scattering-model', 'type')
        self.sm = subclass_where(self.scatteringcls, scattering_model=smn)(backend, cfg, self.vm)
        # register banks [neles][nupts][Nv^3]
        E, U, nv = self.ele.neles, self.ele.nupts, self.vm.vsize()
        self.eles_scal_upts_inb_full = [backend.empty(E, U, nv) for _ in range(nreg)]
        nghost = self.domain.nghost if self.domain is not None else 0
        self._uf_rows = backend.empty(E * self.ele.nfpts + nghost, nv)
        self._uf = self._uf_rows[:E * self.ele.nfpts].view(E, self.ele.nfpts, nv)
        self._send_rows = {}
        if self.domain is not None:
            for r, rows in self.domain.send.items():
                self._send_rows[r] = torch.as_tensor(rows, dtype=torch.int64,
                                                     device=backend.device)
        if initsoln is not None:
            self.eles_scal_upts_inb_full[0].copy_(torch.as_tensor(initsoln).to(
                self.eles_scal_upts_inb_full[0]))
        else:
            icn = cfg.get('soln-ics', 'type')
            ic = subclass_where(DGFSInitCondition, model=icn)(backend, cfg, self.vm, 'soln-ics')
            if hasattr(ic, 'apply_init_vals'):
                ic.apply_init_vals(self.eles_scal_upts_inb_full[0], self.geo.plocupts)
            else:
                f0 = backend.const(ic.get_init_vals())
                self.eles_scal_upts_inb_full[0].copy_(f0.expand(E, U, nv))
        self._gen_kernels()

    # -- kernel registry ------------------------------------------------
    def _gen_kernels(self):
        noop = lambda **kw: None
        self._kernels = {
            ('eles', 'disu'): self._disu,
            ('eles', 'tdisf'): noop, ('eles', 'tdivtpcorf'): noop,
            ('iint', 'comm_flux'): noop, ('bcint', 'comm_flux'): noop,
            ('eles', 'tdivtconf'): noop,
            ('eles', 'negdivconf'): self._fused_rhs,
            ('bcint', 'update_bc'): self._update_bc,
        }
        self._active = (0, 1)

    def _bank(self, i):
        return self.eles_scal_upts_inb_full[i]

    def _disu(self, **kw):
        u = self._bank(self._active[0])
        _lib.check(_lib.lib().bdgfs_fr_disu(_lib.ref(self.ele.struct), _lib.ptr(u),
                                            _lib.ptr(self._uf), _lib.stream_ptr()),
                   'bdgfs_fr_disu')

    def _update_bc(self, **kw):
        _lib.check(_lib.lib().bdgfs_fr_bc_update(_lib.ref(self.ele.struct),
                                                 _lib.ref(self.walls.struct),
                                                 _lib.ptr(self._uf), _lib.stream_ptr()),
                   'bdgfs_fr_bc_update')

    def _exchange(self):
        """Complete the halo exchange of the face values: the one posted by
        ``advect_begin`` when the transport is asynchronous, else a blocking
        one now."""
        pending, self._pending = getattr(self, '_pending', None), None
        if pending is not None:
            self.transport.wait(pending)
        elif self.transport is not None:
            self.transport.exchange(self)

    def _fused_rhs(self, a=0.0, b=1.0, x1=None, c1=0.0, x2=None, c2=0.0, out=None, **kw):
        u = self._bank(self._active[0])
        out = self._bank(self._active[1]) if out is None else out
        L = _lib.lib()
        xs = (float(a), float(b), x1.data_ptr() if x1 is not None else None, float(c1),
              x2.data_ptr() if x2 is not None else None, float(c2), _lib.stream_ptr())
        if self.ele.tensor is not None and self.ele.struct.engine == 0:
            rc = L.bdgfs_fr_rhs_tensor(_lib.ref(self.ele.struct), _lib.ref(self.walls.struct),
                                       _lib.ref(self.ele.tensor), u.data_ptr(),
                                       self._uf_rows.data_ptr(), out.data_ptr(), *xs)
            _lib.check(rc, 'bdgfs_fr_rhs_tensor')
            return
        rc = L.bdgfs_fr_rhs(_lib.ref(self.ele.struct), _lib.ref(self.walls.struct),
                            u.data_ptr(), self._uf_rows.data_ptr(), out.data_ptr(), *xs)
        _lib.check(rc, 'bdgfs_fr_rhs')

    # -- reference system methods ----------------------------------------
    def rhs(self, t, uinbank, foutbank, batch=None, varidx=None):
        """foutbank <- -div F(uinbank) (system.py:140-177); uses the bc0/bc1
        left by the last ``updatebc``."""
        self._active = (uinbank, foutbank)
        k = self._kernels
        k['eles', 'disu']()
        self._exchange()
        for name in (('eles', 'tdisf'), ('eles', 'tdivtpcorf'), ('iint', 'comm_flux'),
                     ('bcint', 'comm_flux'), ('eles', 'tdivtconf')):
            k[name](t=t, varidx=varidx)
        k['eles', 'negdivconf'](t=t)

    def updatebc(self, t, uinbank, foutbank, batch=None, varidx=None):
        """disu + update_bc over all velocities (system.py:180-196)."""
        self._active = (uinbank, foutbank)
        self._kernels['eles', 'disu']()
        self._kernels['bcint', 'update_bc'](t=t)

    def collide(self, t, uinbank, foutbank):
        """foutbank <- Q(uinbank) for every DOF in one launch (system.py:199-218)."""
        self.sm.collide(self._bank(uinbank), self._bank(foutbank))

    def invmass(self, uinbank, foutbank):
        """foutbank <- M12 uinbank per element, M12 the inverse mass matrix
        (system.py:221-231, kernel elements.py:161-164).  The DGFS steppers
        do not call it; the banks must differ."""
        u, out = self._bank(uinbank), self._bank(foutbank)
        _lib.check(_lib.lib().bdgfs_fr_invmass(_lib.ref(self.ele.struct), _lib.ptr(self.ele.minv),
                                               _lib.ptr(u), _lib.ptr(out), _lib.stream_ptr()),
                   'bdgfs_fr_invmass')

    # -- fused stage used by the steppers ---------------------------------
    def advect_combine(self, t, uinbank, outbank, a, b, x1=None, c1=0.0, x2=None, c2=0.0):
        """out = a*u + b*L(u) + c1*x1 + c2*x2 (bc update included)."""
        self.advect_begin(uinbank, outbank)
        self.advect_end(t, a, b, x1, c1, x2, c2)

    def _gathers(self):
        """Face values straight from the state (bdgfs_fr_*_gather): GLL-type
        flux points, one part (no halo rows) and out distinct from u."""
        return (self.ele.fsel is not None and self.domain is None
                and self._active[0] != self._active[1])

    def advect_begin(self, uinbank, outbank):
        """First half of a stage: face values of the stage input, and (with
        an asynchronous transport) the halo exchange posted, to be completed
        by ``advect_end``; work queued in between overlaps it."""
        self._active = (uinbank, outbank)
        if not self._gathers():
            self._disu()
            if self.transport is not None and hasattr(self.transport, 'start'):
                self._pending = self.transport.start(self)

    def advect_end(self, t, a, b, x1=None, c1=0.0, x2=None, c2=0.0):
        """Second half: halo exchange, wall update, fused FR + combination."""
        x1 = self._bank(x1) if x1 is not None else None
        x2 = self._bank(x2) if x2 is not None else None
        if self._gathers():
            L = _lib.lib()
            u, out = self._bank(self._active[0]), self._bank(self._active[1])
            fsel = self.ele.fsel.data_ptr()
            if self.walls.has_diffuse:
                _lib.check(L.bdgfs_fr_bc_update_gather(_lib.ref(self.ele.struct),
                                                       _lib.ref(self.walls.struct), fsel,
                                                       u.data_ptr(), _lib.stream_ptr()),
                           'bdgfs_fr_bc_update_gather')
            xs = (x1.data_ptr() if x1 is not None else None, float(c1),
                  x2.data_ptr() if x2 is not None else None, float(c2), _lib.stream_ptr())
            if self.ele.tensor is not None:
                _lib.check(L.bdgfs_fr_rhs_tensor(_lib.ref(self.ele.struct),
                                                 _lib.ref(self.walls.struct),
                                                 _lib.ref(self.ele.tensor), u.data_ptr(), None,
                                                 out.data_ptr(), float(a), float(b), *xs),
                           'bdgfs_fr_rhs_tensor')
            else:
                _lib.check(L.bdgfs_fr_rhs_gather(_lib.ref(self.ele.struct),
                                                 _lib.ref(self.walls.struct), fsel, u.data_ptr(),
                                                 out.data_ptr(), float(a), float(b), *xs),
                           'bdgfs_fr_rhs_gather')
            return
        self._exchange()
        if self.walls.has_diffuse:
            self._update_bc()
        self._fused_rhs(a=a, b=b, x1=x1, c1=c1, x2=x2, c2=c2)

    # -- diagnostics ------------------------------------------------------
    def moments(self, bank):
        """Non-dimensional rho, U, T, q, P per DOF (FP64 on the GPU)."""
        return macroscopic(self._bank(bank), self.vm)

    def residual(self, a, b):
        out = torch.zeros(2, dtype=torch.float64, device=self.backend.device)
        x, y = self._bank(a), self._bank(b)
        L = _lib.lib()
        _lib.check(L.bdgfs_residual(x.data_ptr(), y.data_ptr(), x.numel(),
                                    int(x.dtype == torch.float64), out.data_ptr(),
                                    _lib.stream_ptr()), 'bdgfs_residual')
        return out


def raw_moments(f, vm):
    """FP64 raw moments [ndof][13] (bdgfs_moments)."""
    n3 = vm.vsize()
    f2 = f.reshape(-1, n3)
    out = torch.empty(f2.shape[0], 13, dtype=torch.float64, device=f.device)
    c0 = torch.as_tensor(vm.c0(), dtype=torch.float64, device=f.device)
    L = _lib.lib()
    _lib.check(L.bdgfs_moments(f2.data_ptr(), f2.shape[0], vm.Nv(), int(f.dtype == torch.float64),
                               c0.data_ptr(), float(vm.cw()), out.data_ptr(), _lib.stream_ptr()),
               'bdgfs_moments')
    return out


def macroscopic(f, vm):
    """rho, U[3], T, q[3], P[6] per DOF from the FP64 raw moments, with the
    definitions of frfs/plugins/dgfsmomwriterstd.py:151-213 (3-D, mr = 1)."""
    m = raw_moments(f, vm)
    rho = m[:, 0]
    U = m[:, 1:4] / rho[:, None]
    Sxx = m[:, 4:10]                                   # xx xy xz yy yz zz
    ij = ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))
    P = torch.stack([2.0 * (Sxx[:, k] - rho * U[:, a] * U[:, b]) for k, (a, b) in enumerate(ij)], 1)
    tr = (P[:, 0] + P[:, 3] + P[:, 5]) / 2.0          # sum f |c-U|^2 cw
    T = tr * (2.0 / 3.0) / rho
    # q_a = sum f |c-U|^2 (c-U)_a cw from raw moments
    S = torch.zeros(m.shape[0], 3, 3, dtype=torch.float64, device=m.device)
    for k, (a, b) in enumerate(ij):
        S[:, a, b] = Sxx[:, k]
        S[:, b, a] = Sxx[:, k]
    trS = S[:, 0, 0] + S[:, 1, 1] + S[:, 2, 2]
    U2 = (U * U).sum(1)
    m1 = m[:, 1:4]
    # |c-U|^2 (c-U) expanded: M3 - tr(S) U - 2 S U + 2 U (U.m1) + |U|^2 m1 - rho |U|^2 U
    q = (m[:, 10:13] - trS[:, None] * U - 2.0 * torch.einsum('nab,nb->na', S, U)
         + 2.0 * U * (U * m1).sum(1, keepdim=True) + U2[:, None] * m1
         - (rho * U2)[:, None] * U)
    return rho, U, T, q, P
