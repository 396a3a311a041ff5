"""DGFS time integrators: controller x stepper, CUDA-graph replay.

Mirrors frfs/integrators: ``get_integrator`` (integrators/__init__.py:9-44)
composes a controller ('none', integrators/std/controllers.py:54-73) with a
stepper chosen by ``[solver-time-integrator] scheme``:

* 'dgfs-euler'   (steppers.py:20-99):  u <- u + dt (L + Q)(u)
* 'dgfs-tvd-rk2' (steppers.py:103-225): u1 = u + dt (L+Q)(u);
                 u <- u/2 + u1/2 + dt/2 (L+Q)(u1)
* 'adgfs-ars-111/222/443' (steppers.py:489-670): IMEX Runge-Kutta with the
                 FR advection explicit and the BGK relaxation implicit
                 ('adgfs' system, frfs_b200.adgfs)
* 'adgfs-bdf-1/2/3' (steppers.py:675-860): IMEX backward differences
                 (BDF-1 is ARS-111)
* 'dgfsbi-euler', 'dgfsbi-tvd-rk2' (steppers.py:229-486): the same per
                 species of the 'dgfsbi' gas-mixture system, the species
                 coupled by the mixture collision operator

Each stage is one ``collide`` launch (all DOFs) plus the disu / bc-update /
fused-rhs launches; the register banks are those of the reference (r0, r1,
r2) and the result lands back in r0, so one step is captured once as a CUDA
graph and replayed.  Per-step hooks: NaN check (plugins/nancheck.py) through
a device status word, FP64 residual (plugins/dgfsresidualstd.py).
"""
import torch

from . import _lib


class BaseDGFSStepper:
    stepper_name = None
    nregs = 2

    def __init__(self, backend, system, cfg):
        self.backend, self.system, self.cfg = backend, system, cfg
        sect = 'solver-time-integrator'
        self.tstart = cfg.getfloat(sect, 'tstart', 0.0)
        self.tend = cfg.getfloat(sect, 'tend')
        self._dt = cfg.getfloat(sect, 'dt')
        self.tcurr = self.tstart
        self.nacptsteps = 0
        self._idxcurr = 0
        self._graph = None
        self.use_graph = cfg.getbool(sect, 'cuda-graph', True)
        self.nancheck_nsteps = cfg.getint('soln-plugin-nancheck', 'nsteps', 0)
        self.resid_nsteps = cfg.getint('soln-plugin-dgfsresidualstd', 'nsteps', 0)
        self._status = torch.zeros(1, dtype=torch.int32, device=backend.device)
        self.residuals = []

    @property
    def soln(self):
        return self.system.eles_scal_upts_inb_full[self._idxcurr]

    def _step_kernels(self, t, dt):
        raise NotImplementedError

    def step(self, t, dt):
        if not self.use_graph:
            self._step_kernels(t, dt)
            return
        if self._graph is None or self._graph_dt != dt:
            # warm-up launch on a side stream (sets kernel attributes), then capture
            s = torch.cuda.Stream(device=self.backend.device)
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                self._step_kernels(t, dt)
            torch.cuda.current_stream().wait_stream(s)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._step_kernels(t, dt)
            self._graph, self._graph_dt = g, dt
            # the warm-up advanced the state: undo by replaying nothing -- the
            # warm-up step is counted as a real step
            self._warm_stepped = True
            return
        self._graph.replay()

    def advance_to(self, t):
        while self.tcurr < t - 1e-12 * max(1.0, abs(t)):
            dt = min(self._dt, t - self.tcurr)
            need_resid = self.resid_nsteps and (self.nacptsteps + 1) % self.resid_nsteps == 0
            if need_resid:
                prev = self.soln.clone()
            self.step(self.tcurr, dt)
            self.tcurr += dt
            self.nacptsteps += 1
            if need_resid:
                self.residuals.append((self.tcurr, self._residual(prev)))
            if self.nancheck_nsteps and self.nacptsteps % self.nancheck_nsteps == 0:
                self.nancheck()
        return self.tcurr

    def run(self):
        return self.advance_to(self.tend)

    def _residual(self, prev):
        out = torch.zeros(2, dtype=torch.float64, device=self.backend.device)
        cur = self.soln
        _lib.check(_lib.lib().bdgfs_residual(cur.data_ptr(), prev.data_ptr(), cur.numel(),
                                             int(cur.dtype == torch.float64), out.data_ptr(),
                                             _lib.stream_ptr()), 'bdgfs_residual')
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
            dist.all_reduce(out)                   # partitioned state: global norms
        o = out.cpu()
        return float((o[0] / o[1]).sqrt())

    def nancheck(self):
        """Raise if the state holds NaN/Inf (plugins/nancheck.py:17-22)."""
        self._status.zero_()
        u = self.soln
        _lib.check(_lib.lib().bdgfs_status_check(u.data_ptr(), u.numel(),
                                                 int(u.dtype == torch.float64),
                                                 self._status.data_ptr(), _lib.stream_ptr()),
                   'bdgfs_status_check')
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
            dist.all_reduce(self._status, op=dist.ReduceOp.MAX)
        if int(self._status.item()):
            raise RuntimeError(f'NaNs detected at t = {self.tcurr}')


class StdEulerDGFSStepper(BaseDGFSStepper):
    stepper_name = 'dgfs-euler'
    nregs = 2
    order = 1

    def _step_kernels(self, t, dt):
        s = self.system
        s.advect_begin(0, 0)                                 # face values (+ halo posted)
        s.collide(t, 0, 1)                                   # r1 = Q(r0)
        s.advect_end(t, a=1.0, b=dt, x1=1, c1=dt)            # r0 += dt (L + Q)


class StdTVDRK2DGFSStepper(BaseDGFSStepper):
    stepper_name = 'dgfs-tvd-rk2'
    nregs = 3
    order = 2

    def _step_kernels(self, t, dt):
        s = self.system
        # each stage: face values first (their halo exchange, when the mesh is
        # partitioned, overlaps the collision launch), then Q, then the
        # fused FR residual + combination
        s.advect_begin(0, 1)
        s.collide(t, 0, 1)                                        # r1 = Q(r0)
        s.advect_end(t, a=1.0, b=dt, x1=1, c1=dt)                 # r1 = r0 + dt (L+Q)(r0)
        s.advect_begin(1, 0)
        s.collide(t + dt, 1, 2)                                   # r2 = Q(r1)
        s.advect_end(t + dt, a=0.5, b=0.5 * dt,                   # r0 = r0/2 + r1/2
                     x1=2, c1=0.5 * dt, x2=0, c2=0.5)             #      + dt/2 (L+Q)(r1)


class _DGFSBiStepperMixin:
    """The 'dgfsbi' system's state is one bank per species; the residual is
    one value per species, ||f_p - f_p,prev|| / ||f_p,prev|| over all ranks
    (plugins/dgfsresidualbi.py:33-80), and the NaN check covers every
    species."""

    def __init__(self, backend, system, cfg):
        super().__init__(backend, system, cfg)
        self.resid_nsteps = cfg.getint('soln-plugin-dgfsresidualbi', 'nsteps', self.resid_nsteps)

    @property
    def soln(self):
        return [sp.eles_scal_upts_inb_full[self._idxcurr] for sp in self.system.species]

    def _residual(self, prev):
        cur = self.soln
        out = torch.zeros(len(cur), 2, dtype=torch.float64, device=self.backend.device)
        for p, (c, old) in enumerate(zip(cur, prev)):
            _lib.check(_lib.lib().bdgfs_residual(c.data_ptr(), old.data_ptr(), c.numel(),
                                                 int(c.dtype == torch.float64), out[p].data_ptr(),
                                                 _lib.stream_ptr()), 'bdgfs_residual')
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
            dist.all_reduce(out)                   # partitioned state: global norms
        o = out.cpu()
        return [float(v) for v in (o[:, 0] / o[:, 1]).sqrt()]

    def advance_to(self, t):
        while self.tcurr < t - 1e-12 * max(1.0, abs(t)):
            dt = min(self._dt, t - self.tcurr)
            need_resid = self.resid_nsteps and (self.nacptsteps + 1) % self.resid_nsteps == 0
            if need_resid:
                prev = [u.clone() for u in self.soln]
            self.step(self.tcurr, dt)
            self.tcurr += dt
            self.nacptsteps += 1
            if need_resid:
                self.residuals.append((self.tcurr, self._residual(prev)))
            if self.nancheck_nsteps and self.nacptsteps % self.nancheck_nsteps == 0:
                self.nancheck()
        return self.tcurr

    def nancheck(self):
        """Raise if any species' state holds NaN/Inf (plugins/nancheck.py)."""
        self._status.zero_()
        for u in self.soln:
            _lib.check(_lib.lib().bdgfs_status_check(u.data_ptr(), u.numel(),
                                                     int(u.dtype == torch.float64),
                                                     self._status.data_ptr(), _lib.stream_ptr()),
                       'bdgfs_status_check')
        if int(self._status.item()):
            raise RuntimeError(f'NaNs detected at t = {self.tcurr}')


class StdEulerDGFSBiStepper(_DGFSBiStepperMixin, BaseDGFSStepper):
    """'dgfsbi-euler' (steppers.py:229-326): u_p <- u_p + dt (L + Q_p)(u)
    for every species, Q_p = sum_q Q_pq in one launch."""
    stepper_name = 'dgfsbi-euler'
    nregs = 2
    order = 1

    def _step_kernels(self, t, dt):
        s = self.system
        s.collide_banks(t, 0, 1)                                # r1_p = Q_p(r0)
        for sp in s.species:
            sp.advect_combine(t, 0, 0, a=1.0, b=dt, x1=1, c1=dt)


class StdTVDRK2DGFSBiStepper(_DGFSBiStepperMixin, BaseDGFSStepper):
    """'dgfsbi-tvd-rk2' (steppers.py:329-486): SSP-RK2 per species with the
    mixture operator coupling the species at each stage."""
    stepper_name = 'dgfsbi-tvd-rk2'
    nregs = 3
    order = 2

    def _step_kernels(self, t, dt):
        s = self.system
        s.collide_banks(t, 0, 1)                                  # r1_p = Q_p(r0)
        for sp in s.species:                                      # r1 = r0 + dt (L+Q)(r0)
            sp.advect_combine(t, 0, 1, a=1.0, b=dt, x1=1, c1=dt)
        s.collide_banks(t + dt, 1, 2)                             # r2_p = Q_p(r1)
        for sp in s.species:                                      # r0 = r0/2 + r1/2
            sp.advect_combine(t + dt, 1, 0, a=0.5, b=0.5 * dt,    #      + dt/2 (L+Q)(r1)
                              x1=2, c1=0.5 * dt, x2=0, c2=0.5)


class ARSabcAstdStepper(BaseDGFSStepper):
    """a-stage explicit, b-stage implicit, c-order ARS IMEX schemes for the
    'adgfs' system (steppers.py:500-585): the explicit part is the FR
    advection L(f) = -div(c f) (bc update included), the implicit part the
    BGK relaxation.  Per stage i (ar = i+1): L_i = L(F_i), then one fused
    launch forms LU_i, U_ar and F_ar (bdgfs_ars_stage).  Banks: F_0 (the
    solution; the last stage updates it in place), F_1..F_{s-1}, L_0..L_{s-1};
    moment rows U_0..U_s, LU_0..LU_{s-1}."""
    _A = A = None

    @classmethod
    def nstages(cls):
        return len(cls._A) - 1

    def __init__(self, backend, system, cfg):
        super().__init__(backend, system, cfg)
        s = self.nstages()
        moms = system.get_nregs_moms(2 * s + 1)
        self._U, self._LU = moms[:s + 1], moms[s + 1:]
        self._F = [0] + list(range(1, s)) + [0]
        self._L = list(range(s, 2 * s))

    def _step_kernels(self, t, dt):
        from .adgfs import ARS_DIST, ARS_MOM0, ARS_MOML, ARS_MOMU
        sysm, s = self.system, self.nstages()
        for i in range(s):
            ar = i + 1
            sysm.advect_combine(t, self._F[i], self._L[i], a=0.0, b=1.0)     # L_i = L(F_i)
            flags = ARS_MOML | ARS_MOMU | ARS_DIST | (ARS_MOM0 if i == 0 else 0)
            sysm.ars_stage(dt, ar, flags, self._A_expl(ar), self._A_impl(ar), self._F[:ar],
                           self._F[ar], self._L[:ar], self._U[:ar + 1], self._LU[:ar])

    @classmethod
    def _A_expl(cls, ar):
        return cls._A[ar][:ar]

    @classmethod
    def _A_impl(cls, ar):
        return cls.A[ar][1:ar + 1]


class ARS111AstdStepper(ARSabcAstdStepper):
    stepper_name = 'adgfs-ars-111'
    order = 1
    _A = [[0., 0.], [1., 0.]]
    A = [[0., 0.], [0., 1.]]
    nregs = 2


class ARS222AstdStepper(ARSabcAstdStepper):
    stepper_name = 'adgfs-ars-222'
    order = 2
    gamma = 1. - (2.**0.5) / 2.
    delta = 1. - 1. / (2. * gamma)
    _A = [[0., 0., 0.], [gamma, 0., 0.], [delta, 1 - delta, 0.]]
    A = [[0., 0., 0.], [0., gamma, 0.], [0., 1 - gamma, gamma]]
    nregs = 4


class ARS443AstdStepper(ARSabcAstdStepper):
    stepper_name = 'adgfs-ars-443'
    order = 3
    _A = [[0., 0., 0., 0., 0.], [1. / 2., 0., 0., 0., 0.], [11. / 18., 1. / 18., 0., 0., 0.],
          [5. / 6., -5. / 6., 1. / 2., 0., 0.], [1. / 4., 7. / 4., 3. / 4., -7. / 4., 0.]]
    A = [[0., 0., 0., 0., 0.], [0., 1. / 2., 0., 0., 0.], [0., 1. / 6., 1. / 2., 0., 0.],
         [0., -1. / 2., 1. / 2., 1. / 2., 0.], [0., 3. / 2., -3. / 2., 1. / 2., 1. / 2.]]
    nregs = 8


class BDF1AstdStepper(ARS111AstdStepper):
    """'adgfs-bdf-1' is ARS-111 (steppers.py:675-676)."""
    stepper_name = 'adgfs-bdf-1'


class BDFqAstdStepper(BaseDGFSStepper):
    """IMEX backward-difference schemes of order q for the 'adgfs' system
    (BDF2AstdStepper / BDF3AstdStepper, steppers.py:680-860).  Per step:
    L_n = L(f_n) (one FR launch) and one fused bdgfs_bdf_step launch that
    reduces the moments of f_n and L_n, forms the new moments and writes
    f_{n+1} over the oldest history bank.  The histories live in rings of q
    banks (f, L) and moment rows (U, LU), so a step copies nothing; each of
    the q ring phases is its own CUDA graph.  The first q - 1 calls each take
    nstepsInit ARS-222 sub-steps (the reference's BDF3 takes both start-up
    steps in its first call and none in its second; the state after two
    calls is the same)."""
    q = bdf_A = bdf_G = bdf_B = nstepsInit = None

    def __init__(self, backend, system, cfg):
        super().__init__(backend, system, cfg)
        q = self.q
        moms = system.get_nregs_moms(2 * q + 1)
        self._FB = list(range(q))                 # f ring: bank 0 holds the solution at start
        self._LB = list(range(q, 2 * q))
        self._S = 2 * q                           # scratch F_1 of the ARS-222 start-up
        self._UR, self._LR, self._UN = moms[:q], moms[q:2 * q], moms[2 * q]
        self._nstart = 0
        self._phase = 1
        self._graphs = {}

    def _ars222(self, t, dt):
        """One ARS-222 sub-step of the solution in bank 0 (ARSabcAstdStepper)."""
        from .adgfs import ARS_DIST, ARS_MOM0, ARS_MOML, ARS_MOMU
        sysm, A = self.system, ARS222AstdStepper
        F, L = [0, self._S, 0], self._LB[:2]
        U, LU = [self._UR[0], self._UR[1], self._LR[0]], [self._LR[1], self._UN]
        for i in range(2):
            ar = i + 1
            sysm.advect_combine(t, F[i], L[i], a=0.0, b=1.0)
            flags = ARS_MOML | ARS_MOMU | ARS_DIST | (ARS_MOM0 if i == 0 else 0)
            sysm.ars_stage(dt, ar, flags, A._A_expl(ar), A._A_impl(ar), F[:ar], F[ar], L[:ar],
                           U[:ar + 1], LU[:ar])

    def _startup(self, t, dt):
        sysm, k = self.system, self._nstart
        sysm._bank(self._FB[k + 1]).copy_(sysm._bank(0))       # keep f(t) as history
        h = dt / self.nstepsInit
        for j in range(self.nstepsInit):
            self._ars222(t + j * h, h)
        self._nstart += 1
        if self._nstart == self.q - 1:
            # history rows of the older states: L_i = L(f_i), U_i, LU_i
            from .adgfs import BDF_MOMN
            q, p = self.q, self._phase
            for i in range(q - 1):
                fb, lb = self._FB[(p + i) % q], self._LB[(p + i) % q]
                sysm.advect_combine(t, fb, lb, a=0.0, b=1.0)
                ii = (p + i) % q
                sysm.bdf_step(dt, 1, BDF_MOMN, [0.0, 1.0], [0.0], 0.0, [fb], fb, [lb],
                              [self._UR[ii]], [self._LR[ii]], self._UN)

    def _bdf_kernels(self, t, dt, p):
        from .adgfs import BDF_DIST, BDF_MOMN, BDF_MOMU
        sysm, q = self.system, self.q
        order = [(p + i) % q for i in range(q)]
        fb = [self._FB[i] for i in order]
        lb = [self._LB[i] for i in order]
        sysm.advect_combine(t, fb[-1], lb[-1], a=0.0, b=1.0)             # L_n = L(f_n)
        sysm.bdf_step(dt, q, BDF_MOMN | BDF_MOMU | BDF_DIST, self.bdf_A, [-x for x in self.bdf_G],
                      self.bdf_B, fb, fb[0], lb, [self._UR[i] for i in order],
                      [self._LR[i] for i in order], self._UN)

    def step(self, t, dt):
        if self._nstart < self.q - 1:
            self._startup(t, dt)
            return
        p = self._phase
        if not self.use_graph:
            self._bdf_kernels(t, dt, p)
        elif (p, dt) in self._graphs:
            self._graphs[(p, dt)].replay()
        else:
            s = torch.cuda.Stream(device=self.backend.device)
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                self._bdf_kernels(t, dt, p)                     # the real step
            torch.cuda.current_stream().wait_stream(s)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._bdf_kernels(t, dt, p)
            self._graphs[(p, dt)] = g
        self._idxcurr = self._FB[p]
        self._phase = (p + 1) % self.q


class BDF2AstdStepper(BDFqAstdStepper):
    stepper_name = 'adgfs-bdf-2'
    order = q = 2
    bdf_A = [1. / 3., -4. / 3., 1.]
    bdf_G = [-2. / 3., 4. / 3.]
    bdf_B = 2. / 3.
    nstepsInit = 10
    nregs = 5


class BDF3AstdStepper(BDFqAstdStepper):
    stepper_name = 'adgfs-bdf-3'
    order = q = 3
    bdf_A = [-2. / 11., 9. / 11., -18. / 11., 1.]
    bdf_G = [6. / 11., -18. / 11., 18. / 11.]
    bdf_B = 6. / 11.
    nstepsInit = 100
    nregs = 7


STEPPERS = {c.stepper_name: c for c in (StdEulerDGFSStepper, StdTVDRK2DGFSStepper,
                                        StdEulerDGFSBiStepper, StdTVDRK2DGFSBiStepper,
                                        ARS111AstdStepper, ARS222AstdStepper, ARS443AstdStepper,
                                        BDF1AstdStepper, BDF2AstdStepper, BDF3AstdStepper)}


def get_integrator(backend, system_or_factory, cfg):
    """Controller 'none' x stepper by scheme name (integrators/__init__.py)."""
    sect = 'solver-time-integrator'
    ctrl = cfg.get(sect, 'controller', 'none')
    if ctrl != 'none':
        raise ValueError(f'unsupported controller {ctrl}')
    scheme = cfg.get(sect, 'scheme')
    if scheme not in STEPPERS:
        raise ValueError(f'unsupported scheme {scheme}; have {sorted(STEPPERS)}')
    cls = STEPPERS[scheme]
    system = system_or_factory(cls.nregs) if callable(system_or_factory) else system_or_factory
    return cls(backend, system, cfg)
