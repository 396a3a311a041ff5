"""Initial / wall distributions (host, FP64).

``DGFSMaxwellianInitCondition`` (frfs/solvers/dgfs/initcond.py:39-117):
f = rho/(pi T)^{3/2} exp(-|c - u|^2 / T) in non-dimensional units (rho, T,
u read from the section and divided by rho0, T0, u0), with the reference's
moment-consistency check (raises ``ValueError`` when the grid cannot
represent the state to 1e-5).  ``DGFSBKWInitCondition``
(initcond.py:120-140): the Bobylev-Krook-Wu solution at t0.
"""
import numpy as np


class DGFSInitCondition:
    model = None

    def __init__(self, backend, cfg, velocitymesh, name):
        self.backend = backend
        self.cfg = cfg
        self.vm = velocitymesh
        self._init_vals = None
        self.load_parameters(name)
        self.perform_precomputation()

    def get_init_vals(self):
        return self._init_vals


class DGFSMaxwellianInitCondition(DGFSInitCondition):
    model = 'maxwellian'

    def load_parameters(self, name):
        vm, cfg = self.vm, self.cfg
        u0 = vm.u0()
        self._rhoini = cfg.getfloat(name, 'rho') / vm.rho0()
        self._Tini = cfg.getfloat(name, 'T') / vm.T0()
        self._uini = np.array([cfg.getfloat(name, 'ux') / u0,
                               cfg.getfloat(name, 'uy') / u0,
                               cfg.getfloat(name, 'uz') / u0]).reshape(3, 1)

    def perform_precomputation(self):
        vm = self.vm
        cv, cw = vm.cv(), vm.cw()
        f = (self._rhoini / (np.pi * self._Tini)**1.5
             * np.exp(-np.sum((cv - self._uini)**2, axis=0) / self._Tini))
        self._init_vals = f
        rho = np.sum(f) * cw
        u = (cv @ f) * cw / rho
        c = cv - u[:, None]
        T = np.sum(f * np.sum(c * c, axis=0)) * (2.0 / 3.0 * cw) / rho
        ok = (np.isclose(self._rhoini * vm.rho0(), rho * vm.rho0(), atol=1e-5)
              and np.allclose(self._uini[:, 0] * vm.u0(), u * vm.u0(), atol=1e-5)
              and np.isclose(self._Tini * vm.T0(), T * vm.T0(), atol=1e-5))
        if not ok:
            raise ValueError('Bulk properties not conserved! Check Nv, dev')

    def unondim(self):
        return self._uini


class DGFSBKWInitCondition(DGFSInitCondition):
    model = 'bkw'

    def load_parameters(self, name):
        self._t0 = self.cfg.getfloat(name, 't0')

    def perform_precomputation(self):
        K = 1.0 - np.exp(-self._t0 / 6.0)
        c2 = np.sum(self.vm.cv()**2, axis=0)
        self._init_vals = (1.0 / (2.0 * (2.0 * np.pi * K)**1.5) * np.exp(-c2 / (2.0 * K))
                           * ((5 * K - 3) / K + (1 - K) / (K * K) * c2))

    def unondim(self):
        raise ValueError('Not defined for bkw')
