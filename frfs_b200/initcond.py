"""Initial / wall distributions (host, FP64).

``DGFSMaxwellianInitCondition`` (frfs/solvers/dgfs/initcond.py:39-117):
f = rho/(pi T)^{3/2} exp(-|c - u|^2 / T) in non-dimensional units (rho, T,
u read from the section and divided by rho0, T0, u0), with the reference's
moment-consistency check (raises ``ValueError`` when the grid cannot
represent the state to 1e-5).  ``DGFSBKWInitCondition``
(initcond.py:120-140): the Bobylev-Krook-Wu solution at t0.
``DGFSMaxwellianExprInitCondition`` (initcond.py:143-212): a Maxwellian per
solution point whose rho, u, T are expressions of x, y, z and the
[constants]; built on the device from its moment rows.
"""
import numpy as np
import torch

from . import _lib
from .util import npeval


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


class DGFSMaxwellianExprInitCondition(DGFSInitCondition):
    model = 'maxwellianExpr'

    def load_parameters(self, name):
        self._vars = self.cfg.items_as('constants', float)
        self.name = name
        if any(d in self._vars for d in 'xyz'):
            raise ValueError('Invalid constants (x, y, or z) in config file')

    def perform_precomputation(self):
        pass

    def unondim(self):
        raise ValueError('this model depends on spatial coordinates!')

    def get_init_vals(self):
        raise ValueError('this model depends on spatial coordinates!')

    def fields(self, ploc):
        """Non-dimensional (rho, ux, uy, uz, T) at the points ploc[..., ndims]."""
        vm = self.vm
        v = dict(self._vars)
        v.update(zip('xyz', np.moveaxis(np.asarray(ploc, dtype=np.float64), -1, 0)))
        shp = np.asarray(ploc).shape[:-1]
        scale = {'rho': vm.rho0(), 'ux': vm.u0(), 'uy': vm.u0(), 'uz': vm.u0(), 'T': vm.T0()}
        return [np.broadcast_to(np.asarray(npeval(self.cfg.getexpr(self.name, k), v),
                                           dtype=np.float64), shp) / scale[k]
                for k in ('rho', 'ux', 'uy', 'uz', 'T')]

    def apply_init_vals(self, bank, ploc):
        """bank[e][upt][:] <- the Maxwellian of the fields at ploc[e][upt]
        (bdgfs_bgk_maxwellian from the rows (rho, rho u, E)); raises when a
        point's density is not represented to 1e-5 (initcond.py:156-169)."""
        vm = self.vm
        rho, ux, uy, uz, T = (a.reshape(-1) for a in self.fields(ploc))
        u2 = ux * ux + uy * uy + uz * uz
        U = np.stack([rho, rho * ux, rho * uy, rho * uz, 1.5 * rho * T + rho * u2], axis=-1)
        dev = bank.device
        Ud = torch.as_tensor(U, dtype=torch.float64, device=dev).contiguous()
        c0 = torch.as_tensor(vm.c0(), dtype=torch.float64, device=dev).contiguous()
        n = vm.vsize()
        _lib.check(_lib.lib().bdgfs_bgk_maxwellian(Ud.data_ptr(), bank.numel() // n, vm.Nv(),
                                                   int(bank.dtype == torch.float64), c0.data_ptr(),
                                                   bank.data_ptr(), _lib.stream_ptr()),
                   'bdgfs_bgk_maxwellian')
        bulk = bank.reshape(-1, n).double().sum(-1).cpu().numpy() * vm.cw()
        if not np.allclose(rho, bulk, atol=1e-5):
            raise ValueError('Bulk properties not conserved! Check Nv, dev')
