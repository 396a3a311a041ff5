"""The FP64 collision oracle (oracle.vhs) on the host cores: a spawned
process pool, each worker holding the oracle's tables for one velocity grid.
Spawned, not forked, so it may start after the GPU is in use.  Test
infrastructure only."""
import multiprocessing as mp
import os
import sys
from concurrent.futures import ProcessPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NONDIM = dict(T0=273.0, H0=1e-3, rho0=0.00011140244750324529, molarMass0=39.96e-3)
_ORCS = {}


def _init(grids):
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from oracle.velocitymesh import VelocityMesh
    from oracle.vhs import VHSOracle
    for key, (Nv, Nrho, sz, dev, omega, scale) in grids.items():
        vm = VelocityMesh(Nv, Nrho, np.asarray(sz), cmax=0.0, Tmax=NONDIM['T0'], dev=dev,
                          **NONDIM)
        _ORCS[key] = (VHSOracle(vm, omega, 4.17e-10, NONDIM['T0']), scale)


def _work(item):
    key, F = item
    orc, scale = _ORCS[key]
    return np.stack([scale * orc.Q(f) for f in F]) if len(F) else np.zeros((0, orc.vm.vsize))


class OraclePool:
    """grids: {key: (Nv, Nrho, sz[M][3], L, omega, scale)}; ``Q(key, F)``
    returns the reference algorithm's Q (times scale) of every row of F."""

    def __init__(self, grids, workers=None):
        self.n = max(1, min(workers or os.cpu_count() or 1, 32))
        self.pool = ProcessPoolExecutor(max_workers=self.n, mp_context=mp.get_context('spawn'),
                                        initializer=_init, initargs=(grids,))

    def Q(self, key, F):
        F = np.asarray(F, dtype=np.float64)
        chunks = [c for c in np.array_split(F, min(len(F), 4 * self.n)) if len(c)]
        return np.concatenate(list(self.pool.map(_work, [(key, c) for c in chunks])))

    def close(self):
        self.pool.shutdown()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def grid_entry(vm, omega, scale=1.0):
    """The pool entry of a product velocity mesh (cmax = 0, Tmax = T0, so
    the oracle's dev equals the mesh half-width L)."""
    return (vm.Nv(), vm.Nrho(), np.asarray(vm.sz()), vm.L(), omega, scale)


def project(Q, c0):
    """The conservation projection the collision launch applies (FP64):
    the minimal-norm change of each row of Q that zeroes its mass, momentum
    and energy sums."""
    cx, cy, cz = np.meshgrid(c0, c0, c0, indexing='ij')
    Phi = np.stack([np.ones_like(cx), cx, cy, cz, cx * cx + cy * cy + cz * cz]).reshape(5, -1)
    lam = np.linalg.solve(Phi @ Phi.T, Phi @ np.asarray(Q).T)
    return Q - (Phi.T @ lam).T
