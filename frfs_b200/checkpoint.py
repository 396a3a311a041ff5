"""Checkpoint / restart of a DGFS run.

The reference writes the distribution with its config and stats to an HDF5
``.frfss`` file (plugins/dgfsdistwriterstd.py:8-66, writers/native.py:
86-186) and restarts from it (``frfs restart``, __main__.py:228-242): the
system takes the stored solution as ``initsoln`` (solvers/dgfs/system.py:
79-112) and the integrator its ``tcurr`` from the stats
(integrators/base.py:36-40).  HDF5 is not available here, so the same
content -- the config text, tcurr, the accepted-step count and the
solution bank of every species -- is stored in one ``.npz`` file.  A
restart needs the same mesh, order and velocity grid (the reference also
interpolates between solution bases; that is not done here and a mismatch
raises ``ValueError``).
"""
import numpy as np
import torch

from .inifile import Inifile

FORMAT = 'frfs_b200-checkpoint-1'


def _banks(integ):
    s = integ.soln
    return list(s) if isinstance(s, (list, tuple)) else [s]


def _npz(path):
    path = str(path)
    return path if path.endswith('.npz') else path + '.npz'


def save(path, integ):
    """Write the integrator's current solution, time and step count, and
    the config it runs, to ``path`` ('.npz' is appended when missing)."""
    path = _npz(path)
    sysm = integ.system
    banks = _banks(integ)
    arrays = {f'soln_{p}': b.detach().cpu().numpy() for p, b in enumerate(banks)}
    np.savez(path, format=np.array(FORMAT), system=np.array(sysm.name),
             config=np.array(integ.cfg.tostr()), tcurr=np.array(float(integ.tcurr)),
             nacptsteps=np.array(int(integ.nacptsteps)), nspcs=np.array(len(banks)), **arrays)


class Checkpoint:
    """The content of a checkpoint file: ``cfg`` (Inifile), ``system``,
    ``tcurr``, ``nacptsteps`` and ``soln`` (one array per species)."""

    def __init__(self, path):
        path = _npz(path)
        with np.load(path, allow_pickle=False) as z:
            if str(z['format']) != FORMAT:
                raise ValueError(f'{path}: not a {FORMAT} file')
            self.system = str(z['system'])
            self.cfg = Inifile(str(z['config']))
            self.tcurr = float(z['tcurr'])
            self.nacptsteps = int(z['nacptsteps'])
            self.soln = [z[f'soln_{p}'] for p in range(int(z['nspcs']))]


def load(path):
    return Checkpoint(path)


def restart(backend, mesh, ckpt, cfg=None):
    """The system named in the checkpoint, started from its solution, and
    its integrator at the stored time and step count.  ``cfg`` overrides the
    stored config (e.g. a new ``tend``)."""
    from .integrators import get_integrator
    cfg = cfg or ckpt.cfg
    name = cfg.get('solver', 'system', ckpt.system)
    if name != ckpt.system:
        raise ValueError(f'checkpoint of system {ckpt.system}, config asks for {name}')
    if name == 'dgfsbi':
        from .dgfsbi import DGFSBiSystem

        def make(nreg):
            for a in ckpt.soln:
                _check_shape(mesh, cfg, a)
            return DGFSBiSystem(backend, mesh, cfg, nreg=nreg, initsoln=ckpt.soln)
    else:
        if name == 'adgfs':
            from .adgfs import ADGFSSystem as cls
        elif name == 'dgfs':
            from .system import DGFSSystem as cls
        else:
            raise ValueError(f'unknown system {name}')

        def make(nreg):
            _check_shape(mesh, cfg, ckpt.soln[0])
            return cls(backend, mesh, cfg, nreg=nreg, initsoln=ckpt.soln[0])
    integ = get_integrator(backend, make, cfg)
    integ.tcurr = ckpt.tcurr
    integ.nacptsteps = ckpt.nacptsteps
    return integ


def _check_shape(mesh, cfg, arr):
    from .mesh import ElementGeometry
    geo = ElementGeometry(mesh, cfg.getint('solver', 'order'))
    Nv = cfg.getint('constants', 'Nv')
    want = (geo.neles, geo.nupts, Nv**3)
    if tuple(arr.shape) != want:
        raise ValueError(f'checkpoint solution {arr.shape} does not fit the system {want}')
