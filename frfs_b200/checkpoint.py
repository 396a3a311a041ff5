"""Checkpoint / restart of a DGFS run.

The reference writes the distribution with its config and stats to an HDF5
``.frfss`` file (plugins/dgfsdistwriterstd.py:8-66, writers/native.py:
86-186) and restarts from it (``frfs restart``, __main__.py:228-242): the
system takes the stored solution as ``initsoln`` (solvers/dgfs/system.py:
79-112) and the integrator its ``tcurr`` from the stats
(integrators/base.py:36-40).  HDF5 is not available here, so the same
content -- the config text, tcurr, the accepted-step count and the
solution bank of every species -- is stored in one ``.npz`` file.  A
restart needs the same mesh and velocity grid; a solution of another order
is interpolated onto the current solution points, as the reference does
(solvers/dgfs/system.py:96-107).
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
            soln = [interp_soln(mesh, cfg, ckpt.cfg, a) for a in ckpt.soln]
            return DGFSBiSystem(backend, mesh, cfg, nreg=nreg, initsoln=soln)
    else:
        if name == 'adgfs':
            from .adgfs import ADGFSSystem as cls
        elif name == 'dgfs':
            from .system import DGFSSystem as cls
        else:
            raise ValueError(f'unknown system {name}')

        def make(nreg):
            soln = interp_soln(mesh, cfg, ckpt.cfg, ckpt.soln[0])
            return cls(backend, mesh, cfg, nreg=nreg, initsoln=soln)
    integ = get_integrator(backend, make, cfg)
    integ.tcurr = ckpt.tcurr
    integ.nacptsteps = ckpt.nacptsteps
    return integ


def interp_soln(mesh, cfg, solncfg, arr):
    """The stored solution ``arr`` ([neles][nupts of the stored order][Nv^3],
    written under ``solncfg``) on the solution points of the order ``cfg``
    asks for: the stored nodal basis evaluated at the current points applied
    per element (solvers/dgfs/system.py:96-107), in FP64 and returned in
    the stored dtype.  Mesh and velocity grid must match (the reference
    checks the field names, i.e. the velocity count)."""
    from .shapes import TensorShape
    order = cfg.getint('solver', 'order')
    sorder = solncfg.getint('solver', 'order', order)
    Nv = cfg.getint('constants', 'Nv')
    if arr.ndim != 3 or arr.shape[0] != mesh.neles or arr.shape[2] != Nv**3:
        raise ValueError(f'checkpoint solution {arr.shape} does not fit the system '
                         f'({mesh.neles}, *, {Nv**3})')
    src = TensorShape(mesh.etype, sorder)
    if arr.shape[1] != src.nupts:
        raise ValueError(f'checkpoint solution {arr.shape} does not fit its order {sorder}')
    if sorder == order:
        return arr
    op = TensorShape(mesh.etype, order).interp_from(sorder)      # (nupts, src.nupts)
    out = np.empty((arr.shape[0], op.shape[0], arr.shape[2]), dtype=arr.dtype)
    step = max(1, (1 << 26) // max(1, arr.shape[1] * arr.shape[2]))
    for e0 in range(0, arr.shape[0], step):
        blk = arr[e0:e0 + step].astype(np.float64)
        out[e0:e0 + step] = np.einsum('ij,ejv->eiv', op, blk)
    return out
