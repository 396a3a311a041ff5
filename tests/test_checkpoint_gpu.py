"""Restart from a checkpoint continues the run exactly: 2 steps, save,
restart, 1 step equals 3 uninterrupted steps (bitwise), for 'dgfs' and for
the 'dgfsbi' mixture."""
import os

import numpy as np
import pytest
import torch

from frfs_b200 import checkpoint
from frfs_b200.backend import CUDABackend
from frfs_b200.dgfsbi import DGFSBiSystem
from frfs_b200.inifile import Inifile
from frfs_b200.integrators import get_integrator
from frfs_b200.mesh import StructuredMesh
from frfs_b200.system import DGFSSystem

from helpers import couette_cfg, dgfsbi_cfg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('kind', ['dgfs', 'dgfsbi'])
def test_restart_continues_bitwise(cuda, tmp_path, kind):
    mesh = StructuredMesh((3, 2), (0.0, -0.5), (1.0, 0.5), periodic='x')
    if kind == 'dgfs':
        cfg = couette_cfg(16, 6, 6, 5, 2, precision='single', dt=2e-4)
        make = lambda be: (lambda nreg: DGFSSystem(be, mesh, cfg, nreg=nreg))
    else:
        cfg = dgfsbi_cfg(precision='single')
        make = lambda be: (lambda nreg: DGFSBiSystem(be, mesh, cfg, nreg=nreg))
    be = CUDABackend(cfg)
    full = get_integrator(be, make(be), cfg)
    part = get_integrator(be, make(be), cfg)
    full.advance_to(3 * 2e-4)
    part.advance_to(2 * 2e-4)
    path = tmp_path / 'ck.npz'
    checkpoint.save(path, part)
    ck = checkpoint.load(path)
    again = checkpoint.restart(be, mesh, ck)
    assert again.nacptsteps == 2 and again.tcurr == pytest.approx(4e-4)
    again.advance_to(3 * 2e-4)
    torch.cuda.synchronize()
    a = full.soln if isinstance(full.soln, list) else [full.soln]
    b = again.soln if isinstance(again.soln, list) else [again.soln]
    assert again.nacptsteps == 3
    for x, y in zip(a, b):
        assert torch.equal(x, y)


def test_restart_onto_another_order(cuda, tmp_path):
    """A solution saved at order 2 restarts at order 3: the new state is the
    reference's interpolation operator applied per element (golden fixture of
    solvers/dgfs/system.py:96-107) and the run continues; the mixture system
    interpolates every species the same way."""
    mesh = StructuredMesh((3, 2), (0.0, -0.5), (1.0, 0.5), periodic='x')
    op = np.load(os.path.join(os.path.dirname(__file__), 'golden',
                              'shapes_quad_p3.npz'))['interp_from_p2']
    for kind in ('dgfs', 'dgfsbi'):
        if kind == 'dgfs':
            cfg2 = couette_cfg(16, 6, 6, 5, 2, precision='double', dt=2e-4)
            make = lambda be: (lambda nreg: DGFSSystem(be, mesh, cfg2, nreg=nreg))
        else:
            cfg2 = dgfsbi_cfg(precision='double')
            make = lambda be: (lambda nreg: DGFSBiSystem(be, mesh, cfg2, nreg=nreg))
        be = CUDABackend(cfg2)
        part = get_integrator(be, make(be), cfg2)
        part.advance_to(2 * 2e-4)
        path = tmp_path / f'ck_{kind}.npz'
        checkpoint.save(path, part)
        ck = checkpoint.load(path)
        cfg3 = Inifile(ck.cfg.tostr())
        cfg3.set('solver', 'order', '3')
        again = checkpoint.restart(be, mesh, ck, cfg=cfg3)
        b = again.soln if isinstance(again.soln, list) else [again.soln]
        assert again.nacptsteps == 2 and len(b) == len(ck.soln)
        for x, y in zip(ck.soln, b):
            assert tuple(y.shape) == (6, 16, x.shape[2])
            want = np.einsum('ij,ejv->eiv', op, x)
            got = y.cpu().numpy()
            assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
        again.advance_to(3 * 2e-4)
        torch.cuda.synchronize()
        assert again.nacptsteps == 3
        for y in (again.soln if isinstance(again.soln, list) else [again.soln]):
            assert bool(torch.isfinite(y).all())
