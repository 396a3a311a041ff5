"""Restart from a checkpoint continues the run exactly: 2 steps, save,
restart, 1 step equals 3 uninterrupted steps (bitwise), for 'dgfs' and for
the 'dgfsbi' mixture."""
import numpy as np
import pytest
import torch

from frfs_b200 import checkpoint
from frfs_b200.backend import CUDABackend
from frfs_b200.dgfsbi import DGFSBiSystem
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
