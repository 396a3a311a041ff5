"""A DGFS time step on a mesh imported from a Gmsh 2.2 file equals the same
step on the in-memory box it was written from."""
import io

import numpy as np
import pytest
import torch

from frfs_b200.backend import CUDABackend
from frfs_b200.gmsh import GmshMesh, write_msh
from frfs_b200.integrators import get_integrator
from frfs_b200.mesh import StructuredMesh
from frfs_b200.system import DGFSSystem

from helpers import couette_cfg, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('kind', ['quad', 'hex'])
def test_step_on_imported_mesh_equals_box(cuda, kind):
    if kind == 'quad':
        box = StructuredMesh((3, 2), (0.0, -0.5), (1.0, 0.5), periodic='x')
    else:
        box = StructuredMesh((2, 2, 2), (0.0, -0.5, 0.0), (1.0, 0.5, 1.0), periodic='xz')
    buf = io.StringIO()
    write_msh(box, buf)
    msh = GmshMesh(buf.getvalue().splitlines())
    out = []
    for mesh in (box, msh):
        cfg = couette_cfg(16, 6, 6, 5, 2, precision='double')
        be = CUDABackend(cfg)
        s = DGFSSystem(be, mesh, cfg, nreg=3)
        u = s.eles_scal_upts_inb_full[0]
        x = s.geo.plocupts
        u.mul_(torch.from_numpy(1.0 + 0.2 * np.sin(2 * np.pi * x[..., 0])
                                + 0.1 * x[..., 1])[..., None].to(u))
        integ = get_integrator(be, s, cfg)
        integ.step(0.0, 2e-4)
        torch.cuda.synchronize()
        out.append(s.eles_scal_upts_inb_full[0].double().cpu().numpy())
    assert rel_l2(out[1], out[0]) < 1e-14
