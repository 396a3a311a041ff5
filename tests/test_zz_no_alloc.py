"""The allocation-free collision entry point (bdgfs_vhs_collide_static).

It serves callers that cannot allocate device memory when they need Q --
their device memory belongs to another allocator or a fixed arena, or their
time loop must not allocate once running.  Called through the C ABI twice in
a row, it must give the same Q as bdgfs_vhs_collide with caller-provided
scratch, within the FP32 tolerance the collision tests use (1e-3 relative
L2; the two paths run identical per-distribution arithmetic).  Collected
last, so that a run stopping at the first failure has run everything else.
"""
import numpy as np
import pytest
import torch

from frfs_b200 import _lib
from frfs_b200.backend import CUDABackend
from frfs_b200.scattering import DGFSVHSGLLScatteringModel
from frfs_b200.velocitymesh import DGFSVelocityMesh

from helpers import vhs_cfg, mixed_maxwellians, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-3


def test_static_scratch_entry_matches_allocating_entry(cuda):
    cfg = vhs_cfg(24, 12, 12, 6, precision='single')
    be = CUDABackend(cfg)
    vm = DGFSVelocityMesh(be, cfg)
    sm = DGFSVHSGLLScatteringModel(be, cfg, vm)
    rng = np.random.default_rng(2024)
    F = np.stack([mixed_maxwellians(vm.cv(), rng) for _ in range(300)])
    fin = torch.from_numpy(F).float().to(be.device)
    q_ref = torch.empty_like(fin)
    sm.collide(fin, q_ref, project=True, exact=False)

    garr = (_lib.VhsGrid * 1)(sm.grid.struct)
    L = _lib.lib()
    outs = []
    for _ in range(2):                          # two calls in a row
        q = torch.full_like(fin, float('nan'))
        b = (_lib.VhsBatch * 1)(_lib.VhsBatch(grid=0, ndof=fin.shape[0], f=fin.data_ptr(),
                                              Q=q.data_ptr(), moments=0))
        rc = L.bdgfs_vhs_collide_static(garr, 1, b, 1, 1, _lib.stream_ptr())
        assert rc == 0, rc
        torch.cuda.synchronize()
        outs.append(q)
    for q in outs:
        assert bool(torch.isfinite(q).all())
        assert rel_l2(q.double().cpu().numpy(), q_ref.double().cpu().numpy()) < TOL


def test_static_scratch_entry_rejects_bad_input(cuda):
    """Unsupported grids and missing buffers are refused with a status code
    before anything is launched; the largest supported grid (Nv = 32) needs
    well under the 16 MiB array per CTA."""
    L = _lib.lib()
    g32 = _lib.VhsGrid(Nv=32, Nrho=16, M=12, fp64=0, tile=0, prefac=1.0, cw=1.0)
    assert 0 < L.bdgfs_vhs_scratch_bytes((_lib.VhsGrid * 1)(g32), 1, 1) < (16 << 20)
    bad = _lib.VhsGrid(Nv=20, Nrho=4, M=6, fp64=0, tile=0, prefac=1.0, cw=1.0)
    b = (_lib.VhsBatch * 1)(_lib.VhsBatch(grid=0, ndof=1, f=16, Q=16, moments=0))
    assert L.bdgfs_vhs_collide_static((_lib.VhsGrid * 1)(bad), 1, b, 1, 0, None) == -3
    nob = (_lib.VhsBatch * 1)(_lib.VhsBatch(grid=0, ndof=1, f=0, Q=0, moments=0))
    assert L.bdgfs_vhs_collide_static((_lib.VhsGrid * 1)(g32), 1, nob, 1, 0, None) == -1
