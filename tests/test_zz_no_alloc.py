"""The allocation-free collision entry point (bdgfs_vhs_collide_static).

It serves callers that cannot allocate device memory when they need Q --
their device memory belongs to another allocator or a fixed arena, or their
time loop must not allocate once running.  Called through the C ABI twice in
a row, it must give exactly the Q of bdgfs_vhs_collide with caller-provided
scratch: both run the same compiled variant (the grid's tile) and every
distribution's arithmetic is done by one CTA in a fixed order, whichever CTA
takes it and however many CTAs run, so the results are bitwise equal.  At
Nv = 32 one CTA's scratch is large enough that only some CTAs fit in the
16 MiB array (fewer CTAs than SMs run): the result must still be the same.
One case is also checked against the FP64 oracle at the FP32 collision
tolerance (1e-3 relative L2).  Collected last, so that a run stopping at the
first failure has run everything else.
"""
import numpy as np
import pytest
import torch

from frfs_b200 import _lib
from frfs_b200.backend import CUDABackend
from frfs_b200.scattering import DGFSVHSGLLScatteringModel, VHSCollider
from frfs_b200.velocitymesh import DGFSVelocityMesh

from helpers import vhs_cfg, mixed_maxwellians, oracle_for, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-3
STATIC_BYTES = 16 << 20


def _static_twice(sm, fin):
    garr = (_lib.VhsGrid * 1)(sm.grid.struct)      # the tuned tile of the allocating path
    L = _lib.lib()
    outs = []
    for _ in range(2):                              # two calls in a row
        q = torch.full_like(fin, float('nan'))
        b = (_lib.VhsBatch * 1)(_lib.VhsBatch(grid=0, ndof=fin.shape[0], f=fin.data_ptr(),
                                              Q=q.data_ptr(), moments=0))
        rc = L.bdgfs_vhs_collide_static(garr, 1, b, 1, 1, _lib.stream_ptr())
        assert rc == 0, rc
        torch.cuda.synchronize()
        outs.append(q)
    return outs


@pytest.mark.parametrize('Nv,Nrho,ndof', [(24, 12, 300), (32, 16, 160)])
def test_static_scratch_entry_equals_allocating_entry(cuda, Nv, Nrho, ndof):
    cfg = vhs_cfg(Nv, Nrho, 12, 6, precision='single')
    be = CUDABackend(cfg)
    vm = DGFSVelocityMesh(be, cfg)
    sm = DGFSVHSGLLScatteringModel(be, cfg, vm)
    rng = np.random.default_rng(2024 + Nv)
    F = np.stack([mixed_maxwellians(vm.cv(), rng) for _ in range(ndof)])
    fin = torch.from_numpy(F).float().to(be.device)
    L = _lib.lib()
    if Nv == 32:
        # the variant with the largest scratch per CTA: fewer CTAs than SMs
        # fit in the array, the case to be run
        def per(t):
            sm.grid.struct.tile = t
            return L.bdgfs_vhs_scratch_bytes((_lib.VhsGrid * 1)(sm.grid.struct), 1, 1)
        ntiles = L.bdgfs_vhs_tiles((_lib.VhsGrid * 1)(sm.grid.struct), 1, None, 0)
        t = max(range(ntiles), key=per)
        nsm = torch.cuda.get_device_properties(cuda).multi_processor_count
        assert (STATIC_BYTES - 256) // per(t) < nsm
    q_ref = torch.empty_like(fin)
    VHSCollider([sm.grid], be.device)([(0, fin, q_ref, None)], project=True, exact=False)
    torch.cuda.synchronize()
    q1, q2 = _static_twice(sm, fin)
    assert bool(torch.isfinite(q1).all())
    assert torch.equal(q1, q2)
    assert torch.equal(q1, q_ref)
    if Nv == 24:
        orc = oracle_for(vm)
        c0 = vm.c0().astype(np.float64)
        cx, cy, cz = np.meshgrid(c0, c0, c0, indexing='ij')
        Phi = np.stack([np.ones_like(cx), cx, cy, cz, cx * cx + cy * cy + cz * cz]).reshape(5, -1)
        rows = [0, ndof - 1]
        Qo = np.stack([orc.Q(F[i]) for i in rows])
        Qo -= (Phi.T @ np.linalg.solve(Phi @ Phi.T, Phi @ Qo.T)).T   # the launch's projection
        assert rel_l2(q1[rows].double().cpu().numpy(), Qo) < TOL


def test_static_scratch_entry_rejects_bad_input(cuda):
    """Unsupported grids and missing buffers are refused with a status code
    before anything is launched; the largest supported grid (Nv = 32) needs
    well under the 16 MiB array per CTA."""
    L = _lib.lib()
    g32 = _lib.VhsGrid(Nv=32, Nrho=16, M=12, fp64=0, tile=0, prefac=1.0, cw=1.0)
    assert 0 < L.bdgfs_vhs_scratch_bytes((_lib.VhsGrid * 1)(g32), 1, 1) < STATIC_BYTES
    bad = _lib.VhsGrid(Nv=20, Nrho=4, M=6, fp64=0, tile=0, prefac=1.0, cw=1.0)
    b = (_lib.VhsBatch * 1)(_lib.VhsBatch(grid=0, ndof=1, f=16, Q=16, moments=0))
    assert L.bdgfs_vhs_collide_static((_lib.VhsGrid * 1)(bad), 1, b, 1, 0, None) == -3
    nob = (_lib.VhsBatch * 1)(_lib.VhsBatch(grid=0, ndof=1, f=0, Q=0, moments=0))
    assert L.bdgfs_vhs_collide_static((_lib.VhsGrid * 1)(g32), 1, nob, 1, 0, None) == -1
