"""Host construction of every C-ABI descriptor from the product classes
(tables built on the CPU here, so that argument order and types are
checked without a GPU)."""
import numpy as np
import torch

from frfs_b200 import _lib
from frfs_b200.mesh import ElementGeometry, StructuredMesh
from frfs_b200.scattering import VHSGrid, vhs_prefactor
from frfs_b200.velocitymesh import DGFSVelocityMesh

from helpers import couette_cfg


class _CPUBackend:
    """Stand-in with the backend's allocation methods, CPU tensors (host
    construction only; nothing is launched)."""
    fpdtype = torch.float32
    device = torch.device('cpu')

    def zeros(self, *shape, dtype=None):
        return torch.zeros(*shape, dtype=dtype or self.fpdtype)

    def empty(self, *shape, dtype=None):
        return torch.empty(*shape, dtype=dtype or self.fpdtype)

    def const(self, a, dtype=None):
        return torch.as_tensor(a, dtype=dtype or self.fpdtype).contiguous()


def test_vhs_grid_struct_fields():
    cfg = couette_cfg(16, 8, 6, 5, 2)
    vm = DGFSVelocityMesh(None, cfg)
    gam, pref, _ = vhs_prefactor(vm, 0.81, 4.17e-10, 273.0)
    g = VHSGrid(vm.Nv(), vm.L(), vm.qz(), vm.qw(), vm.sz(), vm.sw(), gam, pref, vm.cw(),
                vm.c0(), torch.float32, 'cpu')
    s = g.struct
    assert (s.Nv, s.Nrho, s.M, s.fp64, s.tile) == (16, 8, 6, 0, 0)
    assert s.prefac == pref and s.cw == vm.cw()
    assert s.phase == g.phase.data_ptr() and s.gw == g.gw.data_ptr()
    assert s.bb2 == g.bb2.data_ptr() and s.c0 == g.c0.data_ptr() and s.ginv == g.ginv.data_ptr()
    arr = (_lib.VhsGrid * 1)(s)
    assert _lib.lib().bdgfs_vhs_tiles(arr, 1, None, 0) >= 2          # Nv=16 variants
    assert _lib.lib().bdgfs_vhs_scratch_bytes(arr, 1, 4) > 0
    b = _lib.VhsBatch(grid=0, ndof=3, f=16, Q=32, moments=0)
    assert (b.grid, b.ndof, b.f, b.Q) == (0, 3, 16, 32)


def test_fr_structs_fields():
    from frfs_b200.system import DGFSBoundaries, DGFSElements
    cfg = couette_cfg(16, 8, 6, 5, 2)
    be = _CPUBackend()
    vm = DGFSVelocityMesh(be, cfg)
    mesh = StructuredMesh((3, 2), (0.0, -0.5), (1.0, 0.5), periodic='x')
    geo = ElementGeometry(mesh, 2)
    el = DGFSElements(be, geo, vm)
    s = el.struct
    assert (s.ndims, s.nupts, s.nfpts, s.neles, s.nv, s.Nv, s.fp64) == (2, 9, 12, 6, 4096, 16, 0)
    assert s.m0 == el.m0.data_ptr() and s.nbr == el.nbr.data_ptr() and s.c0 == el.c0.data_ptr()
    w = DGFSBoundaries(be, geo, vm, cfg, geo.wall_names)
    ws = w.struct
    assert (ws.nwall, ws.nbc) == (len(geo.wall_fpts), 2)
    assert ws.bcv == w.bcv.data_ptr() and ws.cw == vm.cw()
    assert ws.kind == w.kind.data_ptr() and ws.kinds_used == 1
    assert w.fw.shape == (2, 4096)
