"""Checkpoint file round trip on the host (the restart itself is checked on
the GPU in test_checkpoint_gpu.py)."""
import os

import numpy as np
import pytest
import torch

from frfs_b200 import checkpoint
from frfs_b200.mesh import StructuredMesh

from helpers import couette_cfg


class _Sys:
    name = 'dgfs'


class _Integ:
    def __init__(self, cfg, banks):
        self.cfg, self.system = cfg, _Sys()
        self.soln = banks if len(banks) > 1 else banks[0]
        self.tcurr, self.nacptsteps = 0.0123, 7


@pytest.mark.parametrize('nspcs', [1, 2])
def test_round_trip(tmp_path, nspcs):
    cfg = couette_cfg(8, 4, 6, 5, 2)
    rng = np.random.default_rng(0)
    banks = [torch.from_numpy(rng.standard_normal((6, 9, 512)).astype(np.float32))
             for _ in range(nspcs)]
    path = tmp_path / 'run.npz'
    checkpoint.save(path, _Integ(cfg, banks))
    ck = checkpoint.load(path)
    assert ck.system == 'dgfs' and ck.tcurr == 0.0123 and ck.nacptsteps == 7
    assert ck.cfg.get('scattering-model', 'type') == 'vhs-gll'
    assert len(ck.soln) == nspcs
    for a, b in zip(ck.soln, banks):
        assert a.dtype == np.float32 and np.array_equal(a, b.numpy())


def test_shape_mismatch_and_foreign_files_are_refused(tmp_path):
    cfg = couette_cfg(8, 4, 6, 5, 2)
    path = tmp_path / 'run.npz'
    checkpoint.save(path, _Integ(cfg, [torch.zeros(5, 9, 512)]))
    ck = checkpoint.load(path)
    with pytest.raises(ValueError):
        checkpoint.interp_soln(StructuredMesh((3, 2), (0.0, -0.5), (1.0, 0.5)), ck.cfg,
                               ck.cfg, ck.soln[0])
    with pytest.raises(ValueError):      # another velocity grid
        checkpoint.interp_soln(StructuredMesh((5, 1), (0.0, -0.5), (1.0, 0.5)),
                               couette_cfg(12, 4, 6, 5, 2), ck.cfg, ck.soln[0])
    np.savez(tmp_path / 'other.npz', format=np.array('something-else'))
    with pytest.raises(ValueError):
        checkpoint.load(tmp_path / 'other.npz')


def test_extension_is_added(tmp_path):
    cfg = couette_cfg(8, 4, 6, 5, 2)
    checkpoint.save(tmp_path / 'run', _Integ(cfg, [torch.ones(2, 9, 512)]))
    assert (tmp_path / 'run.npz').exists()
    assert checkpoint.load(tmp_path / 'run').nacptsteps == 7


GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


@pytest.mark.parametrize('new,old', [(2, 3), (3, 2), (2, 1)])
def test_restart_interpolation_equals_reference_operator(new, old):
    """A solution stored at order ``old`` restarts at order ``new`` through
    the reference's own interpolation operator (solvers/dgfs/system.py:
    96-107, the stored basis' nodal_basis_at of the current points, written
    by tests/golden/make_golden.py)."""
    ref = np.load(os.path.join(GOLDEN, f'shapes_quad_p{new}.npz'))[f'interp_from_p{old}']
    mesh = StructuredMesh((3, 2), (0.0, -0.5), (1.0, 0.5))
    rng = np.random.default_rng(new * 10 + old)
    arr = rng.standard_normal((6, (old + 1)**2, 512))
    out = checkpoint.interp_soln(mesh, couette_cfg(8, 4, 6, 5, new),
                                 couette_cfg(8, 4, 6, 5, old), arr)
    assert out.shape == (6, (new + 1)**2, 512) and out.dtype == arr.dtype
    np.testing.assert_allclose(out, np.einsum('ij,ejv->eiv', ref, arr), rtol=0, atol=1e-13)
    # the same order passes through unchanged
    same = checkpoint.interp_soln(mesh, couette_cfg(8, 4, 6, 5, old),
                                  couette_cfg(8, 4, 6, 5, old), arr)
    assert same is arr


def test_restart_interpolation_is_exact_for_polynomials():
    """A field of degree <= the stored order is reproduced exactly at the
    new solution points (hex, order 2 -> 3, FP32 state)."""
    from frfs_b200.shapes import TensorShape
    mesh = StructuredMesh((2, 1, 1), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))

    def field(pts, v):
        x, y, z = pts[:, 0], pts[:, 1], pts[:, 2]
        return (1 + v) * x * x * y - 0.5 * z * y + 0.25 * v * z * z * x + 0.1

    v = np.arange(512) / 512.0
    p2, p3 = TensorShape('hex', 2).upts, TensorShape('hex', 3).upts
    arr = np.stack([field(p2, v[:, None]).T] * 2).astype(np.float32)   # (2, 27, 512)
    out = checkpoint.interp_soln(mesh, couette_cfg(8, 4, 6, 5, 3),
                                 couette_cfg(8, 4, 6, 5, 2), arr)
    want = field(p3, v[:, None]).T
    assert out.dtype == np.float32
    np.testing.assert_allclose(out[0], want, rtol=0, atol=2e-6)
    np.testing.assert_allclose(out[1], want, rtol=0, atol=2e-6)
