"""Checkpoint file round trip on the host (the restart itself is checked on
the GPU in test_checkpoint_gpu.py)."""
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
        checkpoint._check_shape(StructuredMesh((3, 2), (0.0, -0.5), (1.0, 0.5)), ck.cfg,
                                ck.soln[0])
    np.savez(tmp_path / 'other.npz', format=np.array('something-else'))
    with pytest.raises(ValueError):
        checkpoint.load(tmp_path / 'other.npz')


def test_extension_is_added(tmp_path):
    cfg = couette_cfg(8, 4, 6, 5, 2)
    checkpoint.save(tmp_path / 'run', _Integ(cfg, [torch.ones(2, 9, 512)]))
    assert (tmp_path / 'run.npz').exists()
    assert checkpoint.load(tmp_path / 'run').nacptsteps == 7
