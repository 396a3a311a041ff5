"""GPU parity of the gas-mixture VSS operator (bdgfs_vss_collide) against
the FP64 oracle restatement of the reference's algorithm."""
import numpy as np
import pytest
import torch

from frfs_b200.backend import CUDABackend
from frfs_b200.dgfsbi import DGFSBiVelocityMesh, DGFSBiVSSGLLScatteringModel

from helpers import mixture, rel_l2, vss_cfg, vss_oracle_for

pytestmark = pytest.mark.gpu


def _model(Nv, Nrho, M, Mpre, precision='double', masses=(39.96e-3, 83.798e-3), **kw):
    cfg = vss_cfg(Nv, Nrho, M, Mpre, precision=precision, masses=masses, **kw)
    be = CUDABackend(cfg)
    vm = DGFSBiVelocityMesh(be, cfg, len(masses))
    return be, DGFSBiVSSGLLScatteringModel(be, cfg, vm)


def _run(be, sm, ndof, seed):
    o = vss_oracle_for(sm)
    rng = np.random.default_rng(seed)
    S = sm.vm.nspcs()
    F = [mixture(o.vm.cv, o.vm.masses, rng) for _ in range(ndof)]         # [dof][species]
    fs = [torch.tensor(np.stack([F[d][p] for d in range(ndof)]), dtype=be.fpdtype,
                       device=be.device) for p in range(S)]
    Qs = [torch.full_like(f, float('nan')) for f in fs]
    sm.collide(fs, Qs)
    torch.cuda.synchronize()
    want = [o.Q(F[d]) for d in range(ndof)]
    got = [[Qs[p][d].double().cpu().numpy() for p in range(S)] for d in range(ndof)]
    return max(rel_l2(got[d][p], want[d][p]) for d in range(ndof) for p in range(S))


@pytest.mark.parametrize('Nv,Nrho,M,Mpre', [(8, 4, 6, 12), (12, 4, 6, 6), (16, 6, 12, 12)])
def test_vss_fp64_matches_oracle(cuda, Nv, Nrho, M, Mpre):
    be, sm = _model(Nv, Nrho, M, Mpre)
    assert _run(be, sm, 5, Nv) < 1e-11


def test_vss_three_species_and_equal_masses(cuda):
    be, sm = _model(8, 4, 6, 6, masses=(4e-3, 39.96e-3, 39.96e-3), alpha=1.0)
    assert _run(be, sm, 3, 1) < 1e-11


@pytest.mark.parametrize('Nv,Nrho,M,Mpre', [(16, 6, 12, 12), (24, 6, 12, 12), (32, 4, 6, 6)])
def test_vss_fp32_matches_oracle(cuda, Nv, Nrho, M, Mpre):
    be, sm = _model(Nv, Nrho, M, Mpre, precision='single')
    assert _run(be, sm, 4, 7) < 2e-4


def test_vss_per_point_shim(cuda):
    """fs(elem, upt, f_0, f_1, Q_0, Q_1) on banks [neles][nupts][Nv^3]
    equals the batched call for that point."""
    be, sm = _model(8, 4, 6, 6)
    o = vss_oracle_for(sm)
    rng = np.random.default_rng(5)
    banks = [torch.tensor(np.stack([np.stack(mixture(o.vm.cv, o.vm.masses, rng)[p:p + 1] * 3)
                                    for _ in range(2)]), dtype=torch.float64, device=be.device)
             for p in range(2)]                                            # [2][3][n]
    Q = [torch.zeros_like(b) for b in banks]
    sm.fs(1, 2, banks[0], banks[1], Q[0], Q[1])
    Qb = [torch.zeros_like(b[1, 2]) for b in banks]
    sm.collide([b[1, 2] for b in banks], Qb)
    torch.cuda.synchronize()
    for p in range(2):
        assert torch.equal(Q[p][1, 2], Qb[p])
        assert not Q[p][0].any() and not Q[p][1, :2].any()


@pytest.mark.parametrize('Nv', [16, 24, 32])
def test_vss_fp32_several_items_per_cta(cuda, Nv):
    """Three persistent CTAs for ten (distribution, species) items: each CTA
    restarts its on-chip accumulators for every item it takes."""
    be, sm = _model(Nv, 4, 6, 6, precision='single')
    sm._nctas = 3
    sm._scratch = None
    assert _run(be, sm, 5, 11) < 2e-4


@pytest.mark.parametrize('precision,tol', [('double', 1e-11), ('single', 2e-4)])
def test_vss_conservation_projection(cuda, precision, tol):
    """With the FP64 projection on, Q equals the oracle's Q after the same
    minimal-norm projection, and (FP64) each species' mass, the total
    momentum and the total energy of Q vanish to rounding."""
    from oracle.vss import project_mixture
    be, sm = _model(16, 6, 12, 12, precision=precision)
    o = vss_oracle_for(sm)
    rng = np.random.default_rng(8)
    F = [mixture(o.vm.cv, o.vm.masses, rng) for _ in range(4)]
    fs = [torch.tensor(np.stack([F[d][p] for d in range(4)]), dtype=be.fpdtype, device=be.device)
          for p in range(2)]
    Qs = [torch.empty_like(f) for f in fs]
    sm.collide(fs, Qs, project=True)
    torch.cuda.synchronize()
    cv, m = o.vm.cv, o.vm.masses
    for d in range(4):
        want = project_mixture(o.Q(F[d]), cv, m)
        got = [Qs[p][d].double().cpu().numpy() for p in range(2)]
        assert max(rel_l2(got[p], want[p]) for p in range(2)) < tol
        if precision == 'double':
            scale = sum(np.abs(g).sum() for g in got)
            assert max(abs(g.sum()) for g in got) < 1e-12 * scale
            mom = sum(mp * (cv @ g) for mp, g in zip(m, got))
            en = sum(mp * (np.sum(cv * cv, 0) @ g) for mp, g in zip(m, got))
            assert np.abs(mom).max() < 1e-12 * scale * np.abs(cv).max()
            assert abs(en) < 1e-12 * scale * np.sum(cv * cv, 0).max()
