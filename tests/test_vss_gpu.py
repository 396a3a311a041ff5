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


def _reference_model(g, prec):
    return _model(g['Nv'], g['Nrho'], g['M'], g['Mpre'], precision=prec,
                  masses=tuple(g['molar']), alpha=g['alpha'], omega=g['omega'], dev=g['dev'])


def _collide(be, sm, F):
    """Q of the mixture launch for F [dof][species][Nv^3] (FP64 numpy)."""
    S = F.shape[1]
    fs = [torch.tensor(np.ascontiguousarray(F[:, p]), dtype=be.fpdtype, device=be.device)
          for p in range(S)]
    Qs = [torch.full_like(f, float('nan')) for f in fs]
    sm.collide(fs, Qs)
    torch.cuda.synchronize()
    return np.stack([Q.double().cpu().numpy() for Q in Qs], axis=1)


@pytest.mark.parametrize('prec,tol', [('double', 1e-11), ('single', 2e-4)])
def test_vss_equals_reference_kernels(cuda, prec, tol):
    """Q of the mixture launch against the reference's own vss-gll CUDA
    kernels and cuFFT (golden vectors of tests/golden/make_reference_q.py,
    the reference's host order of frfs/solvers/dgfsbi/scattering.py:256-330;
    no conservation projection, as there): FP64 to rounding, FP32 to the
    mixture operator's FP32 tolerance."""
    import os
    from oracle.ref_vss.build import GRIDS
    g = GRIDS['bi16']
    d = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'reference_qbi_bi16.npz'))
    be, sm = _reference_model(g, prec)
    got = _collide(be, sm, d['f'])
    for p in range(2):
        err = rel_l2(got[:, p], d['Q'][:, p])
        print(f'bi16 {prec} species {p}: {err:.2e}')
        assert err < tol


def test_vss_equals_reference_kernels_live(cuda):
    """The mixture launch and the reference's own vss-gll kernels (built in
    oracle/_ref by python -m oracle.ref_vss.build; skipped where they were not
    built) on the same fresh seeded distributions on the same GPU, FP64."""
    import json
    import os
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    so = os.path.join(root, 'oracle', '_ref', 'libref_vss_bi16.so')
    if not os.path.exists(so):
        pytest.skip('reference kernels not built (oracle/_ref)')
    sys.path.insert(0, os.path.join(root, 'tests', 'golden'))
    from make_reference_q import run_vss
    from oracle.ref_vss.build import grid_tables
    with open(os.path.join(root, 'oracle', '_ref', 'ref_vss_bi16.json')) as fh:
        g = json.load(fh)
    vm, _, _, par = grid_tables(g)
    rng = np.random.default_rng(4242)
    F = np.stack([np.stack(mixture(vm.cv, vm.masses, rng, k=3)) for _ in range(2)])
    Qr = run_vss(so, g, vm, par, F)
    be, sm = _reference_model(g, 'double')
    got = _collide(be, sm, F)
    err = max(rel_l2(got[:, p], Qr[:, p]) for p in range(2))
    print(f'live bi16 double: {err:.2e}')
    assert err < 1e-11
