"""The 'adgfs' system on the GPU: BGK moments / Maxwellian kernels and the
ARS-111/222/443 steppers against the FP64 oracle (FR oracle for the
explicit part, oracle/bgk.py for the IMEX stages)."""
import numpy as np
import pytest
import torch

from frfs_b200.adgfs import ADGFSSystem
from frfs_b200.backend import CUDABackend
from frfs_b200.integrators import get_integrator
from frfs_b200.mesh import StructuredMesh

from helpers import couette_cfg, rel_l2
from test_fr_gpu import _fr_oracle, _perturb

pytestmark = pytest.mark.gpu

BGK = """
[scattering-model]
type = bgk-direct-gll
omega = 0.81
muRef = 2.117e-5
Tref = 273
"""


def _cfg(scheme, precision='double', Nv=16, dt=2e-3):
    cfg = couette_cfg(Nv, 4, 6, 5, 2, precision=precision, scheme=scheme, dt=dt)
    for k, v in (('type', 'bgk-direct-gll'), ('muRef', '2.117e-5'), ('Tref', '273'),
                 ('omega', '0.81')):
        cfg.set('scattering-model', k, v)
    cfg.set('solver', 'system', 'adgfs')
    return cfg


def _system(cfg, nreg):
    be = CUDABackend(cfg)
    mesh = StructuredMesh((3, 2), (0.0, -0.5), (1.0, 0.5), periodic='x')
    return be, ADGFSSystem(be, mesh, cfg, nreg=nreg)


def test_moments_and_maxwellian_kernels(cuda):
    from oracle.bgk import maxwellian, moments5
    from oracle.fr import velocities
    cfg = _cfg('adgfs-ars-111', Nv=16)
    be, s = _system(cfg, 2)
    _perturb(s, 3)
    f = s.eles_scal_upts_inb_full[0]
    s.get_nregs_moms(3)
    s.moment(0.0, 0, 0)
    s.constructMaxwellian(0.0, 0, 1)
    torch.cuda.synchronize()
    cv = velocities(s.vm.c0())
    Uo = moments5(f.double().cpu().numpy().reshape(-1, cv.shape[1]), cv, s.vm.cw())
    Ug = s.eles_scal_upts_inb_moms[0].cpu().numpy()
    assert rel_l2(Ug, Uo) < 1e-13
    Mo = maxwellian(Uo, cv)
    Mg = s.eles_scal_upts_inb_full[1].double().cpu().numpy().reshape(Mo.shape)
    assert rel_l2(Mg, Mo) < 1e-13


@pytest.mark.parametrize('scheme', ['adgfs-ars-111', 'adgfs-ars-222', 'adgfs-ars-443'])
def test_ars_steps_match_oracle(cuda, scheme):
    """Three graph-replayed ARS steps (FP64) vs the oracle stepper."""
    from oracle.bgk import step_ars
    from oracle.fr import velocities
    cfg = _cfg(scheme)
    nreg = {'adgfs-ars-111': 2, 'adgfs-ars-222': 4, 'adgfs-ars-443': 8}[scheme]
    be, s = _system(cfg, nreg)
    _perturb(s, 4)
    orc = _fr_oracle(s, 'quad', 2)
    cv = velocities(s.vm.c0())
    u = s.eles_scal_upts_inb_full[0].double().cpu().numpy()
    integ = get_integrator(be, s, cfg)
    dt = 2e-3
    for _ in range(3):
        u = step_ars(u, dt, orc.rhs, scheme, s.sm._prefactor, s.sm._omega, cv, s.vm.cw())
        integ.step(0.0, dt)
    torch.cuda.synchronize()
    g = s.eles_scal_upts_inb_full[0].double().cpu().numpy()
    assert rel_l2(g, u) < 1e-11


def test_ars_single_precision_and_reference_methods(cuda):
    """FP32 state against the FP64 oracle; and the reference-named
    updateMomentARS / updateDistARS calls against the fused stage."""
    from oracle.bgk import step_ars
    from oracle.fr import velocities
    cfg = _cfg('adgfs-ars-222', precision='single', Nv=16)
    be, s = _system(cfg, 4)
    _perturb(s, 5)
    orc = _fr_oracle(s, 'quad', 2)
    cv = velocities(s.vm.c0())
    u0 = s.eles_scal_upts_inb_full[0].double().cpu().numpy()
    integ = get_integrator(be, s, cfg)
    integ.use_graph = False
    integ.step(0.0, 2e-3)
    torch.cuda.synchronize()
    uo = step_ars(u0, 2e-3, orc.rhs, 'adgfs-ars-222', s.sm._prefactor, s.sm._omega, cv,
                  s.vm.cw())
    assert rel_l2(s.eles_scal_upts_inb_full[0].double().cpu().numpy(), uo) < 2e-5
    # reference-style single stage: L0 = L(F0); U1, F1 from the separate calls
    s.eles_scal_upts_inb_full[0].copy_(torch.from_numpy(u0))
    s.advect_combine(0.0, 0, 2, a=0.0, b=1.0)
    U, LU = [0, 1], [4]
    s.moment(0.0, 0, U[0])
    s.moment(0.0, 2, LU[0])
    A_e, A_i = integ._A_expl(1), integ._A_impl(1)
    s.updateMomentARS(2e-3, *A_e, *A_i, *LU, *U)
    s.updateDistARS(2e-3, *A_e, *A_i, 2, *U, None, 0, 1)
    ref1 = s.eles_scal_upts_inb_full[1].clone()
    s.ars_stage(2e-3, 1, 15, A_e, A_i, [0], 3, [2], [0, 1], [4])
    torch.cuda.synchronize()
    assert torch.allclose(ref1, s.eles_scal_upts_inb_full[3], rtol=1e-6, atol=0)
