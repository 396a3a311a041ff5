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


def _es_cfg(scheme, precision='double', Nv=16, dt=2e-3, Pr=None):
    cfg = _cfg(scheme, precision=precision, Nv=Nv, dt=dt)
    cfg.set('scattering-model', 'type', 'esbgk-direct-gll')
    if Pr is not None:
        cfg.set('scattering-model', 'Pr', str(Pr))
    return cfg


def test_esbgk_moments_and_gaussian_kernels(cuda):
    """'esbgk-direct-gll': 11 moments and the ES Gaussian (FP64) vs the oracle."""
    from oracle.bgk import es_gaussian, moments11
    from oracle.fr import velocities
    cfg = _es_cfg('adgfs-ars-111')
    be, s = _system(cfg, 2)
    assert s.sm.nalph == 11 and abs(s.sm._Pr - 2.0 / 3.0) < 1e-15
    _perturb(s, 3)
    f = s.eles_scal_upts_inb_full[0]
    s.get_nregs_moms(3)
    s.moment(0.0, 0, 0)
    s.constructMaxwellian(0.0, 0, 1)
    torch.cuda.synchronize()
    cv = velocities(s.vm.c0())
    Uo = moments11(f.double().cpu().numpy().reshape(-1, cv.shape[1]), cv, s.vm.cw())
    Ug = s.eles_scal_upts_inb_moms[0].cpu().numpy()
    assert Ug.shape == Uo.shape
    assert rel_l2(Ug, Uo) < 1e-13
    Go = es_gaussian(Uo, s.sm._Pr, cv)
    Gg = s.eles_scal_upts_inb_full[1].double().cpu().numpy().reshape(Go.shape)
    assert rel_l2(Gg, Go) < 1e-12


@pytest.mark.parametrize('scheme', ['adgfs-ars-111', 'adgfs-ars-222', 'adgfs-ars-443'])
def test_esbgk_ars_steps_match_oracle(cuda, scheme):
    """Three graph-replayed ES-BGK ARS steps (FP64, Pr = 2/3) vs the oracle."""
    from oracle.bgk import step_ars_es
    from oracle.fr import velocities
    cfg = _es_cfg(scheme)
    nreg = {'adgfs-ars-111': 2, 'adgfs-ars-222': 4, 'adgfs-ars-443': 8}[scheme]
    be, s = _system(cfg, nreg)
    _perturb(s, 4)
    orc = _fr_oracle(s, 'quad', 2)
    cv = velocities(s.vm.c0())
    u = s.eles_scal_upts_inb_full[0].double().cpu().numpy()
    integ = get_integrator(be, s, cfg)
    dt = 2e-3
    for _ in range(3):
        u = step_ars_es(u, dt, orc.rhs, scheme, s.sm._prefactor, s.sm._omega, s.sm._Pr, cv,
                        s.vm.cw())
        integ.step(0.0, dt)
    torch.cuda.synchronize()
    g = s.eles_scal_upts_inb_full[0].double().cpu().numpy()
    assert rel_l2(g, u) < 1e-11


def test_esbgk_single_precision_and_pr_one(cuda):
    """FP32 ES-BGK ARS-222 vs the FP64 oracle; with Pr = 1 the ES-BGK stepper
    gives the BGK result."""
    from oracle.bgk import step_ars, step_ars_es
    from oracle.fr import velocities
    cfg = _es_cfg('adgfs-ars-222', precision='single', Pr=0.8)
    be, s = _system(cfg, 4)
    _perturb(s, 5)
    orc = _fr_oracle(s, 'quad', 2)
    cv = velocities(s.vm.c0())
    u0 = s.eles_scal_upts_inb_full[0].double().cpu().numpy()
    integ = get_integrator(be, s, cfg)
    integ.step(0.0, 2e-3)
    torch.cuda.synchronize()
    uo = step_ars_es(u0, 2e-3, orc.rhs, 'adgfs-ars-222', s.sm._prefactor, s.sm._omega, 0.8,
                     cv, s.vm.cw())
    assert rel_l2(s.eles_scal_upts_inb_full[0].double().cpu().numpy(), uo) < 2e-5
    # Pr = 1: identical to BGK
    cfg1 = _es_cfg('adgfs-ars-222', Pr=1.0)
    be1, s1 = _system(cfg1, 4)
    _perturb(s1, 6)
    orc1 = _fr_oracle(s1, 'quad', 2)
    u1 = s1.eles_scal_upts_inb_full[0].double().cpu().numpy()
    get_integrator(be1, s1, cfg1).step(0.0, 2e-3)
    torch.cuda.synchronize()
    ub = step_ars(u1, 2e-3, orc1.rhs, 'adgfs-ars-222', s1.sm._prefactor, s1.sm._omega, cv,
                  s1.vm.cw())
    assert rel_l2(s1.eles_scal_upts_inb_full[0].double().cpu().numpy(), ub) < 1e-11


def _sk_cfg(scheme, precision='double', Nv=16, dt=2e-3, Pr=None):
    cfg = _cfg(scheme, precision=precision, Nv=Nv, dt=dt)
    cfg.set('scattering-model', 'type', 'shakov-direct-gll')
    if Pr is not None:
        cfg.set('scattering-model', 'Pr', str(Pr))
    return cfg


def test_shakov_moments_and_target_kernels(cuda):
    """'shakov-direct-gll': 14 moments and the Shakov distribution (FP64) vs the oracle."""
    from oracle.bgk import moments14, shakov_target
    from oracle.fr import velocities
    cfg = _sk_cfg('adgfs-ars-111')
    be, s = _system(cfg, 2)
    assert s.sm.nalph == 14 and abs(s.sm._Pr - 2.0 / 3.0) < 1e-15
    _perturb(s, 3)
    f = s.eles_scal_upts_inb_full[0]
    s.get_nregs_moms(3)
    s.moment(0.0, 0, 0)
    s.constructMaxwellian(0.0, 0, 1)
    torch.cuda.synchronize()
    cv = velocities(s.vm.c0())
    Uo = moments14(f.double().cpu().numpy().reshape(-1, cv.shape[1]), cv, s.vm.cw())
    Ug = s.eles_scal_upts_inb_moms[0].cpu().numpy()
    assert Ug.shape == Uo.shape
    assert rel_l2(Ug, Uo) < 1e-13
    So = shakov_target(Uo, s.sm._Pr, cv)
    Sg = s.eles_scal_upts_inb_full[1].double().cpu().numpy().reshape(So.shape)
    assert rel_l2(Sg, So) < 1e-12


@pytest.mark.parametrize('scheme', ['adgfs-ars-111', 'adgfs-ars-222', 'adgfs-ars-443'])
def test_shakov_ars_steps_match_oracle(cuda, scheme):
    """Three graph-replayed Shakov ARS steps (FP64, Pr = 2/3) vs the oracle."""
    from oracle.bgk import step_ars_sk
    from oracle.fr import velocities
    cfg = _sk_cfg(scheme)
    nreg = {'adgfs-ars-111': 2, 'adgfs-ars-222': 4, 'adgfs-ars-443': 8}[scheme]
    be, s = _system(cfg, nreg)
    _perturb(s, 4)
    orc = _fr_oracle(s, 'quad', 2)
    cv = velocities(s.vm.c0())
    u = s.eles_scal_upts_inb_full[0].double().cpu().numpy()
    integ = get_integrator(be, s, cfg)
    dt = 2e-3
    for _ in range(3):
        u = step_ars_sk(u, dt, orc.rhs, scheme, s.sm._prefactor, s.sm._omega, s.sm._Pr, cv,
                        s.vm.cw())
        integ.step(0.0, dt)
    torch.cuda.synchronize()
    g = s.eles_scal_upts_inb_full[0].double().cpu().numpy()
    assert rel_l2(g, u) < 1e-11


def test_shakov_single_precision_and_pr_one(cuda):
    """FP32 Shakov ARS-222 vs the FP64 oracle; with Pr = 1 the Shakov stepper
    gives the BGK result."""
    from oracle.bgk import step_ars, step_ars_sk
    from oracle.fr import velocities
    cfg = _sk_cfg('adgfs-ars-222', precision='single', Pr=0.75)
    be, s = _system(cfg, 4)
    _perturb(s, 5)
    orc = _fr_oracle(s, 'quad', 2)
    cv = velocities(s.vm.c0())
    u0 = s.eles_scal_upts_inb_full[0].double().cpu().numpy()
    get_integrator(be, s, cfg).step(0.0, 2e-3)
    torch.cuda.synchronize()
    uo = step_ars_sk(u0, 2e-3, orc.rhs, 'adgfs-ars-222', s.sm._prefactor, s.sm._omega, 0.75,
                     cv, s.vm.cw())
    assert rel_l2(s.eles_scal_upts_inb_full[0].double().cpu().numpy(), uo) < 2e-5
    cfg1 = _sk_cfg('adgfs-ars-222', Pr=1.0)
    be1, s1 = _system(cfg1, 4)
    _perturb(s1, 6)
    orc1 = _fr_oracle(s1, 'quad', 2)
    u1 = s1.eles_scal_upts_inb_full[0].double().cpu().numpy()
    get_integrator(be1, s1, cfg1).step(0.0, 2e-3)
    torch.cuda.synchronize()
    ub = step_ars(u1, 2e-3, orc1.rhs, 'adgfs-ars-222', s1.sm._prefactor, s1.sm._omega, cv,
                  s1.vm.cw())
    assert rel_l2(s1.eles_scal_upts_inb_full[0].double().cpu().numpy(), ub) < 1e-11


@pytest.mark.parametrize('scheme,model', [
    ('adgfs-bdf-2', 'bgk-direct-gll'), ('adgfs-bdf-3', 'bgk-direct-gll'),
    ('adgfs-bdf-2', 'esbgk-direct-gll'), ('adgfs-bdf-3', 'esbgk-direct-gll'),
    ('adgfs-bdf-2', 'shakov-direct-gll'), ('adgfs-bdf-3', 'shakov-direct-gll')])
def test_bdf_steps_match_oracle(cuda, scheme, model):
    """BDF-2/3 (ARS-222 start-up, then graph-replayed BDF steps over every
    ring phase) vs the oracle stepper, FP64."""
    from oracle.bgk import run_bdf
    from oracle.fr import velocities
    from frfs_b200.integrators import STEPPERS
    q = int(scheme[-1])
    cfg = _cfg(scheme)
    cfg.set('scattering-model', 'type', model)
    be, s = _system(cfg, STEPPERS[scheme].nregs)
    _perturb(s, 8)
    orc = _fr_oracle(s, 'quad', 2)
    cv = velocities(s.vm.c0())
    u0 = s.eles_scal_upts_inb_full[0].double().cpu().numpy()
    integ = get_integrator(be, s, cfg)
    dt, nsteps = 2e-3, q + 3
    for _ in range(nsteps):
        integ.step(0.0, dt)
    torch.cuda.synchronize()
    mdl = {'bgk-direct-gll': 'bgk', 'esbgk-direct-gll': 'esbgk', 'shakov-direct-gll': 'shakov'}[model]
    uo = run_bdf(u0, dt, orc.rhs, nsteps, q, s.sm._prefactor, s.sm._omega, s.sm._Pr, cv, s.vm.cw(),
                 mdl)
    assert rel_l2(integ.soln.double().cpu().numpy(), uo) < 1e-11


def test_bdf_reference_methods_equal_fused_step(cuda):
    """updateMomentBDF + updateDistBDF (the reference's calls, BDF2 order of
    arguments) give the fused bdgfs_bdf_step's result."""
    from frfs_b200.adgfs import BDF_DIST, BDF_MOMN, BDF_MOMU
    from frfs_b200.integrators import BDF2AstdStepper as B
    cfg = _es_cfg('adgfs-bdf-2')
    be, s = _system(cfg, 6)
    _perturb(s, 9)
    s.get_nregs_moms(6)
    s.eles_scal_upts_inb_full[1].copy_(s.eles_scal_upts_inb_full[0] * 0.97)
    s.advect_combine(0.0, 0, 2, a=0.0, b=1.0)
    s.advect_combine(0.0, 1, 3, a=0.0, b=1.0)
    for f, m in ((0, 0), (2, 1), (1, 2), (3, 3)):
        s.moment(0.0, f, m)
    a, g, b, dt = B.bdf_A, [-x for x in B.bdf_G], B.bdf_B, 2e-3
    # reference order: f_0 = bank 1 (older), f_1 = bank 0 (newer)
    s.updateMomentBDF(dt, a[0], 2, g[0], 3, a[1], 0, g[1], 1, a[2], 4, b)
    s.updateDistBDF(dt, a[0], 1, g[0], 3, a[1], 0, g[1], 2, b, None, a[2], 4, 4)
    ref = s.eles_scal_upts_inb_full[4].clone()
    Uref = s.eles_scal_upts_inb_moms[4].clone()
    s.bdf_step(dt, 2, BDF_MOMN | BDF_MOMU | BDF_DIST, a, g, b, [1, 0], 5, [3, 2], [2, 0], [3, 1], 5)
    torch.cuda.synchronize()
    assert torch.equal(s.eles_scal_upts_inb_moms[5], Uref)
    assert torch.equal(s.eles_scal_upts_inb_full[5], ref)


@pytest.mark.parametrize('model', ['bgk', 'esbgk', 'shakov'])
@pytest.mark.parametrize('scheme', ['adgfs-ars-111', 'adgfs-ars-222', 'adgfs-ars-443'])
def test_ars_stages_equal_reference_kernels(cuda, model, scheme):
    """bdgfs_ars_stage, driven stage by stage as the reference's ARS stepper
    (frfs/integrators/std/steppers.py:538-585) with a given explicit part
    L, against the reference's own bgk-, esbgk- and shakov-direct-gll
    kernels (golden vectors of tests/golden/make_reference_ars.py): FP64,
    relative to the change the step makes."""
    import ctypes as C
    import os
    import sys
    from frfs_b200 import _lib
    from oracle.bgk import ARS
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), 'golden'))
    from make_reference_ars import grid, inputs
    d = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'reference_ars.npz'))
    cv, cw = grid()
    rows = d['rows']
    f0, L = inputs(cv)
    f0, L = f0[rows], L[rows]
    Nv, n = 16, f0.shape[0]
    dev = torch.device('cuda')
    nalph = {'bgk': 5, 'esbgk': 11, 'shakov': 14}[model]
    c0 = torch.as_tensor(np.linspace(-5 + 5 / Nv, 5 - 5 / Nv, Nv), dtype=torch.float64, device=dev)
    F = [torch.as_tensor(f0, device=dev)]
    Ld = torch.as_tensor(L, device=dev)
    U = [torch.zeros(n, nalph, dtype=torch.float64, device=dev) for _ in range(5)]
    LU = [torch.zeros(n, nalph, dtype=torch.float64, device=dev) for _ in range(4)]
    _A, A = ARS[scheme]
    s = len(_A) - 1
    for i in range(s):
        ar = i + 1
        F.append(torch.empty_like(F[0]))
        a = _lib.ArsArgs(ndof=n, Nv=Nv, fp64=1, c0=c0.data_ptr(), cw=cw, prefac=float(d['prefac']),
                         omega=0.81, dt=float(d['dt']), stage=ar,
                         flags=(1 if ar == 1 else 0) | 2 | 4 | 8,
                         model={'bgk': 0, 'esbgk': 1, 'shakov': 2}[model],
                         Pr=1.0 if model == 'bgk' else 2.0 / 3.0)
        for j in range(ar):
            a.ae[j] = _A[ar][j]
            a.ai[j] = A[ar][j + 1]
            a.f[j] = F[j].data_ptr()
            a.L[j] = Ld.data_ptr()
            a.LU[j] = LU[j].data_ptr()
        for j in range(ar + 1):
            a.U[j] = U[j].data_ptr()
        a.fout = F[ar].data_ptr()
        _lib.check(_lib.lib().bdgfs_ars_stage(C.byref(a), _lib.stream_ptr()), 'bdgfs_ars_stage')
    torch.cuda.synchronize()
    got = F[s].cpu().numpy()
    want = d[f'{model}:{scheme}']
    err = np.linalg.norm(got - want) / np.linalg.norm(want - f0)
    print(f'{model} {scheme}: {err:.1e}')
    assert err < 1e-12


@pytest.mark.parametrize('model', ['bgk', 'esbgk', 'shakov'])
@pytest.mark.parametrize('q', [2, 3])
def test_bdf_step_equals_reference_kernels(cuda, model, q):
    """bdgfs_bdf_step (moments of the newest history level reduced in the
    launch, the others given) against the reference's own BDF-q update
    kernels (golden vectors of tests/golden/make_reference_ars.py): new
    distribution and moments, FP64."""
    import ctypes as C
    import os
    import sys
    from frfs_b200 import _lib
    from oracle.bgk import BDF, MODELS
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), 'golden'))
    from make_reference_ars import bdf_inputs, grid
    d = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'reference_ars.npz'))
    cv, cw = grid()
    rows = d['rows']
    fs, Ls = bdf_inputs(cv, q)
    fs, Ls = fs[:, rows], Ls[:, rows]
    Nv, n = 16, fs.shape[1]
    dev = torch.device('cuda')
    mom = MODELS[model][0]
    c0 = torch.as_tensor(np.linspace(-5 + 5 / Nv, 5 - 5 / Nv, Nv), dtype=torch.float64, device=dev)
    F = [torch.as_tensor(x, device=dev) for x in fs]
    Ld = [torch.as_tensor(x, device=dev) for x in Ls]
    U = [torch.as_tensor(mom(x, cv, cw), device=dev) for x in fs]
    LU = [torch.as_tensor(mom(x, cv, cw), device=dev) for x in Ls]
    U[-1].zero_()
    LU[-1].zero_()                               # reduced by the launch (MOMN)
    Unew = torch.zeros_like(U[0])
    fout = torch.empty_like(F[0])
    A, G, b, _ = BDF[q]
    x = _lib.BdfArgs(ndof=n, Nv=Nv, fp64=1, c0=c0.data_ptr(), cw=cw, prefac=float(d['prefac']), omega=0.81,
                     dt=float(d['dt']), q=q, model={'bgk': 0, 'esbgk': 1, 'shakov': 2}[model],
                     Pr=1.0 if model == 'bgk' else 2.0 / 3.0, b=b, Unew=Unew.data_ptr(),
                     fout=fout.data_ptr(), flags=1 | 2 | 4)
    for i in range(q + 1):
        x.a[i] = A[i]
    for i in range(q):
        x.g[i] = -G[i]
        x.f[i] = F[i].data_ptr()
        x.L[i] = Ld[i].data_ptr()
        x.U[i] = U[i].data_ptr()
        x.LU[i] = LU[i].data_ptr()
    _lib.check(_lib.lib().bdgfs_bdf_step(C.byref(x), _lib.stream_ptr()), 'bdgfs_bdf_step')
    torch.cuda.synchronize()
    wf, wU = d[f'{model}:bdf{q}:f'], d[f'{model}:bdf{q}:U']
    ef = np.linalg.norm(fout.cpu().numpy() - wf) / np.linalg.norm(wf - fs[-1])
    eU = np.abs(Unew.cpu().numpy() - wU).max() / np.abs(wU).max()
    print(f'{model} BDF-{q}: f {ef:.1e}, U {eU:.1e}')
    assert ef < 1e-12 and eU < 1e-13
