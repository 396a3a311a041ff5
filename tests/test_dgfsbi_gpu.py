"""GPU parity of the 'dgfsbi' gas-mixture system (per-species FR advection,
species walls, mixture collisions, dgfsbi-euler / dgfsbi-tvd-rk2) against
the FP64 oracle: oracle.fr per species with that species' wall rows and
oracle.vss for Q_p = sum_q Q_pq."""
import numpy as np
import pytest
import torch

from frfs_b200.backend import CUDABackend
from frfs_b200.dgfsbi import DGFSBiSystem
from frfs_b200.integrators import get_integrator
from frfs_b200.mesh import StructuredMesh

from helpers import dgfsbi_cfg, rel_l2, vss_oracle_for

pytestmark = pytest.mark.gpu

GOLD = __import__('os').path.join(__import__('os').path.dirname(__file__), 'golden')


def _system(precision='double', scheme='dgfsbi-tvd-rk2', nreg=3):
    cfg = dgfsbi_cfg(precision=precision, scheme=scheme)
    be = CUDABackend(cfg)
    mesh = StructuredMesh((2, 2), (0.0, -0.5), (1.0, 0.5), periodic='x')
    return cfg, be, DGFSBiSystem(be, mesh, cfg, nreg=nreg)


def _perturb(s, seed):
    """Non-uniform, non-equilibrium start: a smooth spatial modulation that
    differs per species and velocity."""
    rng = np.random.default_rng(seed)
    x = s.geo.plocupts
    for p, sp in enumerate(s.species):
        u = sp.eles_scal_upts_inb_full[0]
        amp = 0.2 * np.sin(2 * np.pi * x[..., 0] + p) + 0.1 * np.cos(np.pi * x[..., 1])
        vel = rng.uniform(-0.3, 0.3, size=u.shape[-1])
        u.mul_(torch.from_numpy(1.0 + amp[..., None] * (1.0 + vel[None, None, :])).to(u))


def _oracles(s):
    from oracle.fr import FROracle
    g = np.load(f'{GOLD}/shapes_quad_p2.npz')
    ops = {'M0': g['M0'], 'M132': g['M132'], 'M3': g['M3']}
    frs = []
    for sp in s.species:
        walls, rows = sp.walls.oracle_walls()
        frs.append(FROracle(ops, s.geo, s.vm.c0(), s.vm.cw(), walls, bcid=rows))
    return frs, vss_oracle_for(s.sm)


def _state(s, reg=0):
    return [sp.eles_scal_upts_inb_full[reg].double().cpu().numpy() for sp in s.species]


def _oracle_step(us, dt, frs, vo, scheme):
    S = len(us)
    E, U = us[0].shape[:2]

    def Q(fs):
        out = [np.empty_like(f) for f in fs]
        for e in range(E):
            for j in range(U):
                q = vo.Q([f[e, j] for f in fs])
                for p in range(S):
                    out[p][e, j] = q[p]
        return out
    q0 = Q(us)
    u1 = [us[p] + dt * frs[p].rhs(us[p]) + dt * q0[p] for p in range(S)]
    if scheme == 'dgfsbi-euler':
        return u1
    q1 = Q(u1)
    return [0.5 * us[p] + 0.5 * u1[p] + 0.5 * dt * (frs[p].rhs(u1[p]) + q1[p]) for p in range(S)]


@pytest.mark.parametrize('scheme,nsteps,prec,tol', [
    ('dgfsbi-tvd-rk2', 2, 'double', 1e-11), ('dgfsbi-euler', 2, 'double', 1e-11),
    ('dgfsbi-tvd-rk2', 2, 'single', 1e-5)])
def test_dgfsbi_steps_match_oracle(cuda, scheme, nsteps, prec, tol):
    """Graph-replayed mixture steps against the oracle stepper: each species
    advected with its own diffuse-wall Maxwellians (its mass), coupled by
    Q_p = sum_q Q_pq."""
    cfg, be, s = _system(prec, scheme)
    _perturb(s, 4)
    frs, vo = _oracles(s)
    us = _state(s)
    integ = get_integrator(be, s, cfg)
    dt = 2e-4
    for _ in range(nsteps):
        us = _oracle_step(us, dt, frs, vo, scheme)
        integ.step(integ.tcurr, dt)
        integ.tcurr += dt
    torch.cuda.synchronize()
    got = _state(s)
    assert max(rel_l2(got[p], us[p]) for p in range(len(us))) < tol


def test_dgfsbi_reference_calls_equal_fused_stage(cuda):
    """The reference's call sequence per species -- collide(t, regids),
    updatebc(t, idx, ...), rhs(t, idx, ...) -- gives the same L_p and Q_p
    as the fused stage; walls differ per species (their masses)."""
    cfg, be, s = _system()
    _perturb(s, 9)
    s.collide(0.0, [0, 0, 1, 1])                 # r1_p = Q_p(r0)
    Qa = _state(s, 1)
    s.collide_banks(0.0, 0, 2)
    assert all(np.array_equal(a, b) for a, b in zip(Qa, _state(s, 2)))
    frs, _ = _oracles(s)
    u = _state(s)
    for p in range(s.nspcs()):
        s.updatebc(0.0, str(p), 0, 1)
        s.rhs(0.0, str(p), 0, 1)
        assert rel_l2(_state(s, 1)[p], frs[p].rhs(u[p])) < 1e-12
    fw = [sp.walls.fw.double().cpu().numpy() for sp in s.species]
    assert not np.allclose(fw[0], fw[1])


def test_dgfsbi_initial_moments(cuda):
    """The 'maxwellian' start holds each species' number density (nden over
    n0), zero velocity and T = 1 to the reference's support tolerance."""
    cfg, be, s = _system()
    mom = s.moments(0)
    for p, (n, U, T) in enumerate(mom):
        assert torch.allclose(n, torch.full_like(n, 0.7 if p else 0.3), rtol=1e-6, atol=0)
        assert float(U.abs().max()) < 1e-10
        assert torch.allclose(T, torch.ones_like(T), rtol=1e-6, atol=0)


def test_dgfsbi_partitioned_virtual_ranks_equal_single_domain(cuda):
    """Three slab parts of the mixture, stepped stage by stage with the
    in-process halo exchange of every species, reproduce the single-domain
    SSP-RK2 steps exactly."""
    from frfs_b200.partition import bind_local_transports_bi, slab_partition, step_rk2_virtual_bi
    cfg = dgfsbi_cfg(precision='single')
    be = CUDABackend(cfg)
    mesh = StructuredMesh((6, 2), (0.0, -0.5), (1.0, 0.5), periodic='x')
    s = DGFSBiSystem(be, mesh, cfg, nreg=3)
    _perturb(s, 6)
    parts = slab_partition(mesh, 3)
    systems = [DGFSBiSystem(be, mesh, cfg, nreg=3, partition=(parts, r)) for r in range(3)]
    bind_local_transports_bi(systems)
    for r, b in enumerate(systems):
        idx = torch.as_tensor(parts[r], device=be.device)
        for p in range(s.nspcs()):
            b.bank(p, 0).copy_(s.bank(p, 0).index_select(0, idx))
    integ = get_integrator(be, s, cfg)
    integ.use_graph = False
    for _ in range(2):
        integ.step(0.0, 5e-4)
        step_rk2_virtual_bi(systems, 5e-4)
    torch.cuda.synchronize()
    for r, b in enumerate(systems):
        idx = torch.as_tensor(parts[r], device=be.device)
        for p in range(s.nspcs()):
            assert torch.equal(b.bank(p, 0), s.bank(p, 0).index_select(0, idx)), (r, p)


def test_dgfsbi_macroscopic_matches_oracle(cuda):
    """The mixture moment writer's fields (per species rho, U, T, heat flux
    and pressure tensor about the mixture velocity) from the FP64 device
    moments equal the oracle's on a perturbed state."""
    from oracle.vss import mixture_moments
    cfg, be, s = _system()
    _perturb(s, 13)
    got, mix = s.macroscopic(0)
    us = _state(s)
    cv, cw, m = s.vm.cv(), s.vm.cw(), s.vm.masses()
    E, U = us[0].shape[:2]
    for e in range(E):
        for j in range(U):
            want, wmix = mixture_moments([u[e, j] for u in us], cv, cw, m)
            d = e * U + j
            assert np.isclose(float(mix['rho'][d]), wmix['rho'], rtol=1e-12)
            assert np.allclose(mix['U'][d].cpu().numpy(), wmix['U'], rtol=0, atol=1e-12)
            for p in range(len(us)):
                for k in ('rho', 'T', 'nden'):
                    assert np.isclose(float(got[p][k][d]), want[p][k], rtol=1e-12), k
                for k in ('U', 'q', 'P'):
                    w = np.asarray(want[p][k])
                    assert np.allclose(got[p][k][d].cpu().numpy(), w, rtol=0,
                                       atol=1e-11 * max(1.0, np.abs(w).max())), k


def test_dgfsbi_residual_per_species(cuda):
    """The residual plugin's value per species: ||f_p - f_p,prev|| / ||f_p,prev||."""
    cfg, be, s = _system()
    cfg.set('soln-plugin-dgfsresidualbi', 'nsteps', '1')
    _perturb(s, 21)
    integ = get_integrator(be, s, cfg)
    before = _state(s)
    integ.advance_to(2e-4)
    after = _state(s)
    (t, res), = integ.residuals
    want = [np.linalg.norm(a - b) / np.linalg.norm(b) for a, b in zip(after, before)]
    assert len(res) == 2 and np.allclose(res, want, rtol=1e-10, atol=0)


@pytest.mark.parametrize('prec,tol', [('double', 1e-13), ('single', 1e-6)])
def test_dgfsbi_maxwellian_expr_initial_condition(cuda, prec, tol):
    """'maxwellianExpr': every solution point of species p holds
    nden_p (m_p/(pi T))^1.5 exp(-m_p |c-u|^2/T) of the expressions there."""
    cfg = dgfsbi_cfg(precision=prec)
    u0 = np.sqrt(2 * 8.3144598 / 39.96e-3 * 273.0)
    n0 = 0.00011140244750324529 / 39.96e-3 * 6.0221409e+23
    cfg.set('constants', 'n0', repr(n0))
    for k, v in (('type', 'maxwellianExpr'), ('nden1', 'n0*0.3*(1 + 0.1*sin(2*pi*x))'),
                 ('nden2', 'n0*0.7*(1 - 0.05*y)'), ('ux', f'{0.1 * u0}*y'),
                 ('uy', f'{0.05 * u0}*x'), ('uz', '0'), ('T', '273*(1 + 0.05*x)')):
        cfg.set('soln-ics', k, v)
    be = CUDABackend(cfg)
    s = DGFSBiSystem(be, StructuredMesh((3, 2), (0.0, -0.5), (1.0, 0.5), periodic='x'), cfg)
    torch.cuda.synchronize()
    cv, m = s.vm.cv(), s.vm.masses()
    pl = s.geo.plocupts
    for p in range(2):
        want = np.empty((pl.shape[0], pl.shape[1], cv.shape[1]))
        for e in range(pl.shape[0]):
            for j in range(pl.shape[1]):
                x, y = pl[e, j]
                n = 0.3 * (1 + 0.1 * np.sin(2 * np.pi * x)) if p == 0 else 0.7 * (1 - 0.05 * y)
                u = np.array([0.1 * y, 0.05 * x, 0.0])[:, None]
                T = 1 + 0.05 * x
                want[e, j] = n * (m[p] / (np.pi * T))**1.5 * np.exp(-m[p] * np.sum((cv - u)**2, 0) / T)
        assert rel_l2(s.bank(p, 0).double().cpu().numpy(), want) < tol


def test_dgfsbi_nancheck_covers_every_species(cuda):
    cfg, be, s = _system(precision='single')
    cfg.set('soln-plugin-nancheck', 'nsteps', '1')
    integ = get_integrator(be, s, cfg)
    integ.advance_to(2e-4)
    integ.nancheck()
    s.bank(1, integ._idxcurr)[0, 0, 5] = float('inf')
    with pytest.raises(RuntimeError, match='NaNs detected'):
        integ.nancheck()
