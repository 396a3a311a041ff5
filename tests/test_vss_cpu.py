"""Gas mixtures on the host: the 'vss-gll' model's mesh, parameters and
kernel tables against the oracle, and the oracle's own properties."""
import numpy as np
import pytest
import torch

from frfs_b200.dgfsbi import DGFSBiVelocityMesh, DGFSBiVSSGLLScatteringModel

from helpers import mixture, vss_cfg, vss_oracle_for
from test_host_structs import _CPUBackend


class _Model(DGFSBiVSSGLLScatteringModel):
    """Parameters and tables only (no device upload)."""
    def perform_precomputation(self):
        pass


def _model(Nv=8, Nrho=4, M=6, Mpre=12, **kw):
    cfg = vss_cfg(Nv, Nrho, M, Mpre, **kw)
    be = _CPUBackend()
    vm = DGFSBiVelocityMesh(be, cfg, 2)
    return _Model(be, cfg, vm)


def test_mesh_and_tables_match_oracle():
    sm = _model()
    o = vss_oracle_for(sm)
    vm = sm.vm
    assert np.isclose(vm.L(), o.vm.L) and np.isclose(vm._R, o.vm.R)
    assert np.allclose(vm.qz(), o.vm.qz) and np.allclose(vm.qw(), o.vm.qw)
    assert vm.sz().shape == (6, 3) and np.isclose(vm.sw(), 4 * np.pi / 6)
    for p in range(2):
        for q in range(2):
            assert sm._prefactor[f'{p}{q}'] == pytest.approx(o.par[(p, q)]['prefac'], rel=1e-14)
            b, c = sm.kernel_tables(p, q)
            assert np.allclose(b, o.b[(p, q)], rtol=0, atol=1e-12 * np.abs(o.b[(p, q)]).max())
            assert np.allclose(c, o.c[(p, q)], rtol=0, atol=1e-12 * np.abs(o.c[(p, q)]).max())


def test_full_sphere_designs_are_antipodal():
    from frfs_b200.sphericaldesign import full_sphere_design
    for M in (2, 6, 12, 24):
        s = full_sphere_design(M)
        assert s.shape == (M, 3) and np.allclose(np.linalg.norm(s, axis=1), 1.0)
        assert np.allclose(s[:M // 2], -s[M // 2:])
    with pytest.raises(ValueError):
        full_sphere_design(5)


def test_oracle_mixture_equilibrium_and_conservation():
    """Q of Maxwellians with a common u and T is small, and the mixture
    conserves mass per species, total momentum and energy to the
    resolution of the spectral method (they fall as the grid is refined)."""
    errs = []
    for Nv, Nrho, M, Mpre in ((12, 6, 12, 12), (16, 8, 24, 24)):
        sm = _model(Nv, Nrho, M, Mpre)
        o = vss_oracle_for(sm)
        cv, cw, m = o.vm.cv, o.vm.cw, o.vm.masses
        u = np.array([0.1, -0.05, 0.0])[:, None]
        feq = [n * (mp / np.pi)**1.5 * np.exp(-mp * np.sum((cv - u)**2, axis=0))
               for n, mp in zip((1.0, 0.5), m)]
        Qe = o.Q(feq)
        fs = mixture(cv, m, np.random.default_rng(3))
        Q = o.Q(fs)
        sc = sum(np.abs(Qp).sum() * cw for Qp in Q)
        mass = max(abs(Q[p].sum() * cw) for p in range(2)) / sc
        mom = np.abs(sum(m[p] * (cv @ Q[p]) * cw for p in range(2))).max() / sc
        en = abs(sum(m[p] * (np.sum(cv * cv, 0) @ Q[p]) * cw for p in range(2))) / sc
        eq = max(np.abs(Qe[p]).max() / feq[p].max() for p in range(2))
        errs.append((eq, mass, mom, en))
    assert all(x < 0.06 for x in errs[1])
    assert errs[1][0] < errs[0][0] and errs[1][3] < errs[0][3]


def _bi_cfg(**kw):
    from helpers import dgfsbi_cfg
    return dgfsbi_cfg(**kw)


def test_dgfsbi_maxwellian_and_support_check():
    """Per-species Maxwellians n_p (m_p/(pi T))^1.5 exp(-m_p |c-u|^2/T) with
    the reference's moment check; a grid too coarse for the heavy species
    is refused."""
    from frfs_b200.dgfsbi import DGFSBiMaxwellianInitCondition
    cfg = _bi_cfg()
    vm = DGFSBiVelocityMesh(_CPUBackend(), cfg, 2)
    ic = DGFSBiMaxwellianInitCondition(None, cfg, vm, 'soln-ics')
    cv, cw, m = vm.cv(), vm.cw(), vm.masses()
    for p, f in enumerate(ic.get_init_vals()):
        assert np.isclose(f.sum() * cw, 0.7 if p else 0.3, rtol=1e-6)
        T = (2.0 / 3.0) * m[p] * np.sum(f * np.sum(cv * cv, axis=0)) * cw / (f.sum() * cw)
        assert np.isclose(T, 1.0, rtol=1e-6)
    wall = DGFSBiMaxwellianInitCondition(None, cfg, vm, 'soln-bcs-y+', wall=True)
    fw = wall.get_init_vals()
    assert np.isclose(fw[1].sum() * cw, 1.0, rtol=1e-6)
    assert np.isclose(wall.unondim()[0, 0], 0.3)
    coarse = _bi_cfg(Nv=8, dev=6)
    with pytest.raises(ValueError):
        DGFSBiMaxwellianInitCondition(None, coarse, DGFSBiVelocityMesh(_CPUBackend(), coarse, 2),
                                      'soln-ics')


def test_dgfsbi_species_wall_rows():
    """Each species' diffuse-wall rows carry its own wall Maxwellian; the
    boundary tables of the 'dgfsbi' types resolve on the host."""
    from frfs_b200.dgfsbi import SpeciesMesh
    from frfs_b200.mesh import ElementGeometry, StructuredMesh
    from frfs_b200.system import DGFSBoundaries
    cfg = _bi_cfg()
    be = _CPUBackend()
    be.fpdtype = torch.float64
    vm = DGFSBiVelocityMesh(be, cfg, 2)
    geo = ElementGeometry(StructuredMesh((2, 2), (0.0, -0.5), (1.0, 0.5), periodic='x'), 2)
    walls = [DGFSBoundaries(be, geo, SpeciesMesh(vm, p), cfg, geo.wall_names) for p in range(2)]
    cv, m = vm.cv(), vm.masses()
    for p, w in enumerate(walls):
        fw = w.fw.numpy()
        U = w.uwall.numpy()
        for r in range(fw.shape[0]):
            T = 1.1 if U[r, 0] > 0 else 1.0
            want = (m[p] / (np.pi * T))**1.5 * np.exp(-m[p] * np.sum((cv - U[r][:, None])**2, 0) / T)
            assert np.allclose(fw[r], want, rtol=1e-12, atol=0)
        assert w.has_diffuse


def test_dgfsbi_steppers_registered():
    from frfs_b200.integrators import STEPPERS
    assert STEPPERS['dgfsbi-tvd-rk2'].nregs == 3 and STEPPERS['dgfsbi-euler'].nregs == 2


def test_mixture_gram_inverse_projects_like_the_oracle():
    """The host Gram inverse of the device projection gives the oracle's
    least-squares projection (numpy, both species)."""
    from frfs_b200.dgfsbi import mixture_gram_inverse
    from oracle.vss import project_mixture
    sm = _model()
    o = vss_oracle_for(sm)
    cv, m = o.vm.cv, o.vm.masses
    rng = np.random.default_rng(2)
    Q = [rng.standard_normal(cv.shape[1]) for _ in m]
    Gi = mixture_gram_inverse(sm.vm.c0(), m)
    S = len(m)
    c2 = np.sum(cv * cv, 0)
    r = np.array([q.sum() for q in Q] + [sum(mp * (phi @ q) for mp, q in zip(m, Q))
                                         for phi in (cv[0], cv[1], cv[2], c2)])
    lam = Gi @ r
    got = [q - (lam[p] + m[p] * (lam[S] * cv[0] + lam[S + 1] * cv[1] + lam[S + 2] * cv[2]
                                 + lam[S + 3] * c2)) for p, q in enumerate(Q)]
    want = project_mixture(Q, cv, m)
    assert all(np.allclose(g, w, rtol=0, atol=1e-12) for g, w in zip(got, want))


def test_dgfsbi_other_boundary_types_resolve():
    """Inlet rows carry each species' nden{p+1} Maxwellian, the normal-shock
    inlet the same row with zero velocity shift; outlet / vanish / specular
    resolve to their kernel kinds for every species."""
    from frfs_b200 import _lib
    from frfs_b200.dgfsbi import SpeciesMesh
    from frfs_b200.mesh import ElementGeometry, StructuredMesh
    from frfs_b200.system import DGFSBoundaries
    cfg = _bi_cfg()
    n0 = DGFSBiVelocityMesh(_CPUBackend(), cfg, 2).n0()
    u0 = DGFSBiVelocityMesh(_CPUBackend(), cfg, 2).u0()
    for name, t in (('x-', 'dgfsbi-inlet'), ('x+', 'dgfsbi-outlet'),
                    ('y-', 'dgfsbi-wall-specular'), ('y+', 'dgfsbi-inlet-normalshock')):
        cfg.set(f'soln-bcs-{name}', 'type', t)
        for k, v in (('nden1', 0.2 * n0), ('nden2', 0.9 * n0), ('T', 273.0 * 1.2),
                     ('ux', 0.1 * u0), ('uy', 0.0), ('uz', 0.0)):
            cfg.set(f'soln-bcs-{name}', k, repr(float(v)))
    be = _CPUBackend()
    be.fpdtype = torch.float64
    vm = DGFSBiVelocityMesh(be, cfg, 2)
    geo = ElementGeometry(StructuredMesh((2, 2), (0.0, -0.5), (1.0, 0.5)), 2)
    cv, m, cw = vm.cv(), vm.masses(), vm.cw()
    for p in range(2):
        w = DGFSBoundaries(be, geo, SpeciesMesh(vm, p), cfg, geo.wall_names)
        kinds = dict(zip(w.types, w.kind.tolist()))
        assert kinds['dgfsbi-outlet'] == _lib.BC_OUTLET
        assert kinds['dgfsbi-inlet'] == _lib.BC_INLET == kinds['dgfsbi-inlet-normalshock']
        assert kinds['dgfsbi-wall-specular'] == _lib.BC_SPECULAR_X + 1
        r = w.types.index('dgfsbi-inlet')
        want = (0.9 if p else 0.2) * (m[p] / (np.pi * 1.2))**1.5 * np.exp(
            -m[p] * np.sum((cv - np.array([[0.1], [0.0], [0.0]]))**2, 0) / 1.2)
        assert np.allclose(w.fw[r].numpy(), want, rtol=1e-12, atol=0)
        assert np.isclose(w.fw[r].numpy().sum() * cw, 0.9 if p else 0.2, rtol=1e-6)
        rs = w.types.index('dgfsbi-inlet-normalshock')
        assert np.allclose(w.fw[rs].numpy(), want) and not w.uwall[rs].any()
