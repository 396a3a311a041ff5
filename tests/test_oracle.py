"""The oracle against the reference's own outputs (golden fixtures) and
known-answer properties of the collision operator."""
import os

import numpy as np
import pytest

from oracle.velocitymesh import VelocityMesh, gauss_jacobi
from oracle.vhs import VHSOracle, precompute, vhs_prefactor

from helpers import NONDIM, maxwellian, mixed_maxwellians, rel_l2

GOLD = os.path.join(os.path.dirname(__file__), 'golden')


def _vm(name):
    g = np.load(f'{GOLD}/vmesh_{name}.npz')
    dev = {'c1': 5, 'nv8': 5, 'm16': 6}[name]
    vm = VelocityMesh(int(g['Nv']), int(g['Nrho']), g['sz'], cmax=0.0, Tmax=NONDIM['T0'],
                      dev=dev, **NONDIM)
    return vm, g


@pytest.mark.parametrize('name', ['c1', 'nv8', 'm16'])
def test_velocity_mesh_matches_reference(name):
    vm, g = _vm(name)
    assert np.array_equal(vm.cv, g['cv'])
    assert vm.cw == float(g['cw']) and vm.L == float(g['L'])
    assert np.allclose(vm.qz, g['qz'], rtol=0, atol=1e-14)
    assert np.allclose(vm.qw, g['qw'], rtol=0, atol=1e-14)
    assert vm.sw == float(g['sw'])
    assert np.isclose(vm.u0, float(g['u0'])) and np.isclose(vm.n0, float(g['n0']))


def test_gauss_jacobi_matches_reference():
    d = np.load(f'{GOLD}/sphdesign.npz')
    for n in (8, 12):
        z, w = gauss_jacobi(n)
        assert np.allclose(z, d[f'gj{n}_z'], atol=1e-14)
        assert np.allclose(w, d[f'gj{n}_w'], atol=1e-14)


def test_vhs_tables_match_reference_numpy_formulation():
    vm, _ = _vm('nv8')
    p = np.load(f'{GOLD}/vhs_precompute_nv8.npz')
    aa, bb1, bb2 = precompute(vm, float(p['gamma']))
    assert np.abs(aa.ravel() - p['aa']).max() < 1e-13
    assert np.abs(bb1.ravel() - p['bb1']).max() < 1e-13 * np.abs(p['bb1']).max()
    assert np.abs(bb2 - p['bb2']).max() < 1e-13 * np.abs(p['bb2']).max()


def test_maxwellian_and_bkw_initial_values_match_reference():
    from oracle.fr import velocities
    vm, g = _vm('c1')
    ic = np.load(f'{GOLD}/initcond.npz')
    f = maxwellian(vm.cv, float(ic['rho']), ic['u'], float(ic['T']))
    assert np.allclose(f, ic['maxwellian'], rtol=1e-13, atol=0)
    K = 1.0 - np.exp(-float(ic['bkw_t0']) / 6.0)
    c2 = np.sum(vm.cv**2, axis=0)
    bkw = 1 / (2 * (2 * np.pi * K)**1.5) * np.exp(-c2 / (2 * K)) * ((5 * K - 3) / K + (1 - K) / K**2 * c2)
    assert np.allclose(bkw, ic['bkw'], rtol=1e-13, atol=1e-300)


@pytest.fixture(scope='module')
def c1_oracle():
    vm, _ = _vm('c1')
    return vm, VHSOracle(vm, 0.5, 4.17e-10, 273.0)


def test_prefactor_formula(c1_oracle):
    vm, orc = c1_oracle
    gam, pref, Kn = vhs_prefactor(vm, 0.81, 4.17e-10, 273.0)
    assert np.isclose(gam, 0.38) and Kn > 0 and pref > 0
    # hard sphere: gamma = 1
    assert np.isclose(orc.gamma, 1.0)


def test_q_maxwellian_is_spectrally_small(c1_oracle):
    vm, orc = c1_oracle
    f = maxwellian(vm.cv, 1.0, [0.1, -0.05, 0.0], 1.0)
    gain, loss = orc.gain_loss(f)
    assert np.linalg.norm(orc.Q(f)) < 1e-3 * np.linalg.norm(loss)


def test_q_conserves_mass_momentum_energy(c1_oracle):
    vm, orc = c1_oracle
    rng = np.random.default_rng(0)
    f = mixed_maxwellians(vm.cv, rng, k=2, nrange=(0.5, 1.5), umax=0.5, Trange=(0.7, 1.3),
                          noise=0.0)
    q = orc.Q(f)
    gain, loss = orc.gain_loss(f)
    scale = np.abs(loss).sum() * vm.cw
    c2 = np.sum(vm.cv**2, axis=0)
    for phi in (np.ones_like(c2), vm.cv[0], vm.cv[1], vm.cv[2], c2):
        assert abs(np.sum(phi * q) * vm.cw) < 2e-3 * scale * (1 + np.abs(phi).max())


def test_q_commutes_with_axis_reflection(c1_oracle):
    """Reflecting c_y -> -c_y maps the icosahedral half-sphere design onto
    itself (up to antipodes), so Q commutes with the reflection up to the
    reference's Nyquist-plane asymmetry (l0 holds -N/2 but not +N/2)."""
    vm, orc = c1_oracle
    rng = np.random.default_rng(4)
    N = vm.Nv
    f = mixed_maxwellians(vm.cv, rng, k=2, nrange=(0.5, 1.5), umax=0.5, Trange=(0.7, 1.3),
                          noise=0.0)
    fr = f.reshape(N, N, N)[:, ::-1, :].ravel()        # c_y -> -c_y
    q = orc.Q(f).reshape(N, N, N)[:, ::-1, :].ravel()
    assert rel_l2(orc.Q(fr), q) < 1e-4


def test_bkw_known_answer():
    """Maxwell molecules (omega = 1, gamma = 0): Q(f_BKW(t)) is the time
    derivative of the BKW solution for the operator's own time scale.  With
    the reference normalisation, Q(f) / (df/dt) is one constant; check that
    Q is proportional to the analytic derivative to 2%."""
    dev = 7
    sz = np.load(f'{GOLD}/vmesh_c1.npz')['sz']
    vm = VelocityMesh(24, 12, sz, cmax=0.0, Tmax=NONDIM['T0'], dev=dev, **NONDIM)
    orc = VHSOracle(vm, 1.0, 4.17e-10, 273.0)
    c2 = np.sum(vm.cv**2, axis=0)

    def bkw(t):
        K = 1.0 - np.exp(-t / 6.0)
        return (1 / (2 * (2 * np.pi * K)**1.5) * np.exp(-c2 / (2 * K))
                * ((5 * K - 3) / K + (1 - K) / K**2 * c2))
    t0, h = 5.5, 1e-4
    dfdt = (bkw(t0 + h) - bkw(t0 - h)) / (2 * h)
    q = orc.Q(bkw(t0))
    scale = np.dot(q, dfdt) / np.dot(dfdt, dfdt)
    assert scale > 0
    assert rel_l2(q, scale * dfdt) < 2e-2


def test_fr_oracle_velocity_restriction_and_wall_sums():
    """The restricted FR oracle on a velocity subset, with the diffuse-wall
    sums taken from the full set at the wall points only, equals the full
    oracle on that subset (velocities are independent in the FR operator)."""
    from frfs_b200.mesh import ElementGeometry, StructuredMesh
    from oracle.fr import FROracle
    g = np.load(os.path.join(GOLD, 'shapes_quad_p2.npz'))
    geo = ElementGeometry(StructuredMesh((3, 2), (0.0, -0.5), (1.0, 0.5), periodic='x'), 2)
    c0 = np.linspace(-3, 3, 6)
    N = len(c0)
    idx = np.arange(N**3)
    cv = np.stack([c0[idx // (N * N)], c0[(idx // N) % N], c0[idx % N]])
    fw = np.exp(-np.sum(cv**2, axis=0))
    walls = [(np.array([-0.3, 0, 0]), fw, 'dgfs-wall-diffuse'),
             (np.array([0.3, 0, 0]), fw, 'dgfs-wall-diffuse')]
    nw = len(geo.wall_fpts)
    bcid = np.asarray(geo.wall_bcid)
    assert set(bcid.tolist()) == {0, 1}
    orc = FROracle({'M0': g['M0'], 'M132': g['M132'], 'M3': g['M3']}, geo, c0, 0.1, walls,
                   bcid=bcid)
    rng = np.random.default_rng(1)
    u = fw[None, None, :] * (1 + 0.2 * rng.uniform(size=(geo.smats.shape[0], 9, N**3)))
    assert nw > 0
    bc_full = orc.update_bc(orc.disu(u))
    bc_state = orc.update_bc_from_state(u)
    assert np.allclose(bc_full, bc_state, rtol=1e-14, atol=0)
    vsel = np.sort(rng.choice(N**3, size=40, replace=False))
    L_full = orc.rhs(u)
    L_sub = orc.restrict(vsel).rhs(u[:, :, vsel], bc=bc_state)
    assert np.allclose(L_sub, L_full[:, :, vsel], rtol=1e-13, atol=1e-14 * np.abs(L_full).max())


@pytest.mark.parametrize('tag', ['nv16', 'nv24'])
def test_oracle_q_equals_reference_kernels(tag):
    """The oracle's Q against the reference's own vhs-gll CUDA kernels and
    cuFFT (frfs/solvers/dgfs/kernels/scattering/vhs-gll.mako rendered,
    driven in the order of frfs/solvers/dgfs/scattering.py:227-286; golden
    vectors written by tests/golden/make_reference_q.py on a GPU)."""
    from oracle.ref_vhs.build import GRIDS, grid_tables
    d = np.load(os.path.join(GOLD, f'reference_q_{tag}.npz'))
    g = GRIDS[tag]
    assert int(d['Nv']) == g['Nv'] and int(d['M']) == g['M'] and int(d['Nrho']) == g['Nrho']
    vm, _, _ = grid_tables(g)
    orc = VHSOracle(vm, g['omega'], 4.17e-10, 273.0)
    Qo = np.stack([orc.Q(f) for f in d['f']])
    assert rel_l2(Qo, d['Q']) < 1e-12


def test_oracle_mixture_q_equals_reference_kernels():
    """The mixture oracle's Q_p = sum_q Q_pq against the reference's own
    vss-gll CUDA kernels and cuFFT (frfs/solvers/dgfsbi/kernels/scattering/
    vss-gll.mako rendered, driven in the order of frfs/solvers/dgfsbi/
    scattering.py:256-330; golden vectors written by
    tests/golden/make_reference_q.py on a GPU): two species (argon, krypton),
    every pair VSS with alpha = 1.3, omega = 0.81, Nv = 16."""
    from oracle.ref_vss.build import GRIDS, grid_tables
    from oracle.vss import VSSOracle
    d = np.load(os.path.join(GOLD, 'reference_qbi_bi16.npz'))
    g = GRIDS['bi16']
    assert int(d['Nv']) == g['Nv'] and int(d['M']) == g['M'] and int(d['Mpre']) == g['Mpre']
    vm, szpre, pairs, _ = grid_tables(g)
    orc = VSSOracle(vm, szpre, pairs)
    Qo = np.stack([np.stack(orc.Q(list(f))) for f in d['f']])
    assert rel_l2(Qo, d['Q']) < 1e-12
    # each species' own Q too (the lighter species' Q is not swamped)
    for p in range(2):
        assert rel_l2(Qo[:, p], d['Q'][:, p]) < 1e-12


@pytest.mark.parametrize('kind,ndims,order', [('quad', 2, 2), ('quad', 2, 3), ('hex', 3, 2)])
def test_oracle_inverse_mass_equals_reference(kind, ndims, order):
    """The oracle's inverse mass matrix (the exact nodal mass matrix,
    inverted) equals the reference's own M12 = V^T V (golden fixture written
    from frfs/shapes.py:163-166)."""
    from oracle.fr import inverse_mass, invmass
    ref = np.load(os.path.join(GOLD, f'shapes_{kind}_p{order}.npz'))['M12']
    mine = inverse_mass(ndims, order)
    assert np.abs(mine - ref).max() < 1e-12 * np.abs(ref).max()
    u = np.random.default_rng(order).standard_normal((3, ref.shape[0], 7))
    assert np.allclose(invmass(mine, u), np.einsum('ij,ejv->eiv', ref, u), rtol=0, atol=1e-12)
