"""Gas mixtures on the host: the 'vss-gll' model's mesh, parameters and
kernel tables against the oracle, and the oracle's own properties."""
import numpy as np
import pytest

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
