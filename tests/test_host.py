"""Product host-side precompute against the reference's own outputs
(golden fixtures) and host logic (mesh connectivity, configs)."""
import os

import numpy as np
import pytest

from frfs_b200.inifile import Inifile
from frfs_b200.mesh import ElementGeometry, StructuredMesh
from frfs_b200.quadratures import gauss_jacobi, gll_points, gll_weights
from frfs_b200.scattering import gram_inverse, vhs_prefactor, vhs_tables
from frfs_b200.shapes import TensorShape
from frfs_b200.sphericaldesign import half_sphere_design
from frfs_b200.velocitymesh import DGFSVelocityMesh

from helpers import vhs_cfg

GOLD = os.path.join(os.path.dirname(__file__), 'golden')


@pytest.mark.parametrize('kind,order', [('quad', 2), ('quad', 3), ('hex', 2)])
def test_operator_matrices_match_reference(kind, order):
    g = np.load(f'{GOLD}/shapes_{kind}_p{order}.npz')
    s = TensorShape(kind, order)
    assert np.allclose(s.upts, g['upts'], atol=1e-15)
    assert np.allclose(s.fpts, g['fpts'], atol=1e-15)
    for m in ('M0', 'M1', 'M2', 'M3', 'M12'):
        assert np.allclose(s.opmat(m), g[m], atol=1e-13), m
    for k in g.files:
        if k.startswith('interp_from_p'):
            assert np.allclose(s.interp_from(int(k[len('interp_from_p'):])), g[k], atol=1e-14), k
    assert np.allclose(s.opmat('M1 - M3*M2'), g['M132'], atol=1e-13)
    assert np.array_equal(s.norm_fpts, g['norm_fpts'])


class _Mesh:
    """An arbitrary affine element set (the golden metrics mesh)."""

    def __init__(self, eles):
        self.eles = eles
        self.ndims = eles.shape[2]
        self.neles = eles.shape[1]
        self.etype = 'quad' if self.ndims == 2 else 'hex'
        self.h = np.ones(self.ndims)


@pytest.mark.parametrize('kind,order', [('quad', 2), ('quad', 3), ('hex', 2)])
def test_affine_metrics_match_reference(kind, order, monkeypatch):
    g = np.load(f'{GOLD}/metrics_{kind}_p{order}.npz')
    monkeypatch.setattr(ElementGeometry, '_connect', lambda self: None)
    geo = ElementGeometry(_Mesh(g['eles']), order)
    # reference layout smats (ndims, nupts, ndims, neles) -> ours [e][u][i][k]
    ref = np.transpose(g['smats'], (3, 1, 0, 2))
    assert np.allclose(geo.smats, ref, atol=1e-13)
    assert np.allclose(geo.rcpdjac, g['rcpdjac'].T, rtol=1e-12)
    assert np.allclose(geo.norm_pnorm, np.transpose(g['norm_pnorm_fpts'], (1, 0, 2)), atol=1e-13)
    assert np.allclose(geo.mag_pnorm, g['mag_pnorm_fpts'].T, rtol=1e-12)
    assert np.allclose(geo.plocfpts, np.transpose(g['plocfpts'], (1, 0, 2)), atol=1e-13)


@pytest.mark.parametrize('name,dev', [('c1', 5), ('nv8', 5), ('m16', 6)])
def test_velocity_mesh_matches_reference(name, dev):
    g = np.load(f'{GOLD}/vmesh_{name}.npz')
    M = int(g['M'])
    if M not in (1, 3, 6, 12):
        pytest.skip('design not built in (file input)')
    cfg = vhs_cfg(int(g['Nv']), int(g['Nrho']), M, dev)
    vm = DGFSVelocityMesh(None, cfg)
    assert np.array_equal(vm.cv(), g['cv'])
    assert vm.cw() == float(g['cw']) and vm.L() == float(g['L'])
    assert np.allclose(vm.qz(), g['qz'], atol=1e-14) and np.allclose(vm.qw(), g['qw'], atol=1e-14)
    assert vm.sw() == float(g['sw'])


def test_design_file_input_matches_reference(tmp_path):
    d = np.load(f'{GOLD}/sphdesign.npz')
    p = tmp_path / 'ss32.txt'
    np.savetxt(p, d['pts32'])
    assert np.array_equal(half_sphere_design(16, str(p)), d['pts32'][:16])


def _axes(pts):
    """Set of axes {+s, -s} as a canonical sorted array."""
    out = []
    for s in pts:
        s = s / np.linalg.norm(s)
        k = np.argmax(np.abs(s) > 1e-12)
        out.append(s if s[k] > 0 else -s)
    out = np.array(out)
    return out[np.lexsort(np.round(out, 10).T[::-1])]


def test_builtin_designs():
    d = np.load(f'{GOLD}/sphdesign.npz')
    # M = 6: same axes as the reference's 12-point Womersley design
    assert np.allclose(_axes(half_sphere_design(6)), _axes(d['pts12'][:6]), atol=1e-12)
    # M = 12: the 24-point set is an exact spherical 5-design
    half = half_sphere_design(12)
    full = np.vstack([half, -half])
    from math import gamma
    for a in range(6):
        for b in range(6 - a):
            for c in range(6 - a - b):
                v = np.mean(full[:, 0]**a * full[:, 1]**b * full[:, 2]**c)
                ex = 0.0
                if not (a % 2 or b % 2 or c % 2):
                    ex = (2 * gamma((a + 1) / 2) * gamma((b + 1) / 2) * gamma((c + 1) / 2)
                          / gamma((a + b + c + 3) / 2) / (4 * np.pi))
                assert abs(v - ex) < 1e-14, (a, b, c)
    with pytest.raises(ValueError):
        half_sphere_design(7)


def test_quadratures():
    d = np.load(f'{GOLD}/sphdesign.npz')
    z, w = gauss_jacobi(8)
    assert np.allclose(z, d['gj8_z'], atol=1e-14) and np.allclose(w, d['gj8_w'], atol=1e-14)
    for n in (3, 4, 5):
        x, w = gll_points(n), gll_weights(n)
        assert np.isclose(w.sum(), 2.0)
        for k in range(2 * n - 2):                     # GLL exact to degree 2n-3
            assert np.isclose(np.dot(w, x**k), (1 - (-1)**(k + 1)) / (k + 1))


def test_vhs_tables_consistent_with_oracle():
    from oracle.velocitymesh import VelocityMesh
    from oracle.vhs import precompute
    g = np.load(f'{GOLD}/vmesh_nv8.npz')
    ovm = VelocityMesh(8, 4, g['sz'], cmax=0.0, Tmax=273.0, dev=5, T0=273.0, H0=1e-3,
                       rho0=0.00011140244750324529, molarMass0=39.96e-3)
    gam = 0.38
    aa, bb1, bb2 = precompute(ovm, gam)
    phase, gw, tb2 = vhs_tables(8, ovm.L, ovm.qz, ovm.qw, ovm.sz, ovm.sw, gam)
    N, n = 8, 512
    # phase factors multiply to exp(i a)
    l = np.arange(n)
    ix, iy, iz = l // 64, (l // 8) % 8, l % 8
    for p in range(4):
        for q in range(6):
            e = phase[p, q, 0, ix] * phase[p, q, 1, iy] * phase[p, q, 2, iz]
            assert np.allclose(e, np.exp(1j * aa[p * 6 + q]), atol=1e-13)
    # gw [p][kz][kx][ky] (kx <= N/2) = 2 qw sw / n * bb1 ; bb2 [kz][kx][ky]
    b1 = bb1.reshape(4, N, N, N)                       # [p][kx][ky][kz]
    for p in range(4):
        ref = (2 * ovm.qw[p] * ovm.sw / n) * np.transpose(b1[p], (2, 0, 1))[:, :N // 2 + 1, :]
        assert np.allclose(gw[p], ref, rtol=1e-13)
    assert np.allclose(tb2, np.transpose(bb2.reshape(N, N, N), (2, 0, 1)), rtol=1e-13)


def test_prefactor_mass_one_is_reference_formula():
    from oracle.velocitymesh import VelocityMesh
    from oracle.vhs import vhs_prefactor as ovp
    cfg = vhs_cfg(16, 8, 6, 5)
    vm = DGFSVelocityMesh(None, cfg)
    ovm = VelocityMesh(16, 8, vm.sz(), cmax=0.0, Tmax=273.0, dev=5, T0=273.0, H0=1e-3,
                       rho0=0.00011140244750324529, molarMass0=39.96e-3)
    assert np.allclose(vhs_prefactor(vm, 0.81, 4.17e-10, 273.0), ovp(ovm, 0.81, 4.17e-10, 273.0),
                       rtol=1e-14)


def test_gram_inverse():
    c0 = np.linspace(-5 + 5 / 8, 5 - 5 / 8, 8)
    G = gram_inverse(c0)
    cx, cy, cz = np.meshgrid(c0, c0, c0, indexing='ij')
    phi = np.stack([np.ones_like(cx), cx, cy, cz, cx**2 + cy**2 + cz**2]).reshape(5, -1)
    assert np.allclose(G @ (phi @ phi.T), np.eye(5), atol=1e-10)


@pytest.mark.parametrize('shape,periodic', [((3, 2), 'x'), ((4, 3), 'xy'), ((2, 2, 2), 'xz'),
                                            ((1, 2), 'x')])
def test_connectivity_pairs_coincide(shape, periodic):
    d = len(shape)
    lo, hi = (0.0,) * d, (1.0,) * d
    mesh = StructuredMesh(shape, lo, hi, periodic=periodic)
    g = ElementGeometry(mesh, 2)
    nf = g.nfpts
    seen = set()
    for e in range(g.neles):
        for f in range(nf):
            n = int(g.nbr[e, f])
            if n < 0:
                continue
            e2, f2 = divmod(n, nf)
            assert int(g.nbr[e2, f2]) == e * nf + f          # symmetric
            dx = g.plocfpts[e, f] - g.plocfpts[e2, f2]
            for a, ax in enumerate('xyz'[:d]):
                if ax in periodic:
                    dx[a] = (dx[a] + 0.5) % 1.0 - 0.5
            assert np.abs(dx).max() < 1e-12
            assert np.allclose(g.norm_pnorm[e, f], -g.norm_pnorm[e2, f2])
            seen.add((e, f))
    nwall = len(g.wall_fpts)
    assert len(seen) + nwall == g.neles * nf


def test_inifile_accessors():
    c = Inifile('[constants]\nNv = 24\nx0 = 2.5\n[a]\nb = Nv*x0 ; comment\n')
    assert c.getint('constants', 'Nv') == 24
    assert c.getfloat('a', 'missing', 3.0) == 3.0
    assert c.getexpr('a', 'b', subs=c.items('constants')) == '(24*2.5)'
    assert c.items_as('constants', float) == {'Nv': 24.0, 'x0': 2.5}
