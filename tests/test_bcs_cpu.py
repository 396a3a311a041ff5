"""Host side of the boundary conditions other than the diffuse wall: the
.ini types map to kernel kinds and rows, specular walls to their mirror
axis, and the oracle's specular map is the reference's reflection."""
import numpy as np
import pytest
import torch

from frfs_b200 import _lib
from frfs_b200.mesh import ElementGeometry, StructuredMesh
from frfs_b200.system import DGFSBoundaries
from frfs_b200.velocitymesh import DGFSVelocityMesh

from helpers import bc_cfg
from test_host_structs import _CPUBackend

HEX = {'x-': 'dgfs-inlet', 'x+': 'dgfs-outlet', 'y-': 'dgfs-wall-specular',
       'y+': 'dgfs-wall-diffuse-cyl', 'z-': 'dgfs-wall-specular', 'z+': 'dgfs-vanish'}
QUAD = {'x-': 'dgfs-inlet-normalshock', 'x+': 'dgfs-wall-specular', 'y-': 'dgfs-wall-diffuse',
        'y+': 'dgfs-wall-specular'}


def _bounds(kind, bcs, Nv=16):
    cfg = bc_cfg(Nv, 2, bcs)
    be = _CPUBackend()
    vm = DGFSVelocityMesh(be, cfg)
    if kind == 'quad':
        mesh = StructuredMesh((3, 2), (0.0, -0.5), (1.0, 0.5))
    else:
        mesh = StructuredMesh((2, 2, 2), (0.0, -0.5, 0.0), (1.0, 0.5, 1.0))
    geo = ElementGeometry(mesh, 2)
    return vm, geo, DGFSBoundaries(be, geo, vm, cfg, geo.wall_names)


def test_kinds_rows_and_points():
    vm, geo, b = _bounds('hex', HEX)
    kinds = b.kind.numpy()
    types = dict(zip(geo.wall_names, [bc.type for bc in b.bcs]))
    assert types == HEX
    # one row per face point for the cyl wall, one per other boundary
    ncyl = int(np.sum(geo.wall_bcid == geo.wall_names.index('y+')))
    assert len(kinds) == 5 + ncyl
    rows = b.row_of_point
    for bid, name in enumerate(geo.wall_names):
        k = set(kinds[rows[geo.wall_bcid == bid]])
        want = {'dgfs-inlet': _lib.BC_INLET, 'dgfs-outlet': _lib.BC_OUTLET,
                'dgfs-vanish': _lib.BC_INLET, 'dgfs-wall-diffuse-cyl': _lib.BC_DIFFUSE}.get(HEX[name])
        if HEX[name] == 'dgfs-wall-specular':
            want = _lib.BC_SPECULAR_Y if name == 'y-' else _lib.BC_SPECULAR_Z
        assert k == {want}, name
    assert b.kinds_used == sum(1 << k for k in set(kinds))
    assert b.has_diffuse
    # vanish: zero ghost distribution and U = 0; inlet: its Maxwellian and U
    fw, uw = b.fw.numpy(), b.uwall.numpy()
    iv = rows[geo.wall_bcid == geo.wall_names.index('z+')][0]
    assert not fw[iv].any() and not uw[iv].any()
    ii = rows[geo.wall_bcid == geo.wall_names.index('x-')][0]
    assert uw[ii][0] == pytest.approx(0.2) and fw[ii].sum() * vm.cw() == pytest.approx(1.1, rel=1e-4)


def test_cyl_rows_follow_the_expressions():
    vm, geo, b = _bounds('hex', HEX)
    bid = geo.wall_names.index('y+')
    pts = np.nonzero(geo.wall_bcid == bid)[0]
    cv = vm.cv()
    for w in pts[:5]:
        e, f = geo.wall_fpts[w]
        x, y, _ = geo.plocfpts[e, f]
        U = np.array([0.1 * (1 + y), 0.0, 0.05 * abs(x - 0.5)])
        T = 1.0 + 0.2 * (x < 0.5) * x
        r = b.row_of_point[w]
        assert np.allclose(b.uwall[r].numpy(), U, rtol=1e-6, atol=1e-7)
        want = np.exp(-np.sum((cv - U[:, None])**2, axis=0) / T)
        assert np.allclose(b.fw[r].numpy(), want, rtol=1e-5, atol=1e-7)


def test_quad_specular_axes_and_no_bc_update_without_diffuse():
    vm, geo, b = _bounds('quad', QUAD)
    kinds = b.kind.numpy()[b.row_of_point]
    for bid, name in enumerate(geo.wall_names):
        k = set(kinds[geo.wall_bcid == bid])
        if name == 'x+':
            assert k == {_lib.BC_SPECULAR_X}
        if name == 'y+':
            assert k == {_lib.BC_SPECULAR_Y}
    _, _, b2 = _bounds('quad', {'x-': 'dgfs-inlet', 'x+': 'dgfs-outlet',
                                'y-': 'dgfs-wall-specular', 'y+': 'dgfs-vanish'})
    assert not b2.has_diffuse


def test_unknown_type_raises():
    with pytest.raises(ValueError, match='unsupported boundary condition'):
        _bounds('quad', {'x-': 'dgfs-inlet', 'x+': 'dgfs-outlet', 'y-': 'dgfs-wall-nothing',
                         'y+': 'dgfs-vanish'})


def test_oracle_mirror_is_the_reflection():
    """The oracle's specular index map (nearest grid velocity to c - 2 (c.n) n)
    is an involution that flips one component for axis normals, and maps an
    oblique normal's reflection to the nearest grid point."""
    from oracle.fr import FROracle
    Nv = 8
    c0 = np.linspace(-5 + 5 / Nv, 5 - 5 / Nv, Nv)

    class G:
        smats = np.zeros((1, 1, 2, 2))
        wall_bcid = np.zeros(0, dtype=int)
    o = FROracle({'M0': None, 'M132': None, 'M3': None}, G, c0, 1.0)
    idx = np.arange(Nv**3)
    ix, iy, iz = idx // (Nv * Nv), (idx // Nv) % Nv, idx % Nv
    m = o.mirror(np.array([0.0, -1.0]))
    assert np.array_equal(m, (ix * Nv + (Nv - 1 - iy)) * Nv + iz)
    assert np.array_equal(m[m], idx)
    m = o.mirror(np.array([1.0, 0.0, 0.0]))
    assert np.array_equal(m, ((Nv - 1 - ix) * Nv + iy) * Nv + iz)
    n = np.array([0.6, 0.8])
    m = o.mirror(n)
    cr = o.cv[:2] - 2 * (n @ o.cv[:2]) * n[:, None]
    cr = np.clip(cr, c0[0], c0[-1])         # reflections off the grid: its nearest edge
    assert np.all(np.abs(o.cv[:2, m] - cr) <= (c0[1] - c0[0]) / 2 + 1e-12)


def test_npeval_and_expression_initial_condition_fields():
    from frfs_b200.initcond import DGFSMaxwellianExprInitCondition
    from frfs_b200.util import npeval
    x = np.linspace(0.0, 1.0, 5)
    assert np.allclose(npeval('2 + (x < 0.5)*x + pow(x, 2)', {'x': x}), 2 + (x < 0.5) * x + x**2)
    for bad in ('x**2', 'x.__class__', 'x; y', "__import__('os')"):
        with pytest.raises(ValueError):
            npeval(bad, {'x': x})
    cfg = bc_cfg(16, 2, QUAD)
    u0 = np.sqrt(2 * 8.3144598 / 39.96e-3 * 273.0)
    cfg.set('constants', 'rl', '0.00011140244750324529')
    for k, v in (('type', 'maxwellianExpr'), ('rho', 'rl*(1 + 0.1*sin(2*pi*x))'),
                 ('ux', f'{0.1 * u0}*y'), ('uy', '0'), ('uz', '0'), ('T', '273*(1 + 0.05*x)')):
        cfg.set('soln-ics', k, v)
    vm = DGFSVelocityMesh(_CPUBackend(), cfg)
    ic = DGFSMaxwellianExprInitCondition(_CPUBackend(), cfg, vm, 'soln-ics')
    with pytest.raises(ValueError):
        ic.get_init_vals()
    p = np.array([[0.25, 0.5], [0.75, -0.5]])
    rho, ux, uy, uz, T = ic.fields(p)
    assert np.allclose(rho, [1.1, 0.9]) and np.allclose(ux, [0.05, -0.05])
    assert np.allclose(T, [1.0125, 1.0375]) and not uy.any() and not uz.any()
