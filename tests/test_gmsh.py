"""Gmsh 2.2 mesh import (frfs/readers/gmsh.py conventions): a box written as
.msh and read back gives the same geometry and connectivity as the
in-memory mesh, including periodic pairs; malformed files are refused."""
import io

import numpy as np
import pytest

from frfs_b200.gmsh import GmshMesh, write_msh
from frfs_b200.mesh import ElementGeometry, StructuredMesh


def _roundtrip(mesh):
    buf = io.StringIO()
    write_msh(mesh, buf)
    return GmshMesh(io.StringIO(buf.getvalue()).readlines()), buf.getvalue()


def _same_geometry(a, b):
    assert np.allclose(a.smats, b.smats, rtol=0, atol=1e-13)
    assert np.allclose(a.rcpdjac, b.rcpdjac, rtol=1e-13)
    assert np.allclose(a.norm_pnorm, b.norm_pnorm, atol=1e-13)
    assert np.array_equal(a.nbr >= 0, b.nbr >= 0)
    inner = a.nbr >= 0
    assert np.array_equal(a.nbr[inner], b.nbr[inner])
    assert a.wall_names == b.wall_names
    # the same wall points (their order follows the face lists)
    key = lambda g: sorted(map(tuple, g.wall_fpts.tolist()))
    assert key(a) == key(b)
    for name in a.wall_names:
        assert sorted(map(tuple, a.bc_fpts[name].tolist())) == sorted(map(tuple, b.bc_fpts[name].tolist()))


@pytest.mark.parametrize('shape,lo,hi,periodic,order', [
    ((3, 2), (0.0, -0.5), (1.0, 0.5), 'x', 3),
    ((4, 3), (0.0, 0.0), (2.0, 1.0), '', 2),
    ((2, 2, 2), (0.0, -0.5, 0.0), (1.0, 0.5, 1.0), 'xz', 2),
    ((2, 3, 2), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), '', 2)])
def test_roundtrip_matches_structured(shape, lo, hi, periodic, order):
    m = StructuredMesh(shape, lo, hi, periodic=periodic)
    g, _ = _roundtrip(m)
    assert g.etype == m.etype and g.neles == m.neles
    assert np.allclose(g.eles, m.eles)
    _same_geometry(ElementGeometry(g, order), ElementGeometry(m, order))


def test_named_boundaries_and_sections():
    m = StructuredMesh((2, 2), (0.0, 0.0), (1.0, 1.0), bcnames={'y+': 'lid', 'y-': 'wall',
                                                                 'x-': 'wall2', 'x+': 'wall3'})
    g, text = _roundtrip(m)
    assert sorted(g.interfaces()[1]) == ['lid', 'wall', 'wall2', 'wall3']
    # unknown sections are skipped, the physical names are case-insensitive
    text2 = text.replace('"lid"', '"LID"').replace('$Nodes', '$Comments\nanything\n$EndComments\n$Nodes')
    g2 = GmshMesh(io.StringIO(text2).readlines())
    assert 'lid' in g2.interfaces()[1]


def test_affine_sheared_mesh():
    """A parallelogram mesh (affine, not axis-aligned) reads and gives
    positive Jacobians and unit normals."""
    m = StructuredMesh((3, 2), (0.0, 0.0), (1.0, 1.0))
    g, text = _roundtrip(m)
    lines = text.splitlines()
    i0 = lines.index('$Nodes') + 2
    n = int(lines[i0 - 1])
    for k in range(i0, i0 + n):
        v = lines[k].split()
        x, y = float(v[1]), float(v[2])
        lines[k] = f'{v[0]} {x + 0.3 * y!r} {1.2 * y!r} 0.0'
    geo = ElementGeometry(GmshMesh(lines), 2)
    assert np.all(geo.djac > 0)
    assert np.allclose(np.linalg.norm(geo.norm_pnorm, axis=-1), 1.0)


@pytest.mark.parametrize('edit,msg', [
    (lambda t: t.replace('2.2 0 8', '4.1 0 8'), 'version'),
    (lambda t: t.replace('"fluid"', '"air"'), 'fluid'),
    (lambda t: t.replace('"periodic_x_r"', '"periodic_y_r"'), 'Unpaired'),
    (lambda t: t.replace('$PhysicalNames', '$Foo').replace('$EndPhysicalNames', '$EndFoo'), 'Required'),
])
def test_malformed_files_are_refused(edit, msg):
    m = StructuredMesh((2, 2), (0.0, -0.5), (1.0, 0.5), periodic='x')
    _, text = _roundtrip(m)
    with pytest.raises(ValueError, match=msg):
        GmshMesh(io.StringIO(edit(text)).readlines())
