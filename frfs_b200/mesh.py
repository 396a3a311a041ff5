"""Structured quad/hex meshes, affine metrics and flux-point connectivity.

Meshes come from ``StructuredMesh`` (boxes built in memory) or from a
Gmsh 2.2 file (``frfs_b200.gmsh.GmshMesh``); both give ElementGeometry:
``eles`` (nspts, neles, ndims) corner coordinates in the reference's
``std_ele(1)`` order (x fastest), internal interfaces (periodic pairs
included) and named boundary faces.

Metric terms follow frfs/solvers/base/elements.py:198-354 for affine
elements: smats = |J| J^{-1} (the 2-D adjugate / Kopriva's invariant form,
which coincide for affine maps), rcpdjac = 1/|J|, physical normals
pnorm = smats^T n_ref, with magnitude and unit direction (elements.py:
265-283).  Flux points of the two sides of an interface are paired by
sorting each side's physical locations (``_srtd_face_fpts``,
elements.py:107-112, with the periodic offset removed).
"""
import itertools as it

import numpy as np

from .shapes import TensorShape


def reference_faces(ndims):
    """Face index -> (axis, side) of the quad / hex in the reference's face
    order (the face of side s along axis a holds the corners whose bit a is
    (s > 0))."""
    if ndims == 2:
        return [(1, -1), (0, +1), (1, +1), (0, -1)]
    return [(2, -1), (1, -1), (0, +1), (1, +1), (0, -1), (2, +1)]


class StructuredMesh:
    """nx x ny (x nz) box of quads (hexes) on [x0,x1] x [y0,y1] (x [z0,z1]).

    ``periodic``: axes ('x', 'y', 'z') that wrap; every other side is a
    boundary named by ``bcnames`` (keys 'x-', 'x+', 'y-', ...).
    """

    def __init__(self, shape, lo, hi, periodic=(), bcnames=None):
        self.ndims = len(shape)
        self.shape = tuple(shape)
        self.lo, self.hi = np.asarray(lo, float), np.asarray(hi, float)
        self.periodic = set(periodic)
        self.h = (self.hi - self.lo) / np.asarray(shape)
        d = self.ndims
        self.etype = 'quad' if d == 2 else 'hex'
        ijk = list(it.product(*[range(n) for n in shape[::-1]]))
        self.cells = [c[::-1] for c in ijk]           # x fastest element order
        self.neles = len(self.cells)
        corners = np.array([p[::-1] for p in it.product((0.0, 1.0), repeat=d)])
        eles = np.empty((2**d, self.neles, d))
        for e, c in enumerate(self.cells):
            eles[:, e, :] = self.lo + (np.asarray(c) + corners) * self.h
        self.eles = eles
        self.bcnames = bcnames or {}

    def eidx(self, c):
        idx = 0
        for a in reversed(range(self.ndims)):
            idx = idx * self.shape[a] + c[a]
        return idx

    def faces(self):
        """Face index -> (axis, side) for the reference's face order."""
        return reference_faces(self.ndims)

    def pair_shift(self, e, f, e2, f2):
        """Location of face (e, f) minus that of its partner (e2, f2): the
        box length along the axis for a periodic pair, else zero."""
        a = self.faces()[f][0]
        shift = np.zeros(self.ndims)
        # periodic pair: the + side of the last cell meets the - side of cell 0
        if self.cells[e][a] == self.shape[a] - 1 and self.cells[e2][a] == 0:
            shift[a] = (self.hi - self.lo)[a]
        return shift

    def interfaces(self):
        """Internal pairs [((e, f), (e', f'))] and boundaries {name: [(e, f)]}."""
        fl = self.faces()
        lookup = {af: i for i, af in enumerate(fl)}
        pairs, bcs = [], {}
        axes = 'xyz'
        for e, c in enumerate(self.cells):
            for f, (a, s) in enumerate(fl):
                if s < 0:
                    continue                      # each pair once, from the + side
                nb = list(c)
                nb[a] += 1
                if nb[a] == self.shape[a]:
                    if axes[a] in self.periodic:
                        nb[a] = 0
                    else:
                        name = self.bcnames.get(axes[a] + '+', axes[a] + '+')
                        bcs.setdefault(name, []).append((e, f))
                        continue
                pairs.append(((e, f), (self.eidx(nb), lookup[(a, -1)])))
            for f, (a, s) in enumerate(fl):
                if s > 0 or c[a] != 0 or axes[a] in self.periodic:
                    continue
                name = self.bcnames.get(axes[a] + '-', axes[a] + '-')
                bcs.setdefault(name, []).append((e, f))
        return pairs, bcs


class ElementGeometry:
    """Operators, metrics and connectivity of one element type on a mesh."""

    def __init__(self, mesh, order):
        self.mesh = mesh
        self.shape = shp = TensorShape(mesh.etype, order)
        d, E = mesh.ndims, mesh.neles
        self.ndims, self.neles = d, E
        self.nupts, self.nfpts = shp.nupts, shp.nfpts
        corners = mesh.eles                             # (2^d, E, d)
        # affine map x = x0 + J (r + 1): J columns from corner differences
        x0 = corners[0]
        J = np.empty((E, d, d))                          # J[e][k][i] = dx_k/dr_i
        for i in range(d):
            J[:, :, i] = 0.5 * (corners[2**i] - x0)
        self._check_affine(corners, x0, J)
        det = np.linalg.det(J)
        if np.any(det < -1e-5):
            raise RuntimeError('Negative mesh Jacobians detected')
        Jinv = np.linalg.inv(J)                          # Jinv[e][i][k] = dr_i/dx_k
        sm = det[:, None, None] * Jinv                   # smats[e][i][k]
        self.smats = np.broadcast_to(sm[:, None], (E, self.nupts, d, d)).copy()
        self.rcpdjac = np.broadcast_to((1.0 / det)[:, None], (E, self.nupts)).copy()
        self.djac = 1.0 / self.rcpdjac
        # physical normals at flux points
        pn = np.einsum('eik,fi->efk', sm, shp.norm_fpts)  # (E, nfpts, d)
        mag = np.sqrt(np.einsum('efk,efk->ef', pn, pn))
        if np.any(mag < 1e-10):
            raise RuntimeError('Zero face normals detected')
        self.mag_pnorm = mag
        self.norm_pnorm = pn / mag[..., None]
        # physical flux-point locations
        self.plocfpts = x0[:, None, :] + np.einsum('eki,fi->efk', J, shp.fpts + 1.0)
        self.plocupts = x0[:, None, :] + np.einsum('eki,ui->euk', J, shp.upts + 1.0)
        self._connect()

    @staticmethod
    def _check_affine(corners, x0, J):
        d = J.shape[1]
        for c, r in enumerate(it.product((0.0, 2.0), repeat=d)):
            r = np.array(r[::-1])
            pred = x0 + np.einsum('eki,i->ek', J, r)
            if np.abs(pred - corners[c]).max() > 1e-9 * (1 + np.abs(corners).max()):
                raise ValueError('only affine (parallelepiped) elements are supported')

    def _sorted_face_fpts(self, e, f, shift=None):
        idx = self.shape.facefpts[f]
        pts = self.plocfpts[e, idx].copy()
        if shift is not None:
            pts -= shift
        key = np.round(pts / (np.abs(self.mesh.h).max() * 1e-9)).astype(np.int64)
        order = np.lexsort(key.T[::-1])
        return np.asarray(idx)[order]

    def _connect(self):
        mesh = self.mesh
        pairs, bcs = mesh.interfaces()
        E, nf = self.neles, self.nfpts
        nbr = np.full((E, nf), np.iinfo(np.int32).min, dtype=np.int64)
        for (e, f), (e2, f2) in pairs:
            shift = mesh.pair_shift(e, f, e2, f2)
            l = self._sorted_face_fpts(e, f)
            r = self._sorted_face_fpts(e2, f2, shift=-shift)
            nbr[e, l] = e2 * nf + r
            nbr[e2, r] = e * nf + l
        self.bc_fpts = {}
        wall = []
        for name, faces in sorted(bcs.items()):
            lst = []
            for e, f in faces:
                for fp in self._sorted_face_fpts(e, f):
                    lst.append((e, fp))
            self.bc_fpts[name] = np.array(lst, dtype=np.int64).reshape(-1, 2)
            wall.append((name, self.bc_fpts[name]))
        self.wall_names = [w[0] for w in wall]
        k = 0
        self.wall_fpts = []
        self.wall_bcid = []
        for bid, (name, lst) in enumerate(wall):
            for e, fp in lst:
                nbr[e, fp] = -1 - k
                self.wall_fpts.append((e, fp))
                self.wall_bcid.append(bid)
                k += 1
        self.wall_fpts = np.array(self.wall_fpts, dtype=np.int64).reshape(-1, 2)
        self.wall_bcid = np.array(self.wall_bcid, dtype=np.int64)
        if np.any(nbr == np.iinfo(np.int32).min):
            raise RuntimeError('unconnected flux points')
        self.nbr = nbr.astype(np.int32)
        self.ninterfpts = 2 * len(pairs) * (nf // (2 * mesh.ndims))
