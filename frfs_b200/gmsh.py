"""Gmsh 2.2 ASCII meshes of affine quads (2-D) or hexes (3-D).

Reads what the reference's ``GmshReader`` reads (frfs/readers/gmsh.py:31-204)
and applies its conventions:

* sections ``$MeshFormat`` (version 2.2, ASCII, 8-byte reals),
  ``$PhysicalNames``, ``$Nodes`` and ``$Elements`` are required, any other
  section is skipped;
* the physical group named ``fluid`` holds the volume elements; groups
  named ``periodic_<id>_l`` / ``periodic_<id>_r`` (separators ' ', '_' or
  '-') hold the two sides of a periodic boundary, in pairs; every other
  named group is a boundary whose name selects ``[soln-bcs-<name>]``
  (names are lower-cased);
* an element's physical group is its first tag.

The elements must be first-order quads (Gmsh type 3) or hexes (type 5)
whose maps are affine (parallelepipeds), as ``ElementGeometry`` requires.
Corners are reordered from Gmsh's counter-clockwise numbering to the
tensor-product order of the solver (corner c has reference coordinate
r_i = -1 + 2 bit_i(c)), so the faces follow ``reference_faces``.  Faces are
matched between elements by their corner node sets; the two sides of a
periodic boundary by their centroids, after removing the translation
between the sides.
"""
import re
from collections import defaultdict

import numpy as np

from .mesh import reference_faces

# Gmsh element type -> (kind, corner count)
_ETYPES = {1: ('line', 2), 3: ('quad', 4), 5: ('hex', 8)}
# Gmsh corner index of each tensor-product corner (bit i of the index = r_i)
_CORNER_ORDER = {'quad': [0, 1, 3, 2], 'hex': [0, 1, 3, 2, 4, 5, 7, 6]}


def _section(lines, name):
    """The body lines of one counted section ($<name> ... $End<name>)."""
    n = int(next(lines).strip())
    body = [next(lines).strip() for _ in range(n)]
    end = next(lines).strip()
    if end != f'$End{name}':
        raise ValueError(f'Expected $End{name}')
    return body


class GmshMesh:
    """A mesh for ``ElementGeometry`` from a Gmsh 2.2 ASCII file (a path or
    an iterable of lines): ``eles`` (2^d, neles, d) corner coordinates,
    ``interfaces()`` (internal and periodic face pairs, named boundary
    faces), ``pair_shift`` (the periodic translations)."""

    def __init__(self, msh):
        if isinstance(msh, str):
            with open(msh) as fh:
                lines = fh.read().splitlines()
        else:
            lines = [l.rstrip('\n') for l in msh]
        it = iter([l for l in lines if l.strip()])
        seen = set()
        for l in it:
            l = l.strip()
            if not l.startswith('$'):
                raise ValueError('Expected a mesh section')
            name = l[1:]
            if name == 'MeshFormat':
                ver, ftype, dsize = next(it).split()
                if ver != '2.2':
                    raise ValueError('Invalid mesh version')
                if ftype != '0':
                    raise ValueError('Invalid file type')
                if dsize != '8':
                    raise ValueError('Invalid data size')
                if next(it).strip() != '$EndMeshFormat':
                    raise ValueError('Expected $EndMeshFormat')
            elif name == 'PhysicalNames':
                self._read_names(_section(it, name))
            elif name == 'Nodes':
                self._nodes = {int(v[0]): np.array([float(x) for x in v[1:4]])
                               for v in (b.split() for b in _section(it, name))}
            elif name == 'Elements':
                self._read_eles(_section(it, name))
            else:
                for el in it:
                    if el.strip() == f'$End{name}':
                        break
                else:
                    raise ValueError(f'Expected $End{name}')
                continue
            seen.add(name)
        missing = {'MeshFormat', 'PhysicalNames', 'Nodes', 'Elements'} - seen
        if missing:
            raise ValueError(f'Required sections: {sorted(missing)} not found')
        self._build()

    def _read_names(self, body):
        self._fluid, self._bnd, self._per = None, {}, defaultdict(dict)
        seen = set()
        for l in body:
            m = re.match(r'(\d+) (\d+) "((?:[^"\\]|\\.)*)"$', l)
            if not m:
                raise ValueError('Malformed physical entity')
            pent, name = int(m.group(2)), m.group(3).lower()
            if name in seen:
                raise ValueError(f'Duplicate physical name: {name}')
            seen.add(name)
            if name == 'fluid':
                self._fluid = pent
            elif name.startswith('periodic'):
                p = re.match(r'periodic[ _-]([a-z0-9]+)[ _-](l|r)$', name)
                if not p:
                    raise ValueError('Invalid periodic boundary condition')
                self._per[p.group(1)][p.group(2)] = pent
            else:
                self._bnd[name] = pent
        if self._fluid is None:
            raise ValueError('No fluid elements in mesh')
        if any(len(v) != 2 for v in self._per.values()):
            raise ValueError('Unpaired periodic boundary in mesh')

    def _read_eles(self, body):
        self._elenodes = defaultdict(list)
        for l in body:
            v = [int(x) for x in l.split()]
            etype, ntags = v[1], v[2]
            if etype not in _ETYPES:
                raise ValueError(f'Unsupported element type {etype}')
            nodes = v[3 + ntags:]
            if len(nodes) != _ETYPES[etype][1]:
                raise ValueError('Malformed element')
            self._elenodes[(_ETYPES[etype][0], v[3])].append(nodes)

    def _build(self):
        kinds = {k for (k, pent) in self._elenodes if pent == self._fluid}
        if len(kinds) != 1 or kinds <= {'line'}:
            raise ValueError('the fluid group must hold quads or hexes of one kind')
        self.etype = kinds.pop()
        if self.etype not in _CORNER_ORDER:
            raise ValueError(f'unsupported fluid element {self.etype}')
        d = self.ndims = 2 if self.etype == 'quad' else 3
        order = _CORNER_ORDER[self.etype]
        conn = np.array(self._elenodes[(self.etype, self._fluid)])[:, order]   # (E, 2^d)
        self.neles = len(conn)
        self.corner_nodes = conn
        self.eles = np.stack([np.stack([self._nodes[n][:d] for n in row]) for row in conn], axis=1)
        ext = np.abs(self.eles - self.eles[0][None]).max(axis=(0, 1))
        self.h = np.where(ext > 0, ext, 1.0)
        faces = reference_faces(d)
        fmap = {}
        for e, row in enumerate(conn):
            for f, (a, s) in enumerate(faces):
                key = frozenset(int(row[c]) for c in range(2**d) if ((c >> a) & 1) == (s > 0))
                fmap.setdefault(key, []).append((e, f))
        fkind = 'line' if d == 2 else 'quad'
        bnd_faces = lambda pent: [frozenset(n) for n in self._elenodes.get((fkind, pent), [])]
        self._pairs, self._bcs, self._shift = [], {}, {}
        used = set()
        for key, ef in fmap.items():
            if len(ef) == 2:
                self._pairs.append((ef[0], ef[1]))
                used.add(key)
            elif len(ef) > 2:
                raise ValueError('a face is shared by more than two elements')
        centroid = lambda key: np.mean([self._nodes[n][:d] for n in key], axis=0)
        for pid, lr in sorted(self._per.items()):
            L, R = bnd_faces(lr['l']), bnd_faces(lr['r'])
            if len(L) != len(R) or not L:
                raise ValueError(f'periodic boundary {pid}: sides do not match')
            cl = np.array([centroid(k) for k in L])
            cr = np.array([centroid(k) for k in R])
            t = cr.mean(axis=0) - cl.mean(axis=0)      # translation l -> r
            tol = 1e-8 * float(self.h.max())
            for i, kl in enumerate(L):
                j = int(np.argmin(np.abs(cr - (cl[i] + t)).max(axis=1)))
                if np.abs(cr[j] - (cl[i] + t)).max() > tol:
                    raise ValueError(f'periodic boundary {pid}: no partner face')
                kr = R[j]
                if kl not in fmap or kr not in fmap:
                    raise ValueError(f'periodic boundary {pid}: face not on an element')
                a, b = fmap[kl][0], fmap[kr][0]
                self._pairs.append((b, a))
                self._shift[(b, a)] = t                # r-side location minus l-side
                used.update((kl, kr))
        for name, pent in sorted(self._bnd.items()):
            lst = []
            for k in bnd_faces(pent):
                if k not in fmap:
                    raise ValueError(f'boundary {name}: face not on an element')
                lst.append(fmap[k][0])
                used.add(k)
            if lst:
                self._bcs[name] = lst
        if set(fmap) - used:
            raise ValueError('boundary faces without a physical group')

    def faces(self):
        return reference_faces(self.ndims)

    def interfaces(self):
        """Internal and periodic pairs [((e, f), (e', f'))] and boundaries
        {name: [(e, f)]}."""
        return list(self._pairs), {k: list(v) for k, v in self._bcs.items()}

    def pair_shift(self, e, f, e2, f2):
        """Location of face (e, f) minus that of its partner: the periodic
        translation, else zero."""
        return np.asarray(self._shift.get(((e, f), (e2, f2)), np.zeros(self.ndims)))


def read_mesh(path):
    """The reference's mesh import for this path: a Gmsh 2.2 ASCII file."""
    return GmshMesh(path)


def write_msh(mesh, fh, periodic_names=None):
    """Write a ``StructuredMesh`` as Gmsh 2.2 ASCII (corner nodes shared
    between elements, boundaries as named groups, periodic axes as
    periodic_<axis>_l / _r groups).  Used to exchange the in-memory box
    meshes with Gmsh-based tools."""
    d = mesh.ndims
    axes = 'xyz'
    nodes, nid = {}, {}

    def node(x):
        k = tuple(np.round(np.asarray(x) / mesh.h * 2).astype(np.int64))
        if k not in nid:
            nid[k] = len(nid) + 1
            nodes[nid[k]] = x
        return nid[k]
    # gmsh corner slot order[c] holds tensor corner c
    inv = np.argsort(_CORNER_ORDER[mesh.etype])
    vols = []
    for e in range(mesh.neles):
        ids = [node(mesh.eles[c, e]) for c in range(2**d)]
        vols.append([ids[inv[k]] for k in range(2**d)])
    groups = {'fluid': 1}
    faces_by_group = defaultdict(list)
    fl = reference_faces(d)
    for e, c in enumerate(mesh.cells):
        for f, (a, s) in enumerate(fl):
            edge = (s > 0 and c[a] == mesh.shape[a] - 1) or (s < 0 and c[a] == 0)
            if not edge:
                continue
            side = axes[a] + ('+' if s > 0 else '-')
            if axes[a] in mesh.periodic:
                g = f"periodic_{axes[a]}_{'r' if s > 0 else 'l'}"
            else:
                g = mesh.bcnames.get(side, side)
            cs = [cc for cc in range(2**d) if ((cc >> a) & 1) == (s > 0)]
            ids = [node(mesh.eles[cc, e]) for cc in cs]
            if d == 2:
                faces_by_group[g].append(ids)
            else:                                     # counter-clockwise quad
                faces_by_group[g].append([ids[0], ids[1], ids[3], ids[2]])
    for g in sorted(faces_by_group):
        groups.setdefault(g, len(groups) + 1)
    w = fh.write
    w('$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$PhysicalNames\n')
    w(f'{len(groups)}\n')
    for g, pid in groups.items():
        w(f'{d if g == "fluid" else d - 1} {pid} "{g}"\n')
    w('$EndPhysicalNames\n$Nodes\n')
    w(f'{len(nodes)}\n')
    for i in sorted(nodes):
        x = [float(v) for v in nodes[i]] + [0.0] * (3 - d)
        w(f'{i} {x[0]!r} {x[1]!r} {x[2]!r}\n')
    w('$EndNodes\n$Elements\n')
    lst = []
    ft = 1 if d == 2 else 3
    for g in sorted(faces_by_group):
        for ids in faces_by_group[g]:
            lst.append((ft, groups[g], ids))
    vt = 3 if d == 2 else 5
    for ids in vols:
        lst.append((vt, 1, ids))
    w(f'{len(lst)}\n')
    for i, (t, g, ids) in enumerate(lst):
        w(f"{i + 1} {t} 2 {g} {g} {' '.join(map(str, ids))}\n")
    w('$EndElements\n')
